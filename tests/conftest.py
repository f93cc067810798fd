import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdfn_b200.so")


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    from demystification_dfn_b200 import build, _lib

    build.build()
    return _lib.load()


@pytest.fixture(autouse=True)
def _skip_gpu_without_device(request):
    if request.node.get_closest_marker("gpu") and not gpu_available():
        pytest.skip("no CUDA device")
