"""Generate tests/golden/reference_configs.npz from the reference's shipped inputs.

Reads problems/BP6QD_A_4000/config and problems/network_rate_strengthening/config
of the reference checkout (the only input files it ships; it ships no outputs)
with the package's HDF5 reader and stores every dataset as a flat array, so
that tests can rebuild the exact problems on machines without the reference.

Usage: python tests/golden/make_reference_configs.py REFERENCE_ROOT
(or with DFN_REFERENCE_ROOT set in the environment).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from demystification_dfn_b200.hdf5 import read_file  # noqa: E402

NAMES = {"bp6": "problems/BP6QD_A_4000/config", "network": "problems/network_rate_strengthening/config"}


def flatten(tree, prefix, out):
    for k, v in tree.items():
        key = f"{prefix}/{k}"
        if isinstance(v, dict):
            flatten(v, key, out)
        elif isinstance(v, str):
            out[key] = np.array(v)
        else:
            out[key] = np.asarray(v)


def main(ref_root):
    out = {}
    for tag, rel in NAMES.items():
        flatten(read_file(os.path.join(ref_root, rel)), tag, out)
    np.savez_compressed(os.path.join(HERE, "reference_configs.npz"), **out)
    print(f"wrote {len(out)} datasets")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DFN_REFERENCE_ROOT")
    if not root:
        raise SystemExit("usage: make_reference_configs.py REFERENCE_ROOT (or set DFN_REFERENCE_ROOT)")
    main(root)
