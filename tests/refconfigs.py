"""Problems rebuilt from tests/golden/reference_configs.npz (the reference's
two shipped config files, parsed by tests/golden/make_reference_configs.py)."""
import os

import numpy as np

from demystification_dfn_b200.hdf5 import problem_from_tree

NPZ = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_configs.npz")


def tree(tag):
    z = np.load(NPZ, allow_pickle=False)
    out = {}
    for key in z.files:
        parts = key.split("/")
        if parts[0] != tag:
            continue
        d = out
        for p in parts[1:-1]:
            d = d.setdefault(p, {})
        v = z[key]
        d[parts[-1]] = str(v) if v.dtype.kind == "U" else (v[()] if v.ndim == 0 else v)
    return out


def problem(tag):
    return problem_from_tree(tree(tag))
