"""HDF5 config reader against the reference's shipped config files."""
import os

import numpy as np
import pytest

from demystification_dfn_b200 import build_arrays
from demystification_dfn_b200.hdf5 import read_config
import refconfigs

REF = "/root/reference/problems"


def test_golden_bp6_problem():
    p = refconfigs.problem("bp6")
    hp = p.hyperparameter
    assert (hp.fracture_mode, hp.static_kernel, hp.tol_solver, hp.max_it) == ("modeIII", "hmatrix", 1e-6, 30000)
    f = p.faults[0]
    assert f.nb_element == 4000 and f.node.shape == (2, 4001)
    assert np.allclose(np.diff(f.node[0]), 10.0)
    assert f.nb_source == 1 and int(f.index_injection[0]) == 2000 and f.Q[0] == 1.25e-6
    a = build_arrays(p)
    assert a.N == 4000 and a.fracture_mode == 3


def test_golden_network_problem():
    p = refconfigs.problem("network")
    assert p.nb_fault == 10
    assert [f.nb_element for f in p.faults] == [100, 100, 90, 130, 120, 70, 120, 80, 110, 100]
    a = build_arrays(p)
    assert a.N == 1020 + 9
    assert a.src_fault.tolist() == [10] and a.src_index.tolist() == [80]
    assert a.fracture_mode == 2


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference checkout not present")
def test_reader_matches_golden_on_shipped_files():
    for tag, rel in (("bp6", "BP6QD_A_4000"), ("network", "network_rate_strengthening")):
        p = read_config(os.path.join(REF, rel, "config"))
        q = refconfigs.problem(tag)
        a, b = build_arrays(p), build_arrays(q)
        for k in ("node", "a", "b", "V", "theta", "sigmaN", "P", "permeability", "src_Q"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k
