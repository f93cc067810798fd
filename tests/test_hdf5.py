"""HDF5 config reader against the reference's shipped config files."""
import os

import numpy as np
import pytest

from demystification_dfn_b200 import build_arrays
from demystification_dfn_b200.hdf5 import read_config
import refconfigs

# the reference checkout's problems/ folder, when the environment names a
# checkout (DFN_REFERENCE_ROOT); the golden fixture covers the other tests
_ROOT = os.environ.get("DFN_REFERENCE_ROOT", "")
REF = os.path.join(_ROOT, "problems") if _ROOT else ""


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


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="DFN_REFERENCE_ROOT does not name a reference checkout")
def test_reader_matches_golden_on_shipped_files():
    for tag, rel in (("bp6", "BP6QD_A_4000"), ("network", "network_rate_strengthening")):
        p = read_config(os.path.join(REF, rel, "config"))
        q = refconfigs.problem(tag)
        a, b = build_arrays(p), build_arrays(q)
        for k in ("node", "a", "b", "V", "theta", "sigmaN", "P", "permeability", "src_Q"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k


# --- writer -----------------------------------------------------------------

def _same_tree(a, b, path=""):
    assert set(a) == set(b), path
    for k in a:
        if isinstance(a[k], dict):
            _same_tree(a[k], b[k], path + k + "/")
            continue
        va, vb = np.asarray(a[k]), np.asarray(b[k])
        if va.dtype.kind in "OUS":
            assert str(a[k]) == str(b[k]), path + k
        else:
            assert va.dtype.kind == vb.dtype.kind, path + k
            assert np.array_equal(va.reshape(-1), vb.reshape(-1)), path + k


@pytest.mark.parametrize("tag", ["bp6", "network"])
def test_config_writer_round_trip_of_reference_configs(tmp_path, tag):
    """Problem from the shipped config -> DemystiFicatioN.write -> reader:
    the same datasets (names, groups, integer/float kinds, values)."""
    from demystification_dfn_b200.hdf5 import config_tree, read_file

    p = refconfigs.problem(tag)
    path = p.write(str(tmp_path) + "/case/")
    assert path.endswith("case/config") and os.path.exists(path)
    t = read_file(path)
    _same_tree(t, config_tree(p))
    # every dataset the reference's reader opens is present (configuration.f90:70-379)
    assert t["fault1"]["node"].shape == (p.faults[0].nb_node, 2)
    q = read_config(path)
    a, b = build_arrays(p), build_arrays(q)
    for k in ("node", "a", "b", "Dc", "V", "theta", "sigmaN", "P", "permeability", "src_Q", "src_index"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_config_writer_many_faults_uses_multilevel_group_btree(tmp_path):
    """800 faults: the root group has 802 links, more than one B-tree node of
    symbol-table nodes holds, so the group B-tree gets a second level."""
    from demystification_dfn_b200 import networks
    from demystification_dfn_b200.hdf5 import read_file

    p = networks.fault_network(n_faults=800, seed=0)
    path = p.write(str(tmp_path) + "/")
    t = read_file(path)
    assert len(t) == 802 and t["fault800"]["nb_element"] == p.faults[799].nb_element
    a, b = build_arrays(p), build_arrays(read_config(path))
    for k in ("node", "a", "b", "V", "theta", "P"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_output_writer_layout_and_stale_rows(tmp_path):
    """output%07d: six (nb_element, freq) fields and time (freq); a short
    last file keeps the previous file's rows past its own."""
    from demystification_dfn_b200.hdf5 import OUTPUT_FIELDS, read_file, read_output, write_output

    rng = np.random.default_rng(0)
    N, F = 7, 4
    snaps = [dict({k: rng.normal(size=N) for k in OUTPUT_FIELDS}, time=float(i)) for i in range(6)]
    ring = write_output(str(tmp_path / "output0000004"), snaps[:4], F, N)
    raw = read_file(str(tmp_path / "output0000004"))
    assert raw["V"].shape == (N, F) and raw["time"].shape == (F,)
    assert np.array_equal(raw["V"][:, 2], snaps[2]["V"])
    write_output(str(tmp_path / "output0000006"), snaps[4:], F, N, stale=ring)
    o = read_output(str(tmp_path / "output0000006"))
    assert np.array_equal(o["time"], [4.0, 5.0, 2.0, 3.0])
    assert np.array_equal(o["P"][1], snaps[5]["P"]) and np.array_equal(o["P"][3], snaps[3]["P"])
