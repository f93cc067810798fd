"""CPU tests of the host layer and of the C ABI library (no GPU calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from demystification_dfn_b200 import networks, build_arrays, DemystiFicatioN
from demystification_dfn_b200.layout import DfnOptions, DfnProblem, DfnReport

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_layout_fake_elements_and_nodes():
    p = networks.small_network(seed=0, n_faults=3)
    a = build_arrays(p)
    n = [f.nb_element for f in p.faults]
    assert a.N == sum(n) + 2
    first = a.fault_first
    assert list(first) == [0, n[0] + 1, n[0] + n[1] + 2]
    fk = a.fake_mask
    assert list(np.where(fk)[0]) == [n[0], n[0] + n[1] + 1]
    # fake elements carry the reader's presets and zero state
    assert np.all(a.a[fk] == 1) and np.all(a.V0[fk] == 1) and np.all(a.V[fk] == 0)
    assert np.all(a.permeability[fk] == 0)
    # nodes: fault f occupies node rows first_f .. first_f + n_f
    for f, s in zip(p.faults, first):
        assert np.array_equal(a.node[s:s + f.nb_element + 1], f.node.T)


def test_sources_are_one_based():
    p = networks.single_fault(n_el=100, length=1000.0)
    a = build_arrays(p)
    assert a.src_fault.tolist() == [1]
    assert 1 <= a.src_index[0] <= 100
    assert np.isclose(a.src_Q[0], 1.25e-6 * 50 / 50)


def test_network_is_seeded_and_gapped():
    p1 = networks.fault_network(n_faults=40, box=2000.0, seed=7)
    p2 = networks.fault_network(n_faults=40, box=2000.0, seed=7)
    assert all(np.array_equal(f.node, g.node) for f, g in zip(p1.faults, p2.faults))
    segs = np.array([[f.node[0, 0], f.node[1, 0], f.node[0, -1], f.node[1, -1]] for f in p1.faults])
    d = networks._seg_dist(segs[0, :2][None], segs[0, 2:][None], segs[1:, :2], segs[1:, 2:])
    assert d.min() >= 10.0


def test_problem_setters_reallocate():
    p = DemystiFicatioN(2)
    p.faults[0].nb_element = 7
    assert p.faults[0].a.shape == (7,) and p.faults[0].node.shape == (2, 8)
    p.faults[0].nb_source = 2
    assert p.faults[0].Q.shape == (2,) and p.faults[0].index_injection.dtype == np.int64
    with pytest.raises(ValueError):
        p.faults[0].nb_element = 0


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "dfn_b200.h")).read()
    return sorted(set(re.findall(r"\b(dfn_[A-Za-z0-9_]+)\s*\(", txt)) - {"dfn_status"})


def test_library_exports_every_header_symbol(lib):
    from demystification_dfn_b200.build import LIB

    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dfn_\w+)", out))
    missing = [f for f in _header_functions() if f not in exported]
    assert not missing, missing


def test_struct_layouts_match(lib):
    assert lib.dfn_problem_struct_size() == ctypes.sizeof(DfnProblem)
    assert lib.dfn_options_struct_size() == ctypes.sizeof(DfnOptions)
    assert lib.dfn_report_struct_size() == ctypes.sizeof(DfnReport)
    assert lib.dfn_abi_version() == 1
    assert lib.dfn_status_string(1).startswith(b"pressure CG")


def test_create_fails_loudly_without_gpu(lib):
    from conftest import gpu_available

    if gpu_available():
        pytest.skip("a GPU is present")
    from demystification_dfn_b200.simulation import Simulation
    from demystification_dfn_b200._lib import DfnError

    with pytest.raises(DfnError) as e:
        Simulation(networks.small_network(seed=0, n_faults=2))
    assert e.value.status == 6


def test_create_rejects_bad_problem(lib):
    from demystification_dfn_b200.layout import to_c

    a = build_arrays(networks.small_network(seed=0, n_faults=2))
    c = to_c(a)
    c.nb_element = a.N + 1       # inconsistent with the fault sizes
    h = ctypes.c_void_p()
    assert lib.dfn_create(ctypes.byref(c), None, ctypes.byref(h)) == 5
    assert b"nb_element" in lib.dfn_last_error()


def test_create_rejects_nonfinite_state(lib):
    """A NaN or Inf in the initial state is refused before any device work
    (DFN_ERR_NONFINITE), with or without a GPU."""
    import numpy as np
    from demystification_dfn_b200.layout import to_c

    for field, bad in (("V", np.nan), ("sigmaN", np.inf), ("P", -np.inf)):
        p = networks.small_network(seed=0, n_faults=2)
        getattr(p.faults[1], field)[3] = bad
        c = to_c(build_arrays(p))
        h = ctypes.c_void_p()
        assert lib.dfn_create(ctypes.byref(c), None, ctypes.byref(h)) == 4
        assert b"non-finite" in lib.dfn_last_error()


def test_tectonic_loading_and_crossing_pair_builders():
    """Network builders: v_load sets each fault's shear stressing rate to
    mu * v_load / L_f; crossing_pair shares exactly one node between its two
    faults (shift 0) and none when shifted."""
    import numpy as np

    p = networks.fault_network(n_faults=12, box=1500.0, seed=3, v_load=1e-9)
    mu = p.material_loading.mu
    for f in p.faults:
        L = float(np.hypot(*(f.node[:, -1] - f.node[:, 0])))
        assert np.allclose(f.shear_loading_dot, mu * 1e-9 / L, rtol=1e-9)
    q = networks.fault_network(n_faults=12, box=1500.0, seed=3)
    assert all(np.all(f.shear_loading_dot == 0.0) for f in q.faults)
    for shift, shared in ((0.0, 1), (1.0, 0)):
        c = networks.crossing_pair(n_el=20, shift=shift)
        a, b = c.faults[0].node.T, c.faults[1].node.T
        d = np.sqrt(((a[:, None, :] - b[None, :, :]) ** 2).sum(-1))
        assert int((d < 1e-9).sum()) == shared


def test_bench_summary_and_hmatrix_variants():
    """The bench line ends with a compact summary of the 64-network
    comparison, the shared-geometry batch and the H-matrix K.V fraction; the
    H-matrix variants of the comparison take their ACA tolerance and leaf
    size from their names."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
    import bench

    assert bench.hmat_eps("newton_hmat_fp32") == 1e-7
    assert bench.hmat_eps("newton_hmat_eps1e-6_fp32") == 1e-6
    assert bench.hmat_eps("newton_hmat_leaf96_eps1e-5_fp32") == 1e-5
    assert bench.hmat_leaf("newton_hmat_eps1e-5_fp32") == 64
    assert bench.hmat_leaf("newton_hmat_leaf128_eps1e-5_fp32") == 128
    extras = {
        "ensemble64": {"networks": 64,
                       "v_fp64": {"network_steps_per_s": 2790.123, "steps_per_s_vs_v_fp64": 1.0,
                                  "time_to_t_end_vs_v_fp64": 1.0, "kv_frac_of_measured_hbm": 1.0712},
                       "newton_hmat_fp32": {"network_steps_per_s": 9410.5, "steps_per_s_vs_v_fp64": 3.3812,
                                            "time_to_t_end_vs_v_fp64": 11.04, "slip_rel_err_vs_fp64": 3.7745e-07,
                                            "kv_frac_of_measured_hbm": 0.5192}},
        "tensor_core": {"tc_v": {"network_steps_per_s": 21800.4, "kv_avg_ms": 0.3797},
                        "tc_over_fp64_shared_v": {"network_steps_per_s": 6.7812, "time_to_t_end": 7.41}},
        "hmatrix": {"kv_frac_of_measured_hbm": 0.65812},
    }
    s = bench.metric_summary(extras)
    assert set(s) == {"ensemble64", "shared_geometry64", "hmatrix_kv_frac_of_measured_hbm"}
    assert set(s["ensemble64"]) == {"v_fp64", "newton_hmat_fp32"}
    assert s["ensemble64"]["newton_hmat_fp32"]["steps_per_s_vs_v_fp64"] == 3.38
    assert s["ensemble64"]["newton_hmat_fp32"]["slip_rel_err_vs_fp64"] == 3.77e-07
    assert s["shared_geometry64"]["tc_over_fp64_shared_v"]["network_steps_per_s"] == 6.78
    assert s["hmatrix_kv_frac_of_measured_hbm"] == 0.658
