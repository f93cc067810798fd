"""GPU parity: the CUDA path through the C ABI against the CPU FP64 oracle.

Tolerances (relative to the largest magnitude of the compared quantity):
* K.V with FP64 storage: 1e-12 (entry rounding and summation order only)
* K.V with FP32 storage: 2e-6; BF16 hi+lo: 5e-5
* friction RHS: 1e-10; pressure (tridiagonal vs exact): 1e-12
* pressure CG vs oracle CG: both stop at max|r| < tol_solver, so they agree
  to well below 1e3 * tol_solver Pa
* whole RK45 steps: slip rate and log-state within 1e-8 (the parity target)
"""
import os

import numpy as np
import pytest

from oracle import Oracle
from demystification_dfn_b200 import build_arrays, networks
from demystification_dfn_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def rel(a, b):
    s = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / s


def net(seed=1, n=4, mode="modeII", **kw):
    return networks.small_network(seed=seed, n_faults=n, mode=mode, **kw)


@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
@pytest.mark.parametrize("storage,tol", [("fp64", 1e-12), ("fp32", 2e-6), ("bf16x2", 5e-5)])
@pytest.mark.parametrize("gemv", ["tma", "ldg"])
def test_kernel_matches_oracle(mode, storage, tol, gemv):
    p = net(seed=2, n=5, mode=mode)
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, storage=storage, gemv=gemv) as s:
        rng = np.random.default_rng(3)
        v = 1e-9 * np.exp(rng.normal(size=s.N))
        v[s.arrays.fake_mask] = 0.0
        gT, gN = s.kernel(v)
        oT, oN = o.kernel(v)
        assert rel(gT, oT) < tol
        if mode == "modeII":
            assert rel(gN, oN) < tol


def test_kernel_large_single_fault_and_linearity():
    p = networks.single_fault(n_el=3000, length=30e3, mode="modeII")
    o = Oracle(p, threads=8)
    with Simulation(p) as s:
        rng = np.random.default_rng(0)
        v1, v2 = rng.normal(size=s.N), rng.normal(size=s.N)
        g1, _ = s.kernel(v1)
        g2, _ = s.kernel(v2)
        g12, _ = s.kernel(2.0 * v1 - 3.0 * v2)
        assert rel(g12, 2.0 * g1 - 3.0 * g2) < 1e-12
        oT, _ = o.kernel(v1)   # matrix-free reference routine
        assert rel(g1, oT) < 1e-11


def test_tma_and_ldg_agree_bitwise():
    p = net(seed=4, n=6)
    with Simulation(p, gemv="tma") as a, Simulation(p, gemv="ldg") as b:
        v = np.random.default_rng(1).normal(size=a.N)
        ta, na = a.kernel(v)
        tb, nb = b.kernel(v)
        assert np.array_equal(ta, tb) and np.array_equal(na, nb)


@pytest.mark.parametrize("dt", [1.0, 100.0, 5000.0])
def test_pressure_cg_matches_oracle(dt):
    p = networks.single_fault(n_el=300, length=3000.0, mode="modeIII", tol=1e-6)
    o = Oracle(p)
    with Simulation(p, pressure="cg") as s:
        gP, gd, gi = s.compute_P(dt)
        oP, od, oi = o.compute_P(dt)
        assert gi == oi == 0
        assert np.abs(gP - oP).max() < 1e3 * 1e-6
        ex = o.pressure_exact(dt)
        assert np.abs(gP - ex).max() < 1e3 * 1e-6


def _cluster_case(case):
    # N >= 2048: the CG runs on a thread-block cluster of 2 (N = 4 000),
    # 4 (N = 5 748) or 8 CTAs (N = 10 215, the last range one element shorter)
    if case == "single4000":
        return networks.single_fault(n_el=4000, length=40e3, mode="modeII", tol=1e-8)
    if case == "net300":
        return networks.fault_network(n_faults=300, box=4000.0, seed=5, tol=1e-8)
    return networks.fault_network(n_faults=500, box=5500.0, seed=6, tol=1e-8)


@pytest.mark.parametrize("case", ["single4000", "net300", "net500"])
@pytest.mark.parametrize("dt", [10.0, 3600.0, 86400.0])
@pytest.mark.parametrize("form", ["cluster", "cta_smem", "cta"])
def test_pressure_cg_cluster_matches_oracle(case, dt, form):
    """Each form of the CG (a cluster of CTAs with the vectors in shared
    memory and reductions across the cluster; one CTA with the vectors in
    shared memory, the lean layout for N = 5 748, the global-memory solver
    for N = 10 215; one CTA on global memory) stops at the same criterion
    max|r| < tol_solver as the reference CG: all are within 1e3 * tol_solver
    Pa of it and of the exact implicit step, or all report non-convergence."""
    p = _cluster_case(case)
    o = Oracle(p)
    with Simulation(p, pressure="cg") as s:
        assert s.N >= 2048
        s.set_cg_form(form)
        gP, gd, gi = s.compute_P(dt)
        oP, od, oi = o.compute_P(dt)
        assert gi == oi
        if oi == 0:
            assert np.abs(gP - oP).max() < 1e3 * 1e-8
            assert np.abs(gP - o.pressure_exact(dt)).max() < 1e3 * 1e-8
            scale = max(np.abs(od).max(), 1e-300)
            assert np.abs(gd - od).max() / scale < 1e-6


def test_pressure_cg_cluster_lean_layout_matches_oracle():
    """70 000 elements: ranges of 4 375 elements on a cluster of 16 CTAs,
    too long to keep x and M p in shared memory (x in the global work area,
    M p recomputed). Where the device cannot schedule clusters of 16 the
    one-CTA solver runs instead; the parity bound is the same."""
    p = networks.single_fault(n_el=70000, length=700e3, mode="modeIII", tol=1e-8, kernel="hmatrix")
    o = Oracle(p)
    with Simulation(p, storage="fp32", pressure="cg", hmat_leaf=256, hmat_eta=2.0, hmat_eps=1e-4) as s:
        for dt in (60.0, 20000.0):
            gP, gd, gi = s.compute_P(dt)
            oP, od, oi = o.compute_P(dt)
            assert gi == oi == 0
            assert np.abs(gP - oP).max() < 1e3 * 1e-8
        ctas = s.autotune()["cg_cluster_ctas"]
        assert ctas in (0, 16)


def test_pressure_cg_cluster_nonconvergence_sets_ier():
    p = networks.single_fault(n_el=4000, length=40e3, mode="modeIII", tol=1e-14)
    with Simulation(p, pressure="cg") as s:
        P0 = s.state()["P"]
        _, _, ier = s.compute_P(86400.0)
        assert ier == 1
        _, _, ier2 = s.compute_P(1e-3)
        assert ier2 in (0, 1)
        assert np.array_equal(s.state()["P"], P0)


@pytest.mark.parametrize("dt", [1.0, 100.0, 1000.0, 5000.0])
def test_pressure_cg_exact_is_bitwise_reference_cg(dt):
    """Sequential dot products and the reference's operand order: the same
    iterates, the same iteration count, the same ier as the oracle (on this
    network CG stalls at dt = 1000 and 5000 s, as in the reference)."""
    p = net(seed=22, n=6, tol=1e-6)
    o = Oracle(p)
    with Simulation(p, pressure="cg_exact") as s:
        gP, gd, gi = s.compute_P(dt)
        oP, od, oi = o.compute_P(dt)
        assert gi == oi
        if oi == 0:
            assert np.array_equal(gP, oP) and np.array_equal(gd, od)


def test_pressure_cg_nonconvergence_sets_ier():
    p = networks.single_fault(n_el=400, length=4000.0, mode="modeIII", tol=1e-14)
    with Simulation(p, pressure="cg") as s:
        _, _, ier = s.compute_P(86400.0)
        assert ier == 1
        # the handle stays usable after ier=1
        _, _, ier2 = s.compute_P(1e-3)
        assert ier2 in (0, 1)


@pytest.mark.parametrize("case", ["pair", "shipped"])
@pytest.mark.parametrize("dt", [60.0, 3600.0, 86400.0])
def test_pressure_with_fault_crossings_matches_oracle(case, dt):
    """Fault-crossing coupling: the same crossings as the oracle, and the
    reference-order CG (cg_exact) bitwise the oracle's; the tree-reduced CG
    within the solver tolerance."""
    import refconfigs

    p = networks.crossing_pair(n_el=100) if case == "pair" else refconfigs.problem("network")
    o = Oracle(p)
    oP, od, oi = o.compute_P(dt)
    with Simulation(p, pressure="cg_exact") as s:
        assert s.crossing_count == o.crossings() > 0
        gP, gd, gi = s.compute_P(dt)
        assert gi == oi
        if oi == 0:
            assert np.array_equal(gP, oP) and np.array_equal(gd, od)
    with Simulation(p, pressure="cg") as s:
        gP, gd, gi = s.compute_P(dt)
        assert gi == oi
        if oi == 0:
            assert np.abs(gP - oP).max() < 1e3 * p.hyperparameter.tol_solver


def test_tridiagonal_pressure_rejects_fault_crossings():
    from demystification_dfn_b200 import _lib

    with pytest.raises(_lib.DfnError):
        Simulation(networks.crossing_pair(n_el=100), pressure="tridiag")


def test_batch_with_fault_crossings_equals_separate_runs():
    """Networks with crossings in one batch follow their own runs bit for bit."""
    from demystification_dfn_b200.ensemble import Ensemble

    ps = [networks.crossing_pair(n_el=100, angle_deg=a, q_kgs=20.0, tol=1e-6) for a in (45.0, 70.0)]
    with Ensemble(ps, pressure="cg") as ens:
        assert ens.crossing_count == 2
        reps = ens.solve(n_steps=8)
        assert all(r["status"] == 0 for r in reps)
        for i, p in enumerate(ps):
            with Simulation(p, pressure="cg") as s:
                s.solve_steps(8)
                a, b = ens.state(i), s.state()
                assert a["time"] == b["time"]
                assert np.array_equal(a["Y"], b["Y"]) and np.array_equal(a["P"], b["P"])


@pytest.mark.parametrize("dt", [0.5, 300.0, 86400.0])
def test_pressure_tridiag_is_exact(dt):
    p = net(seed=6, n=5, mode="modeII", q_kgs=20.0)
    o = Oracle(p)
    with Simulation(p, pressure="tridiag") as s:
        gP, gd, gi = s.compute_P(dt)
        assert gi == 0
        ex = o.pressure_exact(dt)
        assert rel(gP, ex) < 1e-12


@pytest.mark.parametrize("case", ["fault4000", "fault6000", "mixed"])
@pytest.mark.parametrize("dt", [0.5, 300.0, 86400.0])
def test_pressure_tridiag_long_segments_are_exact(case, dt):
    """Segments longer than 48 elements go to the CTA-parallel (scan) Thomas
    solve: rows in registers up to 4096 elements, in global memory above;
    the mixed network has segments on both sides of the 48-element split."""
    if case == "mixed":
        p = networks.fault_network(n_faults=6, box=3000.0, length_range=(300.0, 1500.0), seed=3, q_kgs=20.0)
    else:
        n = int(case[5:])
        p = networks.single_fault(n_el=n, length=10.0 * n, mode="modeII")
    o = Oracle(p)
    with Simulation(p, pressure="tridiag") as s:
        gP, gd, gi = s.compute_P(dt)
        assert gi == 0
        ex = o.pressure_exact(dt)
        assert rel(gP, ex) < 1e-12
        # P_dot = (P_new - P)/dt carries the error of P_new divided by dt
        P0 = s.arrays.P
        assert np.abs(gd - (ex - P0) / dt).max() <= 1e-11 * np.abs(ex).max() / dt


@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
def test_friction_law_matches_oracle(mode):
    p = net(seed=7, n=4, mode=mode, tol=1e-6)
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, pressure="cg") as s:
        Y = s.arrays.Y0().copy()
        rng = np.random.default_rng(2)
        N = s.N
        Y[:N] *= np.exp(rng.normal(0, 0.3, N))
        Y[:N][s.arrays.fake_mask] = 0
        # stage offsets where the reference's CG converges (at dt=1000 s it
        # stalls on this network in the oracle too, and the probe would halve)
        for x in (0.0, 1.0, 10.0):
            assert o.compute_P(x)[2] == 0
            g = s.friction_law(x, Y)
            r = o.friction_law(x, Y)
            for j in range(3):
                assert rel(g[j * N:(j + 1) * N], r[j * N:(j + 1) * N]) < 1e-9, (x, j)


def test_rkqs_matches_oracle():
    p = net(seed=8, n=4, tol=1e-6)
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, pressure="cg") as s:
        Y = s.arrays.Y0()
        ht = 50.0
        dydx = o.friction_law(ht, Y)
        yscal = np.abs(Y) + np.abs(dydx * ht) + 1e-6
        gy, gx, ghd, ghn = s.rkqs(Y, dydx, 0.0, ht, 1e-6, yscal)
        oy, ox, ohd, ohn = o.rkqs(Y, dydx, 0.0, ht, 1e-6, yscal)
        assert np.isclose(ghd, ohd, rtol=1e-12) and np.isclose(ghn, ohn, rtol=1e-9)
        assert rel(gy, oy) < 1e-10


@pytest.mark.parametrize("pressure", ["cg", "cg_exact", "tridiag"])
def test_solve_steps_match_oracle(pressure):
    p = net(seed=9, n=4, tol=1e-6)
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, pressure=pressure) as s:
        nsteps = 25
        rep = s.solve_steps(nsteps)
        st, log = o.solve_steps(nsteps)
        assert st == 0 and rep["status"] == 0
        g, r = s.state(), o.state()
        assert g["it_count"] == r["it_count"] == nsteps
        assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
        N = s.N
        for j in range(3):
            assert rel(g["Y"][j * N:(j + 1) * N], r["Y"][j * N:(j + 1) * N]) < 1e-8, j
        assert rel(g["P"], r["P"]) < 1e-8


def test_single_fault_injection_run_matches_oracle():
    p = networks.single_fault(n_el=500, length=5000.0, mode="modeII", tol=1e-6)
    o = Oracle(p, threads=8)
    o.use_dense()
    with Simulation(p, pressure="cg_exact") as s:
        rep = s.solve_steps(30)
        st, _ = o.solve_steps(30)
        g, r = s.state(), o.state()
        assert st == 0 and rep["status"] == 0
        assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
        N = s.N
        assert rel(g["Y"][:N], r["Y"][:N]) < 1e-8
        assert rel(g["Y"][N:2 * N], r["Y"][N:2 * N]) < 1e-8
        assert rel(g["P"], r["P"]) < 1e-8


def test_snapshot_and_step_host():
    p = net(seed=10, n=3, tol=1e-6)
    with Simulation(p) as s:
        s.solve_steps(3)
        snap = s.snapshot()
        st = s.state()
        N = s.N
        assert np.array_equal(snap["V"], st["Y"][:N])
        a = s.arrays
        assert np.allclose(snap["theta"], a.Dc / a.V0 * np.exp(st["Y"][N:2 * N]), rtol=1e-14)
        assert np.array_equal(snap["tractionNel"], st["Y"][2 * N:])
        assert snap["time"] == st["time"]


def test_snapshot_matches_oracle():
    """save_data's fields after 7 accepted steps (src/solver.f90:211-222):
    V, theta = Dc/V0 exp(psi), P, tractionTel (the shear stress rate of the
    last right-hand side: stage 6 of the accepted attempt) and tractionNel
    (sigmaN), against the oracle's state and its last stress rates."""
    p = net(seed=10, n=4, tol=1e-6)
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, pressure="cg_exact") as s:
        s.solve_steps(7)
        snap = s.snapshot()
    st, _ = o.solve_steps(7)
    assert st == 0
    r = o.state()
    sT, sN, _ = o.last_stress()
    N = len(r["P"])
    a = build_arrays(p)
    assert abs(snap["time"] - r["time"]) <= 1e-8 * r["time"]
    assert rel(snap["V"], r["Y"][:N]) < 1e-8
    assert rel(snap["theta"], a.Dc / a.V0 * np.exp(r["Y"][N:2 * N])) < 1e-8
    assert rel(snap["P"], r["P"]) < 1e-8
    assert rel(snap["tractionTel"], sT) < 1e-8
    assert rel(snap["tractionNel"], r["Y"][2 * N:]) < 1e-8
    assert np.array_equal(snap["permeability"], a.permeability)


def test_benchmark_network_rhs_and_steps_match_oracle():
    """The benchmarked workload itself: the seeded 800-fault network (N =
    16 013, mode II, dense FP64 kernel, 10 MPa pore-pressure step, tol 1e-8).
    One right-hand side at the initial state against the oracle's
    matrix-free directII (src/kernel_calculation/directModeII.f90:33-103) at
    1e-9, then 5 accepted solve() steps (src/solver.f90:59-198) with the
    bitwise reference CG against the oracle's: slip rate, log-state, normal
    traction, pressure and time within 1e-8."""
    import bench

    p = bench.make_problem(0)
    o = Oracle(p, threads=os.cpu_count() or 1)
    with Simulation(p, pressure="cg_exact") as s:
        N = s.N
        assert N == 16013
        Y = s.arrays.Y0()
        # the network starts at steady state, where dpsi/dt = V0/Dc e^-psi -
        # V/Dc is rounding noise: it is measured against the size of its
        # terms, V/Dc
        psi_scale = np.abs(Y[:N] / s.arrays.Dc).max()
        for x in (1.0, 100.0):
            g = s.friction_law(x, Y)
            r = o.friction_law(x, Y)
            assert rel(g[:N], r[:N]) < 1e-9, x
            assert np.abs(g[N:2 * N] - r[N:2 * N]).max() < 1e-9 * psi_scale, x
            assert rel(g[2 * N:], r[2 * N:]) < 1e-9, x
        rep = s.solve_steps(5)
        g = s.state()
    st, _ = o.solve_steps(5)
    r = o.state()
    assert st == 0 and rep["status"] == 0 and g["it_count"] == r["it_count"] == 5
    assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
    for j in range(3):
        assert rel(g["Y"][j * N:(j + 1) * N], r["Y"][j * N:(j + 1) * N]) < 1e-8, j
    assert rel(g["P"], r["P"]) < 1e-8


@pytest.mark.parametrize("pressure", ["cg_exact", "tridiag"])
def test_single_fault_config_mode2_run_matches_oracle(pressure):
    """The single-fault configuration in plane strain (mode II): one 40 km
    fault of 4000 x 10 m elements, a = 0.007, b = 0.005, 50 kg/s injection at
    the centre, tol 1e-8; 40 accepted steps against the oracle (matrix-free
    directII, reference CG) within 1e-8. The tridiagonal solve is the exact
    solution of the same implicit step, so its pressure agrees with the CG's
    to the CG tolerance, far below the state tolerance."""
    p = networks.single_fault(mode="modeII")
    o = Oracle(p, threads=os.cpu_count() or 1)
    with Simulation(p, pressure=pressure) as s:
        rep = s.solve_steps(40)
        g = s.state()
    st, _ = o.solve_steps(40)
    r = o.state()
    N = len(r["P"])
    assert N == 4000 and st == 0 and rep["status"] == 0
    assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
    for j in range(3):
        assert rel(g["Y"][j * N:(j + 1) * N], r["Y"][j * N:(j + 1) * N]) < 1e-8, j
    assert rel(g["P"], r["P"]) < 1e-8


def test_fp32_storage_run_close_to_fp64():
    p = net(seed=11, n=5, tol=1e-6)
    with Simulation(p, storage="fp64", pressure="tridiag") as a, Simulation(p, storage="fp32", pressure="tridiag") as b:
        a.solve_steps(20)
        b.solve_steps(20)
        ga, gb = a.state(), b.state()
        N = a.N
        assert rel(gb["Y"][:N], ga["Y"][:N]) < 1e-4


@pytest.mark.parametrize("tag,steps", [("network", 30), ("bp6", 20)])
def test_reference_shipped_problems(tag, steps):
    """The reference's own shipped inputs (rebuilt from the golden fixture):
    the 10-fault mode II network and the 4000-element mode III injection
    problem, run through solve() on the GPU and in the oracle."""
    import refconfigs

    p = refconfigs.problem(tag)
    o = Oracle(p, threads=8)
    o.use_dense()
    with Simulation(p, pressure="cg_exact") as s:
        rep = s.solve_steps(steps)
        st, _ = o.solve_steps(steps)
        assert st == 0 and rep["status"] == 0
        g, r = s.state(), o.state()
        assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
        N = s.N
        assert rel(g["Y"][:N], r["Y"][:N]) < 1e-8
        assert rel(g["Y"][N:2 * N], r["Y"][N:2 * N]) < 1e-8
        assert rel(g["P"], r["P"]) < 1e-8


def test_solve_writes_reference_output_files(tmp_path):
    """Simulation.solve with an output directory: save_data every stride_time
    steps, an output%07d file every freq_writing_file saved rows and a last
    one at max_it (src/solver.f90:180-201), holding the same snapshots as a
    run that keeps them in memory."""
    from demystification_dfn_b200.hdf5 import read_output

    p = net(seed=12, n=3, tol=1e-6)
    with Simulation(p) as s:
        mem = s.solve(max_it=25, stride_time=2, freq_writing_file=5)
    with Simulation(p) as s:
        s.solve(max_it=25, stride_time=2, freq_writing_file=5, output_dir=str(tmp_path))
    files = sorted(os.listdir(tmp_path))
    # saved at it_count 1, 3, ..., 25: 13 rows -> files after rows 5, 10 and the last 3
    assert files == ["output0000009", "output0000019", "output0000025"]
    rows = []
    for f in files:
        o = read_output(str(tmp_path / f))
        rows += [{k: o[k][r] for k in ("V", "theta", "P", "time")} for r in range(5)]
    rows = rows[:13]
    assert len(mem) == 13
    for a, b in zip(mem, rows):
        assert a["time"] == b["time"]
        for k in ("V", "theta", "P"):
            assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
def test_event_onset_matches_oracle(mode):
    """A velocity-weakening fault (a = 0.010 < b = 0.015) loaded by a 200 kg/s
    injection reaches seismic slip rates within ~70 steps: the first accepted
    step with max V > 1e-3 m/s comes at the same step and, in simulated time,
    within 1e-6 of the simulated span (the event-onset tolerance of the
    seismic-cycle runs)."""
    p = networks.single_fault(n_el=200, length=2000.0, a=0.010, b=0.015, Dc=1e-3, q_kgs=200.0, tol=1e-6,
                              mode=mode)
    o = Oracle(p, threads=4)
    o.use_dense()

    def onset(step, state):
        for k in range(1, 400):
            step()
            s = state()
            N = len(s["P"])
            if np.abs(s["Y"][:N]).max() > 1e-3:
                return k, s["time"]
        return None, None

    ko, to = onset(lambda: o.solve_steps(1), o.state)
    with Simulation(p, pressure="cg_exact") as s:
        kg, tg = onset(lambda: s.solve_steps(1), s.state)
    assert ko is not None and kg == ko
    assert abs(tg - to) <= 1e-6 * to
