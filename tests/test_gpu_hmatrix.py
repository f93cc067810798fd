"""H-matrix K.V (static_kernel = hmatrix) on the GPU against the oracle.

* the cluster order (the reference's mat_corr) must equal the oracle's
  restatement of src/hmatrix/cluster_tree.f90 exactly;
* H.V must match the dense K.V within a few eps_ACA (relative to max|K.V|):
  both the GPU's partial-pivot ACA + recompression and the oracle's
  full-pivot ACA approximate the same blocks to the same tolerance;
* whole RK45 runs on the H-matrix stay within 1e-6 of the dense oracle run.
"""
import numpy as np
import pytest

from oracle import Oracle
from demystification_dfn_b200 import networks
from demystification_dfn_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def hnet(mode="modeII", seed=3, n=40, box=1500.0, **kw):
    return networks.fault_network(n_faults=n, box=box, seed=seed, mode=mode, kernel="hmatrix", tol=1e-6, **kw)


@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
@pytest.mark.parametrize("storage", ["fp64", "fp32"])
def test_hmat_kv_against_dense_oracle(mode, storage):
    p = hnet(mode)
    eps = 1e-6
    o = Oracle(p)
    with Simulation(p, storage=storage, hmat_leaf=32, hmat_eta=2.0, hmat_eps=eps) as s:
        st = s.hmat_stats()
        assert st["lowrank_leaves"] > 0 and st["values"] < s.N * s.N * (2 if mode == "modeII" else 1)
        o.use_hmatrix(leaf=32, eta=2.0, eps=eps)
        assert np.array_equal(s.hmat_perm(), o.hmat_perm())
        assert st["leaves"] == o.hmat_stats()["leaves"] * (2 if mode == "modeII" else 1)
        v = np.random.default_rng(1).normal(size=s.N) * 1e-9
        gT, gN = s.kernel(v)
        hT, hN = o.kernel(v)
        o.use_dense()
        dT, dN = o.kernel(v)
        tol = 20 * eps
        assert rel(gT, dT) < tol and rel(hT, dT) < tol
        if mode == "modeII":
            assert rel(gN, dN) < tol and rel(hN, dN) < tol


@pytest.mark.parametrize("storage", ["fp64", "fp32"])
def test_hmat_small_leaves_by_warp_or_cta(storage):
    """Whole low-rank leaves of a few KB by one warp each (default) or by one
    CTA each: the same products summed in another order, so K.V agrees to
    rounding, and the warp form repeats bit for bit."""
    p = hnet("modeII", seed=4, n=60, box=2000.0)
    kw = dict(storage=storage, pressure="tridiag", hmat_leaf=32, hmat_eta=2.0, hmat_eps=1e-6)
    with Simulation(p, **kw) as s:
        assert s.hmat_stats()["lowrank_leaves"] > 400
        v = np.random.default_rng(3).normal(size=s.N) * 1e-9
        warp = s.kernel(v)
        assert all(np.array_equal(a, b) for a, b in zip(s.kernel(v), warp))
        s.set_hmat_small_leaves("cta")
        cta = s.kernel(v)
        for a, b in zip(warp, cta):
            assert rel(a, b) < 1e-12
        s.set_hmat_small_leaves("warp")
        assert all(np.array_equal(a, b) for a, b in zip(s.kernel(v), warp))


@pytest.mark.parametrize("storage", ["fp64", "fp32"])
def test_hmat_persistent_grids_are_bitwise(storage):
    """The dense-row and small-leaf kernels on persistent grids (a few CTAs
    looping over the tasks) do each row's arithmetic as with one CTA per
    task: K.V and a few solve steps are bitwise identical, and the
    autotuner's pick keeps them so."""
    p = hnet("modeII", seed=4, n=60, box=2000.0)
    kw = dict(storage=storage, pressure="tridiag", hmat_leaf=32, hmat_eta=2.0, hmat_eps=1e-6)
    with Simulation(p, **kw) as s:
        v = np.random.default_rng(5).normal(size=s.N) * 1e-9
        base = s.kernel(v)
        for dense, warp in ((148, 296), (1, 1), (37, 5)):
            s.set_hmat_grids(dense, warp)
            assert all(np.array_equal(a, b) for a, b in zip(s.kernel(v), base)), (dense, warp)
        s.set_hmat_grids(0, 0)
        s.solve_steps(6)
        ref = s.state()
    with Simulation(p, **kw) as s:
        tune = s.autotune()
        assert "hm_dense_grid" in tune
        assert all(np.array_equal(a, b) for a, b in zip(s.kernel(v), base))
        s.solve_steps(6)
        g = s.state()
    assert np.array_equal(g["Y"], ref["Y"]) and g["time"] == ref["time"]


def test_hmat_reference_defaults_on_shipped_bp6():
    """The reference's own BP6 input uses static_kernel = hmatrix with its
    defaults (nleaf 100, eta 3, eps 1e-8)."""
    import refconfigs

    p = refconfigs.problem("bp6")
    o = Oracle(p, threads=8)
    with Simulation(p) as s:
        st = s.hmat_stats()
        assert st["lowrank_leaves"] > 0
        v = np.random.default_rng(2).normal(size=s.N)
        gT, _ = s.kernel(v)
        o.use_dense()
        dT, _ = o.kernel(v)
        assert rel(gT, dT) < 1e-6


def test_hmat_run_close_to_dense_oracle():
    p = hnet("modeII", seed=5, n=30, box=1200.0)
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, pressure="cg_exact", hmat_leaf=32, hmat_eta=2.0, hmat_eps=1e-8) as s:
        rep = s.solve_steps(10)
        st, _ = o.solve_steps(10)
        assert st == 0 and rep["status"] == 0
        g, r = s.state(), o.state()
        N = s.N
        assert abs(g["time"] - r["time"]) <= 1e-6 * r["time"]
        assert rel(g["Y"][:N], r["Y"][:N]) < 1e-6


def test_hmat_batch_equals_single():
    from demystification_dfn_b200.ensemble import Ensemble

    ps = [hnet("modeII", seed=s, n=12, box=700.0) for s in (7, 8)]
    kw = dict(hmat_leaf=32, hmat_eta=2.0, hmat_eps=1e-6, pressure="tridiag")
    with Ensemble(ps, **kw) as ens:
        ens.solve(n_steps=8)
        for i, p in enumerate(ps):
            with Simulation(p, **kw) as s:
                s.solve_steps(8)
                assert np.array_equal(ens.state(i)["Y"], s.state()["Y"])


def test_loaded_network_event_onset_hmatrix():
    """Config-3 physics at test size: a velocity-weakening network under
    tectonic shear loading (0.05 Pa/s) reaches seismic slip (max V > 1e-3
    m/s) after ~1.2 simulated years and ~500 adaptive steps. The GPU
    H-matrix (partial-pivot ACA + recompression, FP64 factors) and the
    oracle's restatement of the reference's H-matrix (full-pivot ACA) agree
    to the ACA tolerance, not bit for bit, so the onset times agree to 1e-3;
    FP32 factors follow FP64 factors to 1e-4."""
    p = networks.fault_network(n_faults=6, box=3000.0, length_range=(300.0, 1200.0), seed=3, dP=0.0,
                               kernel="hmatrix", tol=1e-6)
    for f in p.faults:
        f.shear_loading_dot[:] = 0.05
    o = Oracle(p, threads=4)
    assert o.use_hmatrix(leaf=32, eta=2.0, eps=1e-6)

    def onset(step, state):
        for k in range(1, 3000):
            step()
            s = state()
            N = len(s["P"])
            if np.abs(s["Y"][:N]).max() > 1e-3:
                return k, s["time"]
        return None, None

    ko, to = onset(lambda: o.solve_steps(1), o.state)
    assert ko is not None
    res = {}
    for store in ("fp64", "fp32"):
        with Simulation(p, storage=store, pressure="cg", hmat_leaf=32, hmat_eta=2.0, hmat_eps=1e-6) as s:
            res[store] = onset(lambda: s.solve_steps(1), s.state)
    kg, tg = res["fp64"]
    kf, tf = res["fp32"]
    assert kg is not None and kf is not None
    assert abs(tg - to) <= 1e-3 * to
    assert abs(tf - tg) <= 1e-4 * tg
