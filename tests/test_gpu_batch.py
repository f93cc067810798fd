"""Batched networks: one handle, one launch per kernel for the whole batch,
per-network step control. A network inside a batch must follow exactly the
trajectory it follows alone (same kernels, same per-network arithmetic)."""
import numpy as np
import pytest

from oracle import Oracle
from demystification_dfn_b200 import networks
from demystification_dfn_b200.ensemble import Ensemble
from demystification_dfn_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def members(mode="modeII"):
    # uneven sizes, different injection and diffusivity
    return [networks.small_network(seed=s, n_faults=n, mode=mode, tol=1e-6, q_kgs=q)
            for s, n, q in ((21, 3, 20.0), (22, 6, None), (23, 4, 60.0))]


@pytest.mark.parametrize("pressure", ["cg", "tridiag"])
def test_batch_equals_separate_runs_bitwise(pressure):
    ps = members()
    with Ensemble(ps, pressure=pressure) as ens:
        reps = ens.solve(n_steps=15)
        assert all(r["status"] == 0 for r in reps)
        for i, p in enumerate(ps):
            with Simulation(p, pressure=pressure) as s:
                s.solve_steps(15)
                a, b = ens.state(i), s.state()
                assert a["it_count"] == b["it_count"] == 15
                assert a["time"] == b["time"]
                assert np.array_equal(a["Y"], b["Y"]) and np.array_equal(a["P"], b["P"])


def test_batch_member_matches_oracle():
    """Network 1 stalls the reference CG at its 200-iteration cap from step
    13 on (the probe halves t_try there), where an ulp decides the halving;
    the first 12 steps are compared, with the bitwise reference CG."""
    ps = members()
    with Ensemble(ps, pressure="cg_exact") as ens:
        ens.solve(n_steps=12)
        o = Oracle(ps[1])
        o.use_dense()
        st, _ = o.solve_steps(12)
        assert st == 0
        g, r = ens.state(1), o.state()
        N = len(r["P"])
        assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
        assert np.abs(g["Y"][:N] - r["Y"][:N]).max() <= 1e-8 * np.abs(r["Y"][:N]).max()


def test_batch_runs_to_t_end_with_done_masks():
    ps = members()
    t_end = 3000.0
    with Ensemble(ps, pressure="tridiag") as ens:
        reps = ens.solve(t_end=t_end)
        for i, r in enumerate(reps):
            assert r["status"] == 0
            st = ens.state(i)
            # the last step is shortened to land on t_end
            assert abs(st["time"] - t_end) <= 1e-12 * t_end
            assert st["time"] - r["last_hdid"] < t_end
        # networks stopped independently: different step counts
        assert len({r["it_count"] for r in reps}) > 1


def test_stage_cg_cap_policy_matches_oracle():
    """Network 1 drives the reference CG to its cap inside RK stages; the
    GPU and the oracle both go on with the last CG iterate (the reference's
    P_temp is undefined there) and both finish the steps."""
    p = members()[1]
    o = Oracle(p)
    o.use_dense()
    st, _ = o.solve_steps(20)
    with Simulation(p, pressure="cg_exact") as s:
        rep = s.solve_steps(20)
    assert st == 0 and rep["status"] == 0
    assert rep["it_count"] == 20


def test_ensemble_members_run():
    ps = networks.ensemble(4)
    with Ensemble(ps, pressure="cg") as ens:
        reps = ens.solve(n_steps=5, check=False)
        for r in reps:
            assert r["status"] == 0, r
            assert r["it_count"] == 5


def test_mode3_batch():
    ps = members("modeIII")
    with Ensemble(ps, pressure="cg", storage="fp32") as ens:
        reps = ens.solve(n_steps=10)
        assert all(r["status"] == 0 and r["it_count"] == 10 for r in reps)


@pytest.mark.parametrize("pressure", ["cg", "tridiag"])
def test_graph_replay_matches_single_launches_bitwise(pressure):
    """The solve loop replayed as CUDA graphs of 8 rounds gives the state of
    the same rounds launched one by one, bit for bit, for a batch run to a
    step count (graphs, then single rounds for the remainder) and to t_end."""
    ps = [networks.small_network(seed=s, n_faults=3 + s % 3, tol=1e-7) for s in range(4)]
    out = []
    for graphs in (True, False):
        with Ensemble(ps, pressure=pressure) as ens:
            ens.set_graphs(graphs)
            ens.solve(n_steps=21)
            ens.solve(t_end=ens.state(0)["time"] * 3.0)
            out.append([ens.state(i) for i in range(len(ps))])
    for a, b in zip(*out):
        assert a["it_count"] == b["it_count"] and a["time"] == b["time"]
        assert np.array_equal(a["Y"], b["Y"]) and np.array_equal(a["P"], b["P"])


def test_autotune_keeps_results():
    """The autotuner picks among launch shapes with equal results: the K.V
    copy path is bitwise neutral, the short-segment pressure solve (thread or
    warp per segment) equal to rounding."""
    ps = members()
    out = {}
    for pressure in ("cg", "tridiag"):
        for tune in (False, True):
            with Ensemble(ps, pressure=pressure) as ens:
                if tune:
                    t = ens.autotune()
                    assert t["gemv_impl"] in ("tma", "ldg") and t["ms"]["kv_tma"] > 0 and t["ms"]["kv_ldg"] > 0
                    if pressure == "tridiag":
                        assert t["ms"]["pressure_warp"] > 0 and t["ms"]["pressure_thread"] > 0
                ens.solve(n_steps=12)
                out[(pressure, tune)] = [ens.state(i) for i in range(len(ps))]
    for a, b in zip(out[("cg", False)], out[("cg", True)]):
        assert np.array_equal(a["Y"], b["Y"]) and a["time"] == b["time"]
    for a, b in zip(out[("tridiag", False)], out[("tridiag", True)]):
        N = len(a["P"])
        assert abs(a["time"] - b["time"]) <= 1e-10 * b["time"]
        assert np.abs(a["Y"][:N] - b["Y"][:N]).max() <= 1e-9 * np.abs(b["Y"][:N]).max()


def test_autotune_cg_cluster_choice_equal_to_rounding():
    """Networks of 2048 elements or more: the autotuner times the stage
    pressure systems solved by one CTA each on global memory, by a cluster of
    CTAs each and by one CTA each on shared memory; all stop at
    max|r| < tol_solver, so runs with any of them agree to the solver
    tolerance (here after 6 steps: slip rate to 1e-6 relative)."""
    ps = [networks.fault_network(n_faults=150, box=3000.0, seed=s, tol=1e-8) for s in (31, 32)]
    out = []
    for tune in (False, True):
        with Ensemble(ps, pressure="cg") as ens:
            if tune:
                t = ens.autotune()
                ms = t["ms"]
                assert ms["pressure_cg_cta"] > 0 and ms["pressure_cg_cluster"] > 0 and ms["pressure_cg_cta_smem"] > 0
                best = min(("cta", "cluster", "cta_smem"), key=lambda f: ms["pressure_cg_" + f])
                assert t["cg_form"] == best
            reps = ens.solve(n_steps=6)
            assert all(r["status"] == 0 for r in reps)
            out.append([ens.state(i) for i in range(len(ps))])
    for a, b in zip(*out):
        N = len(a["P"])
        assert abs(a["time"] - b["time"]) <= 1e-9 * a["time"]
        assert np.abs(a["Y"][:N] - b["Y"][:N]).max() <= 1e-6 * np.abs(a["Y"][:N]).max()


def test_cg_forms_agree_on_an_uneven_batch():
    """A batch of four ensemble networks of uneven size (some fit the shared
    memory of one CTA, some do not and use the global-memory solver in the
    same launch): every CG form gives the same run to the solver tolerance."""
    ps = [networks.ensemble_member(s) for s in (3, 5, 9, 12)]
    sizes = None
    out = {}
    for form in ("default", "cta", "cta_smem"):
        with Ensemble(ps, pressure="cg") as ens:
            sizes = ens.n_elements
            ens.set_cg_form(form)
            reps = ens.solve(n_steps=6)
            assert all(r["status"] == 0 for r in reps)
            out[form] = [ens.state(i) for i in range(len(ps))]
    assert min(sizes) < 5700 < max(sizes)
    for form in ("cta", "cta_smem"):
        for a, b in zip(out["default"], out[form]):
            N = len(a["P"])
            assert abs(a["time"] - b["time"]) <= 1e-9 * a["time"]
            assert np.abs(a["Y"][:N] - b["Y"][:N]).max() <= 1e-6 * np.abs(a["Y"][:N]).max()
            assert np.abs(a["P"] - b["P"]).max() <= 1e-6 * np.abs(a["P"]).max()


@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
def test_tridiagonal_tiles_equal_threads_bitwise(mode):
    """Short segments solved in shared-memory tiles give the bits of the
    thread-per-segment solve (the same recurrence); the warp scans agree to
    rounding. A batch of ensemble networks: many short segments, tiles
    across fault and fake elements."""
    ps = [networks.ensemble_member(s, n_faults=60, mode=mode) for s in (2, 4, 6)]
    out = {}
    for shape in ("thread", "tile", "warp"):
        with Ensemble(ps, pressure="tridiag") as ens:
            ens.set_tri_shape(shape)
            reps = ens.solve(n_steps=10)
            assert all(r["status"] == 0 for r in reps)
            out[shape] = [ens.state(i) for i in range(len(ps))]
    for a, b in zip(out["thread"], out["tile"]):
        assert a["time"] == b["time"]
        assert np.array_equal(a["Y"], b["Y"]) and np.array_equal(a["P"], b["P"])
    for a, b in zip(out["thread"], out["warp"]):
        N = len(a["P"])
        assert np.abs(a["Y"][:N] - b["Y"][:N]).max() <= 1e-6 * np.abs(a["Y"][:N]).max()
