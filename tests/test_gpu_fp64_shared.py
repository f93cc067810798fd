"""Shared-geometry batches in FP64 (DFN_STORE_FP64_SHARED): one FP64 kernel
matrix for R networks and one FP64 GEMM per stage on the CUDA cores, the
counterpart of the tensor-core batch without its BF16 arithmetic.

Tolerances: K.V within 1e-12 of the oracle's dense FP64 K.V (the sums run
in another order than the oracle's, with FMAs); whole RK45 runs within 1e-9
of the per-network FP64 path (the same arithmetic up to summation order,
which rounding then carries through the steps)."""
import numpy as np
import pytest

from oracle import Oracle
from demystification_dfn_b200 import networks
from demystification_dfn_b200.ensemble import Ensemble
from demystification_dfn_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def _members(R, n_faults=5, seed=3, mode="modeII", **kw):
    base = networks.small_network(seed=seed, n_faults=n_faults, mode=mode, tol=1e-7, **kw)
    return networks.shared_geometry_ensemble(R, base=base, seed=seed)


@pytest.mark.parametrize("R", [1, 7, 64, 65, 200])
@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
def test_fp64_shared_kv_matches_oracle(R, mode):
    """R = 1..200: one to four member tiles of 64, partial last tiles."""
    ps = _members(R, mode=mode)
    o = Oracle(ps[0])
    o.use_dense()
    rng = np.random.default_rng(R)
    with Ensemble(ps, storage="fp64_shared") as e:
        N = e.n_elements[0]
        slips = [1e-9 * np.exp(rng.normal(0.0, 1.0, N)) * rng.choice([-1.0, 1.0], N) for _ in range(R)]
        gT, gN = e.kernel(slips)
        for r in range(R):
            oT, oN = o.kernel(slips[r])
            assert np.abs(gT[r] - oT).max() <= 1e-12 * np.abs(oT).max(), r
            if mode == "modeII":
                assert np.abs(gN[r] - oN).max() <= 1e-12 * np.abs(oN).max(), r


def test_fp64_shared_long_reduction_and_splits():
    """~2500 elements: 79 row tiles, 79 column chunks split over several
    CTAs; two calls in a row."""
    base = networks.fault_network(n_faults=120, box=3500.0, seed=5)
    ps = networks.shared_geometry_ensemble(24, base=base, seed=5)
    rng = np.random.default_rng(0)
    with Ensemble(ps, storage="fp64_shared") as e, Ensemble(ps, storage="fp64") as ref:
        N = e.n_elements[0]
        assert N > 2000
        for _ in range(2):
            slips = [rng.normal(0.0, 1.0, N) for _ in ps]
            gT, gN = e.kernel(slips)
            rT, rN = ref.kernel(slips)
            for r in range(len(ps)):
                assert np.abs(gT[r] - rT[r]).max() <= 1e-12 * np.abs(rT[r]).max(), r
                assert np.abs(gN[r] - rN[r]).max() <= 1e-12 * np.abs(rN[r]).max(), r


@pytest.mark.parametrize("formulation", ["v", "newton"])
def test_fp64_shared_batch_follows_the_per_network_path(formulation):
    ps = _members(6, n_faults=4, seed=8)
    t_end = 3000.0
    with Ensemble(ps, storage="fp64_shared", pressure="tridiag", formulation=formulation) as e:
        reps = e.solve(t_end=t_end)
        assert all(r["status"] == 0 for r in reps)
        for i, p in enumerate(ps):
            a = e.state(i)
            with Simulation(p, pressure="tridiag", formulation=formulation) as s:
                s.solve_to(t_end)
                b = s.state()
                sb = s.slip()
            N = len(a["P"])
            assert abs(a["time"] - t_end) <= 1e-12 * t_end
            for j in range(2):
                x, y = a["Y"][j * N:(j + 1) * N], b["Y"][j * N:(j + 1) * N]
                assert np.abs(x - y).max() <= 1e-9 * np.abs(y).max(), (i, j)
            sa = e.slip(i)
            assert np.abs(sa - sb).max() <= 1e-9 * np.abs(sb).max(), i


def test_fp64_shared_needs_shared_geometry():
    a = networks.small_network(seed=1, n_faults=3)
    b = networks.small_network(seed=2, n_faults=3)
    from demystification_dfn_b200._lib import DfnError

    with pytest.raises(DfnError) as e:
        Ensemble([a, b], storage="fp64_shared")
    assert e.value.status == 5
