"""Shared-geometry batches on tensor cores (DFN_STORE_BF16X2_TC): K.V of R
networks as one tcgen05 GEMM with BF16 hi + lo operands and FP32
accumulation, against the FP64 dense K.V of the same networks.

Tolerance: 1e-4 of the largest stress rate (BF16 hi + lo keeps 16 mantissa
bits of every K entry and V value; the dropped lo x lo term and the FP32
accumulation stay below that)."""
import numpy as np
import pytest

from demystification_dfn_b200 import networks
from demystification_dfn_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def _members(R, n_faults=5, seed=3, mode="modeII"):
    base = networks.small_network(seed=seed, n_faults=n_faults, mode=mode, tol=1e-7)
    return networks.shared_geometry_ensemble(R, base=base, seed=seed)


@pytest.mark.parametrize("R", [1, 5, 40, 100, 200])
@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
def test_tensor_core_kv_matches_fp64(R, mode):
    """R = 1..200 covers all GEMM widths (16, 64, 128, 256 columns)."""
    ps = _members(R, mode=mode)
    rng = np.random.default_rng(R)
    with Ensemble(ps, storage="bf16x2_tc") as tc, Ensemble(ps, storage="fp64") as ref:
        N = tc.n_elements[0]
        slips = [1e-9 * np.exp(rng.normal(0.0, 1.0, N)) * rng.choice([-1.0, 1.0], N) for _ in range(R)]
        gT, gN = tc.kernel(slips)
        rT, rN = ref.kernel(slips)
        for r in range(R):
            assert np.abs(gT[r] - rT[r]).max() <= 1e-4 * np.abs(rT[r]).max(), r
            if mode == "modeII":
                assert np.abs(gN[r] - rN[r]).max() <= 1e-4 * np.abs(rN[r]).max(), r


def test_tensor_core_long_reduction_and_many_tiles():
    """A network of ~2500 elements: 39 row tiles, 39 reduction stages, the
    reduction split over several CTAs, two calls in a row (the pipeline
    state of one launch does not leak into the next)."""
    base = networks.fault_network(n_faults=120, box=3500.0, seed=5)
    ps = networks.shared_geometry_ensemble(24, base=base, seed=5)
    rng = np.random.default_rng(0)
    with Ensemble(ps, storage="bf16x2_tc") as tc, Ensemble(ps, storage="fp64") as ref:
        N = tc.n_elements[0]
        assert N > 2000
        for _ in range(2):
            slips = [rng.normal(0.0, 1.0, N) for _ in ps]
            gT, gN = tc.kernel(slips)
            rT, rN = ref.kernel(slips)
            for r in range(len(ps)):
                assert np.abs(gT[r] - rT[r]).max() <= 1e-4 * np.abs(rT[r]).max(), r
                assert np.abs(gN[r] - rN[r]).max() <= 1e-4 * np.abs(rN[r]).max(), r


def test_tensor_core_batch_solve_follows_fp64():
    """Whole RK45 runs of a shared-geometry batch to the same time: slip rate
    and log-state of every member within 1e-3 of the FP64 batch."""
    ps = _members(12, n_faults=4, seed=8)
    with Ensemble(ps, storage="bf16x2_tc") as tc, Ensemble(ps, storage="fp64") as ref:
        t_end = 2000.0
        rr = ref.solve(t_end=t_end)
        rep = tc.solve(t_end=t_end)
        assert min(r["it_count"] for r in rr) >= 10
        assert all(r["status"] == 0 for r in rep)
        for i in range(len(ps)):
            a, b = tc.state(i), ref.state(i)
            N = len(a["P"])
            assert abs(a["time"] - b["time"]) <= 1e-9 * t_end
            assert np.abs(a["Y"][:N] - b["Y"][:N]).max() <= 1e-3 * np.abs(b["Y"][:N]).max()
            assert np.abs(a["Y"][N:2 * N] - b["Y"][N:2 * N]).max() <= 1e-3 * np.abs(b["Y"][N:2 * N]).max()


def test_tensor_core_storage_needs_shared_geometry():
    from demystification_dfn_b200 import _lib

    ps = [networks.small_network(seed=s, n_faults=3) for s in (1, 2)]
    with pytest.raises(_lib.DfnError):
        Ensemble(ps, storage="bf16x2_tc")


def test_tensor_core_autotune_keeps_results():
    """The persistent GEMM and the two unit-per-CTA rings sum every unit in
    the same order: K.V after the autotuner's choice equals K.V before, bit
    for bit."""
    ps = _members(40)
    rng = np.random.default_rng(4)
    with Ensemble(ps, storage="bf16x2_tc") as e:
        N = e.n_elements[0]
        slips = [rng.normal(size=N) for _ in ps]
        a, _ = e.kernel(slips)
        t = e.autotune()
        assert t["gemv_impl"] in ("tc_persistent", "tc_ring_deep", "tc_ring_2stage")
        assert t["ms"]["kv_tc_persistent"] > 0 and t["ms"]["kv_tc_ring_deep"] > 0
        assert t["ms"]["kv_tc_ring_2stage"] > 0   # BN = 64 has a deeper ring than two stages
        b, _ = e.kernel(slips)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("count", [3, 40, 130])
def test_tensor_core_shapes_identical(count):
    """Each K.V shape of the GEMM (persistent, deepest ring, 2-stage ring),
    chosen at creation, gives the same bits; batch sizes cover BN = 16, 64
    and 256 (BN = 256 has no shallower ring: shapes 1 and 2 coincide)."""
    # 250 faults, N of about 5000: more work units than SMs, so every
    # persistent CTA walks several units and both TMEM accumulators
    base = networks.fault_network(n_faults=250, box=3500.0, seed=2)
    ps = networks.shared_geometry_ensemble(count, base=base, seed=count)
    rng = np.random.default_rng(count)
    outs = []
    for gemv in ("tc_persistent", "tc_ring_deep", "tc_ring_2stage"):
        with Ensemble(ps, storage="bf16x2_tc", gemv=gemv) as e:
            N = e.n_elements[0]
            if not outs:
                slips = [rng.normal(size=N) for _ in ps]
            outs.append(e.kernel(slips))
    for o in outs[1:]:
        for x, y in zip(outs[0][0], o[0]):
            assert np.array_equal(x, y)
        for x, y in zip(outs[0][1], o[1]):
            assert np.array_equal(x, y)