"""Failure detection: the reference's stop rules and the library's own limits.

Every failure here is made on the host (a parameter, a state or a limit set
by the test); no GPU fault, trap or hang is involved. Where the reference
has the rule, the oracle is run on the same input and must stop at the same
step with the same status:

* extensional normal traction after a step (check_errors,
  src/solver.f90:412-418): DFN_ERR_EXTENSIONAL, state, pressure and time of
  the failing step committed first, as the reference does;
* "stepsize underflow in rkqs" (src/ode_solver/ode_bs.f90:164):
  DFN_ERR_UNDERFLOW;
* non-finite state from the caller: DFN_ERR_NONFINITE;
* the library's budget of RK attempts per step: DFN_ERR_ATTEMPTS, and a
  network that fails inside a batch leaves the others bit for bit as they
  run alone;
* a bounded wait of the TMA K.V pipeline that runs out (limit set to zero
  polls): DFN_ERR_TIMEOUT once, then the handle goes on after the caller
  restores its state.
"""
import numpy as np
import pytest

from oracle import Oracle
from demystification_dfn_b200 import networks
from demystification_dfn_b200._lib import DfnError
from demystification_dfn_b200.ensemble import Ensemble
from demystification_dfn_b200.layout import build_arrays
from demystification_dfn_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

DFN_ERR_UNDERFLOW, DFN_ERR_EXTENSIONAL, DFN_ERR_NONFINITE, DFN_ERR_ATTEMPTS, DFN_ERR_TIMEOUT = 2, 3, 4, 8, 10


def unloading_fault(mode):
    """200 elements under normal unloading of 1 Pa/s from -0.1 MPa, with a
    friction coefficient near zero (a = 0.5, b = 0.1, f0 = 0.1 at V = 1e-12
    m/s), so that the fault creeps and sigmaN crosses zero at t = 1e5 s
    after about two thousand steps."""
    p = networks.single_fault(n_el=200, length=2000.0, mode=mode, q_kgs=0.0, tol=1e-6, sigmaN=-1e5, a=0.5,
                              b=0.1, f0=0.1)
    p.faults[0].normal_loading_dot[:] = 1.0
    return p


@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
def test_extensional_traction_stops_at_the_oracle_step(mode):
    p = unloading_fault(mode)
    o = Oracle(p, threads=4)
    o.use_dense()
    st_o, _ = o.solve_steps(5000)
    r = o.state()
    assert st_o == DFN_ERR_EXTENSIONAL
    with Simulation(p, pressure="cg") as s:
        with pytest.raises(DfnError) as e:
            s.solve_steps(5000)
        assert e.value.status == DFN_ERR_EXTENSIONAL
        g = s.state()
    N = len(r["P"])
    assert g["it_count"] == r["it_count"]
    # the failing step is committed (time, state) before the rule stops the run
    assert abs(g["time"] - r["time"]) <= 1e-9 * r["time"] and g["time"] > 1e5
    assert np.abs(g["Y"][:N] - r["Y"][:N]).max() <= 1e-8 * np.abs(r["Y"][:N]).max()
    assert np.abs(g["Y"][2 * N:] - r["Y"][2 * N:]).max() <= 1e-8 * np.abs(r["Y"][2 * N:]).max()
    assert (g["Y"][2 * N:] > 0).any()


def test_rkqs_step_underflow_like_the_oracle():
    """rkqs from x = 1e20 with a tolerance no step meets: the first shrunk
    step no longer changes x, and both stop with the underflow status."""
    p = networks.single_fault(n_el=200, length=2000.0, mode="modeIII", q_kgs=0.0, tol=1e-6)
    Y = build_arrays(p).Y0()
    x = 1e20
    o = Oracle(p)
    o.use_dense()
    dydx = o.friction_law(x, Y)
    yscal = np.abs(Y) + np.abs(dydx * 1e3) + 1e-6
    with pytest.raises(RuntimeError, match="status 2"):
        o.rkqs(Y, dydx, x, 1e3, 1e-300, yscal)
    with Simulation(p, pressure="cg") as s:
        with pytest.raises(DfnError) as e:
            s.rkqs(Y, dydx, x, 1e3, 1e-300, yscal)
        assert e.value.status == DFN_ERR_UNDERFLOW


def test_nonfinite_state_is_rejected_and_the_handle_goes_on():
    p = networks.small_network(seed=31, n_faults=3, tol=1e-6)
    a = build_arrays(p)
    with Simulation(p, pressure="tridiag") as s:
        st = s.state()
        for bad in (np.nan, np.inf):
            Y = st["Y"].copy()
            Y[1] = bad
            with pytest.raises(DfnError) as e:
                s.set_state(Y, st["P"], st["time"], st["t_try"])
            assert e.value.status == DFN_ERR_NONFINITE
        P = st["P"].copy()
        P[0] = np.nan
        outs = [np.empty(a.N) for _ in range(5)]
        with pytest.raises(DfnError) as e:
            s.step_host(st["Y"], P, st["time"], st["t_try"], outs)
        assert e.value.status == DFN_ERR_NONFINITE
        rep = s.solve_steps(5)
        assert rep["status"] == 0 and rep["it_count"] == 5
    bad = networks.small_network(seed=31, n_faults=3, tol=1e-6)
    bad.faults[1].V[2] = np.nan
    with pytest.raises(DfnError) as e:
        Simulation(bad)
    assert e.value.status == DFN_ERR_NONFINITE


def hopeless_fault():
    """A fault no RK attempt can satisfy (tol 1e-300), without pore pressure
    (its CG converges at once at any tolerance)."""
    return networks.single_fault(n_el=300, length=3000.0, mode="modeII", q_kgs=0.0, tol=1e-300)


def test_attempt_budget_stops_the_step():
    with Simulation(hopeless_fault(), pressure="cg", max_attempts=1) as s:
        with pytest.raises(DfnError) as e:
            s.solve_steps(3)
        assert e.value.status == DFN_ERR_ATTEMPTS
        g = s.state()
        assert g["it_count"] == 1 and g["time"] == 0.0


@pytest.mark.parametrize("pressure", ["cg", "tridiag"])
def test_failing_network_leaves_the_batch_bitwise(pressure):
    ok = [networks.small_network(seed=s, n_faults=n, tol=1e-6, q_kgs=q) for s, n, q in ((41, 3, 20.0), (42, 4, 40.0))]
    ps = [ok[0], hopeless_fault(), ok[1]]
    t_end = 4000.0
    with Ensemble(ps, pressure=pressure) as ens:
        reps = ens.solve(t_end=t_end, check=False)
        assert reps[1]["status"] == DFN_ERR_ATTEMPTS
        assert reps[0]["status"] == 0 and reps[2]["status"] == 0
        got = [ens.state(0), ens.state(2)]
    for p, a in zip(ok, got):
        assert abs(a["time"] - t_end) <= 1e-12 * t_end
        with Simulation(p, pressure=pressure) as s:
            s.solve_to(t_end)
            b = s.state()
        assert a["it_count"] == b["it_count"] and a["time"] == b["time"]
        assert np.array_equal(a["Y"], b["Y"]) and np.array_equal(a["P"], b["P"])


@pytest.mark.parametrize("storage", ["fp64", "fp32"])
def test_bounded_wait_expiry_reports_timeout(storage):
    """With zero polls every wait of the TMA K.V pipeline gives up at once:
    the kernel drains its own copies with the full limit, raises the flag,
    and the call reports DFN_ERR_TIMEOUT once. After the default limit is
    back and the state is restored, the handle follows a fresh handle bit
    for bit."""
    p = networks.small_network(seed=33, n_faults=4, tol=1e-6)
    with Simulation(p, storage=storage, pressure="tridiag", gemv="tma") as s:
        s.solve_steps(3)
        st = s.state()
        s.set_wait_limit(0)
        with pytest.raises(DfnError) as e:
            s.solve_steps(1)
        assert e.value.status == DFN_ERR_TIMEOUT
        s.set_wait_limit(None)
        s.set_state(st["Y"], st["P"], st["time"], st["t_try"], st["it_count"])
        s.solve_steps(12)
        g = s.state()
        v = np.random.default_rng(0).normal(size=s.N)
        kv = s.kernel(v)
    with Simulation(p, storage=storage, pressure="tridiag", gemv="tma") as r:
        r.set_state(st["Y"], st["P"], st["time"], st["t_try"], st["it_count"])
        r.solve_steps(12)
        h = r.state()
        kr = r.kernel(v)
    assert g["time"] == h["time"] and np.array_equal(g["Y"], h["Y"]) and np.array_equal(g["P"], h["P"])
    assert np.array_equal(kv[0], kr[0]) and np.array_equal(kv[1], kr[1])
