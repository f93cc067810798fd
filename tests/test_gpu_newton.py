"""Slip against the oracle, in both formulations.

* V formulation (the reference's ODE, src/friction/RateStateAgingModeII.f90):
  slip is carried by the same Cash-Karp stages as a passive component
  outside the error norm (the reference allocates slip and never updates it,
  src/configuration.f90:190). GPU and oracle integrate it with the same
  5th-order combination: slip within 1e-8 of the oracle's.
* Newton slip formulation (DFN_FORM_NEWTON: state [slip, psi, sigmaN0], V
  solved from the friction law at every stage, pressure linear in the stage
  time): the oracle restates it (oracle/dfn_oracle.c, orc_newton_*), and the
  GPU FP64 path must follow it with pore pressure on (a 10 MPa pressure step
  diffusing along one fault, and a 50 kg/s injection): slip, log-state,
  slip rate, pressure and time within 1e-8 over 25 steps.

Tolerances are relative to the largest magnitude of the compared quantity.
"""
import numpy as np
import pytest

from oracle import Oracle
from demystification_dfn_b200 import networks
from demystification_dfn_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("pressure", ["cg_exact", "tridiag"])
def test_v_formulation_slip_matches_oracle(pressure):
    p = networks.small_network(seed=9, n_faults=4, tol=1e-6)
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, pressure=pressure) as s:
        s.solve_steps(25)
        g, gs = s.state(), s.slip()
    st, _ = o.solve_steps(25)
    assert st == 0
    r, rs = o.state(), o.slip()
    assert g["it_count"] == r["it_count"] == 25
    assert np.abs(rs).max() > 0
    assert rel(gs, rs) < 1e-8
    # slip is the time integral of V: between two steps it grows by about h V
    N = len(r["P"])
    assert np.all(gs[~s.arrays.fake_mask] > 0) and np.all(gs[s.arrays.fake_mask] == 0)
    assert rel(g["Y"][:N], r["Y"][:N]) < 1e-8


def newton_cases():
    pressure_step = networks.small_network(seed=9, n_faults=4, tol=1e-6)
    injection = networks.single_fault(n_el=500, length=5000.0, mode="modeII", tol=1e-6, q_kgs=50.0)
    return {"pressure_step": pressure_step, "injection": injection}


@pytest.mark.parametrize("case", ["pressure_step", "injection"])
def test_newton_formulation_matches_oracle_with_pore_pressure(case):
    p = newton_cases()[case]
    o = Oracle(p, threads=4)
    o.use_dense()
    o.set_formulation("newton")
    with Simulation(p, formulation="newton", pressure="cg_exact") as s:
        N = s.N
        # the initial V is a root of the friction law at slip 0 (both to the
        # Newton tolerance, 1e-13 of the stress: about 1e-11 in V)
        assert rel(s.velocity(), o.velocity()) < 1e-10
        rep = s.solve_steps(25)
        g, gv = s.state(), s.velocity()
    st, _ = o.solve_steps(25)
    r, rv = o.state(), o.velocity()
    assert st == 0 and rep["status"] == 0 and rep["newton_fail"] == 0
    assert g["it_count"] == r["it_count"] == 25
    assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
    assert np.abs(r["P"]).max() > 1e5          # pore pressure is on
    assert rel(g["Y"][:N], r["Y"][:N]) < 1e-8, "slip"
    assert rel(g["Y"][N:2 * N], r["Y"][N:2 * N]) < 1e-8, "log-state"
    assert rel(gv, rv) < 1e-8, "slip rate"
    assert rel(g["P"], r["P"]) < 1e-8, "pressure"
    c = o.newton_counters()
    assert c["fail"] == 0 and c["solves"] > 0
