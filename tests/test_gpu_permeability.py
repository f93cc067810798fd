"""Permeability evolution (permeability_coupling = 1) on the GPU against the
oracle: before every pressure solve the permeability follows the committed
sigmaN and P, k = (k* - kmin) exp(-|sigmaN + P| / |Snk|) + kmin
(src/fluid_diffusion.f90:68-70), with k* fixed from the initial state
(src/initialisation.f90:256-261); the commit solve of a step sees the new
sigmaN and the old P, as the reference's compute_P(t_did) after rkqs.

Tolerances as the other whole-run tests: state, pressure and time within
1e-8 of the oracle; the permeability of the last solve within 1e-12."""
import numpy as np
import pytest

from oracle import Oracle
from demystification_dfn_b200 import networks
from demystification_dfn_b200._lib import DfnError
from demystification_dfn_b200.simulation import Simulation
from test_oracle import coupled_fault

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("pressure", ["cg_exact", "cg"])
def test_permeability_coupling_matches_oracle(pressure):
    """(The exact tridiagonal solve is not in this comparison: on this
    problem the reference's CG stalls at its cap for the trial step of a
    later step, and the probe halves t_try, which an exact solve never
    does.)"""
    p = coupled_fault()
    o = Oracle(p)
    o.use_dense()
    with Simulation(p, pressure=pressure) as s:
        rep = s.solve_steps(30)
        g = s.state()
        snap = s.snapshot()
    st, _ = o.solve_steps(30)
    r = o.state()
    assert st == 0 and rep["status"] == 0
    assert abs(g["time"] - r["time"]) <= 1e-8 * r["time"]
    N = len(r["P"])
    for j in range(3):
        assert rel(g["Y"][j * N:(j + 1) * N], r["Y"][j * N:(j + 1) * N]) < 1e-8, j
    assert rel(g["P"], r["P"]) < 1e-8
    k0 = s.arrays.permeability
    assert rel(snap["permeability"], o.permeability()) < 1e-12
    assert (snap["permeability"] / k0).max() > 1.05     # the coupling moved it


def test_permeability_coupling_batch_equals_single():
    ps = [coupled_fault(n_el=300), coupled_fault(n_el=420, Snk=10e6)]
    from demystification_dfn_b200.ensemble import Ensemble

    with Ensemble(ps, pressure="tridiag") as e:
        e.solve(n_steps=12)
        for i, p in enumerate(ps):
            with Simulation(p, pressure="tridiag") as s:
                s.solve_steps(12)
                a, b = e.state(i), s.state()
                assert a["time"] == b["time"] and np.array_equal(a["Y"], b["Y"]) and np.array_equal(a["P"], b["P"])


def test_permeability_coupling_limits():
    """Outside what is built: the Newton formulation (its state holds sigmaN
    at slip 0, not the traction) and networks with fault crossings (their
    coupling coefficients hold the permeabilities of set-up)."""
    with pytest.raises(DfnError) as e:
        Simulation(coupled_fault(), formulation="newton")
    assert e.value.status == 7
    c = networks.crossing_pair(n_el=40)
    c.hyperparameter.permeability_coupling = 1
    for f in c.faults:
        f.kmin[:] = 1e-16
        f.Snk[:] = 20e6
    with pytest.raises(DfnError) as e:
        Simulation(c, pressure="cg")
    assert e.value.status == 7
