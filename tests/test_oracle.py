"""CPU checks of the FP64 oracle against known answers (parity unpinned:
the reference ships no golden outputs, so the restatement is pinned by the
mathematics of each routine)."""
import ctypes

import numpy as np
import pytest

from oracle import Oracle, load
from demystification_dfn_b200 import networks
from demystification_dfn_b200.layout import build_arrays, ptr


def straight(n=64, mode="modeIII", **kw):
    kw.setdefault("q_kgs", 50.0)
    return networks.single_fault(n_el=n, length=10.0 * n, mode=mode, **kw)


def test_geometry_straight_fault():
    o = Oracle(straight(32))
    g = o.geometry()
    assert np.allclose(g["ds"], 10.0, rtol=0, atol=1e-12)
    assert np.allclose(g["tangent"], [1.0, 0.0])
    assert np.allclose(g["normal"], [0.0, 1.0])
    # harmonic mean of equal permeabilities, zero at the two ends
    px = g["permeability_x"]
    assert px[0] == 0 and px[-1] == 0 and np.allclose(px[1:-1], 1e-13, rtol=1e-15)


def test_mode3_uniform_slip_telescopes_to_tips():
    # directModeIII.f:59-65: with uniform slip only the two tip nodes remain
    n = 50
    o = Oracle(straight(n))
    a = o.arrays
    sT, _ = o.kernel(np.ones(a.N))
    g = o.geometry()
    el = g["element"]
    x0, x1 = a.node[0, 0], a.node[-1, 0]
    mu = a.mu
    # I(node) = t.(e-node)/r^2 = 1/(e_x - node_x) on the x axis
    expect = mu / (2 * np.pi) * (-1.0 / (el[:, 0] - x0) + 1.0 / (el[:, 0] - x1))
    assert np.allclose(sT, expect, rtol=1e-12, atol=1e-6)


@pytest.mark.parametrize("mode", ["modeII", "modeIII"])
def test_direct_equals_dense(mode):
    p = networks.small_network(seed=3, n_faults=3, mode=mode)
    o = Oracle(p)
    rng = np.random.default_rng(0)
    v = rng.normal(size=o.N) * 1e-9
    v[o.arrays.fake_mask] = 0.0
    d_T, d_N = o.kernel(v)
    o.use_dense()
    k_T, k_N = o.kernel(v)
    scale = np.abs(d_T).max()
    if mode == "modeII":
        # identical pair terms in identical order: bitwise equal
        assert np.array_equal(d_T, k_T) and np.array_equal(d_N, k_N)
    else:
        # directIII sums node differences, the entries element differences
        assert np.allclose(d_T, k_T, rtol=0, atol=1e-11 * scale)


def test_entries_match_dense_matrix():
    p = networks.small_network(seed=5, n_faults=2)
    o = Oracle(p)
    KT, KN = o.dense()
    for (k, l) in [(0, 0), (3, 7), (o.N - 1, 2)]:
        assert KT[k, l] == o.entry(k, l, 1)
        assert KN[k, l] == o.entry(k, l, 2)


def test_steady_state_has_no_state_rate():
    o = Oracle(straight(40, q_kgs=0.0))
    Y = o.arrays.Y0()
    Yd = o.friction_law(10.0, Y)
    N = o.N
    # psi = ln(V0/V): dpsi/dt = V0/Dc e^-psi - V/Dc = 0
    assert np.abs(Yd[N:2 * N]).max() < 1e-20
    # uniform V on a straight fault with no pressure: no normal stress rate
    assert np.abs(Yd[2 * N:]).max() == 0.0


def test_fake_elements_have_zero_derivatives():
    o = Oracle(networks.small_network(seed=2, n_faults=4))
    Yd = o.friction_law(5.0, o.arrays.Y0())
    fk = o.arrays.fake_mask
    N = o.N
    assert fk.sum() == 3
    for j in range(3):
        assert np.all(Yd[j * N:(j + 1) * N][fk] == 0.0)


def test_cg_matches_exact_and_conserves_mass():
    p = straight(200, q_kgs=50.0)
    p.hyperparameter.tol_solver = 1e-6
    o = Oracle(p)
    a = o.arrays
    for dt in (10.0, 1000.0, 20000.0):
        Pt, Pd, ier = o.compute_P(dt)
        assert ier == 0
        ex = o.pressure_exact(dt)
        assert np.abs(Pt - ex).max() < 1e-3
        # implicit Euler with no-flux ends conserves the injected volume
        injected = dt * a.src_Q[0] / (a.porosity * (a.fluid_comp + a.rock_comp)) / 10.0
        assert abs(ex.sum() - a.P.sum() - injected) < 1e-9 * injected
        assert np.allclose(Pd, (Pt - a.P) / dt)


def test_cg_iteration_cap_reports_ier():
    p = straight(400, q_kgs=50.0)
    p.hyperparameter.tol_solver = 1e-14      # unreachable: max|r| < 1e-14 Pa
    o = Oracle(p)
    Pt, Pd, ier = o.compute_P(86400.0)
    assert ier == 1
    assert np.all(Pt == 0)                  # outputs untouched, as in the reference


CB = ctypes.CFUNCTYPE(None, ctypes.c_double, ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                      ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)


def _rkqs_generic(f, y0, x_end, eps=1e-8, h0=0.1):
    lib = load()
    fn = lib.orc_rkqs_cb
    fn.restype = ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    fn.argtypes = [CB, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), dp, dp, ctypes.c_int64, dp,
                   ctypes.c_double, ctypes.c_double, dp, dp, dp]

    def derivs(x, n, y, dy, ctx):
        yy = np.ctypeslib.as_array(y, shape=(n,))
        out = f(x, yy)
        for i in range(n):
            dy[i] = out[i]

    cb = CB(derivs)
    y = np.array(y0, dtype=float)
    x, h, steps = 0.0, h0, 0
    cnt = (ctypes.c_int64 * 2)()
    while x < x_end - 1e-12:
        h = min(h, x_end - x)
        dydx = np.array(f(x, y))
        yscal = np.abs(y) + np.abs(dydx * h) + 1e-30
        xx, hd, hn = ctypes.c_double(x), ctypes.c_double(), ctypes.c_double()
        assert fn(cb, None, cnt, ptr(y), ptr(dydx), y.size, ctypes.byref(xx), h, eps, ptr(yscal),
                  ctypes.byref(hd), ctypes.byref(hn)) == 0
        x, h = xx.value, hn.value
        steps += 1
    return y, steps


def test_rkqs_exponential_decay():
    y, steps = _rkqs_generic(lambda x, y: -y, [1.0], 5.0)
    assert abs(y[0] - np.exp(-5.0)) < 1e-9 and steps < 200


def test_rkqs_cosine():
    y, _ = _rkqs_generic(lambda x, y: [np.cos(x)], [0.0], 3.0)
    assert abs(y[0] - np.sin(3.0)) < 1e-8


def test_solve_loop_policies():
    p = straight(80, q_kgs=50.0, tol=1e-6)
    p.faults[0].t_injection_beg[:] = 5000.0   # clamp to 10 s before the injection starts
    o = Oracle(p)
    st, log = o.solve_steps(12)
    assert st == 0
    s = o.state()
    assert s["it_count"] == 12
    assert np.isclose(s["time"], log.sum(), rtol=1e-12)
    assert log.max() <= 86400.0
    assert o.counters()["rhs_evals"] >= 6 * 12


def test_fault_crossing_couples_the_pressure():
    """find_fault_crossing restated: two faults sharing a node cross once;
    fluid at 1 MPa on fault 1 reaches the elements of fault 2 around the
    crossing in one implicit step (and only near it), while the same faults
    1 m apart stay decoupled (fault 2 keeps exactly 0)."""
    n = 100
    p = networks.crossing_pair(n_el=n, shift=0.0)
    o = Oracle(p)
    assert o.crossings() == 1
    Pt, _, ier = o.compute_P(3600.0)
    assert ier == 0
    f2 = Pt[n + 1:]
    near, far = f2[n // 2 - 1:n // 2 + 1], np.concatenate([f2[:5], f2[-5:]])
    assert near.min() > 1e5 and np.abs(far).max() < 1e-3 * near.min()
    assert Pt[n // 2 - 1:n // 2 + 1].max() < 1e6        # fault 1 loses fluid at the crossing
    o2 = Oracle(networks.crossing_pair(n_el=n, shift=1.0))
    assert o2.crossings() == 0
    Pt2, _, _ = o2.compute_P(3600.0)
    assert np.all(Pt2[n + 1:] == 0.0)


def test_shipped_network_has_fault_crossings():
    """The reference's shipped 10-fault network shares nodes between faults
    (13 crossings by the reference's criterion)."""
    import refconfigs

    o = Oracle(refconfigs.problem("network"))
    assert o.crossings() == 13


def _run_capped(p, form, hmax, T):
    """The oracle in one formulation with every step capped at hmax (the
    first one too), to simulated time T."""
    o = Oracle(p)
    o.use_dense()
    o.set_formulation(form)
    o.set_max_step(hmax)
    s = o.state()
    o.set_state(s["Y"], s["P"], s["time"], hmax, 0)
    st, _ = o.solve_steps(int(round(T / hmax)))
    assert st == 0 and abs(o.state()["time"] - T) <= 1e-9 * T
    return o


def test_newton_restatement_agrees_with_the_v_formulation_without_pressure():
    """Without pore-pressure forcing the two formulations integrate the same
    ODE (the reference's dV/dt is the time derivative of the friction law the
    Newton formulation solves). With the same steps (a tolerance every
    attempt meets, steps capped at 10 s) slip rate and slip agree to 1e-9;
    the Newton formulation's first V is the initial V (a root of the friction
    law at slip 0, to the Newton tolerance)."""
    p = networks.small_network(seed=31, n_faults=4, tol=1e-3, dP=0.0)
    real = ~build_arrays(p).fake_mask
    o = Oracle(p)
    o.set_formulation("newton")
    V0 = build_arrays(p).Y0()[:o.N]
    # the Newton residual test (1e-13 of the stress) resolves w to about
    # 1e-13 w, so V = (2 V0/C) sinh w to about 1e-11
    assert np.abs(o.velocity() - V0)[real].max() <= 1e-10 * np.abs(V0).max()
    a, b = _run_capped(p, "v", 10.0, 600.0), _run_capped(p, "newton", 10.0, 600.0)
    for x, y in ((b.velocity(), a.velocity()), (b.slip(), a.slip())):
        assert np.abs(x - y)[real].max() <= 1e-9 * np.abs(y).max()
    assert b.newton_counters()["fail"] == 0


def test_formulation_gap_under_pressure_is_first_order_in_the_step():
    """With a 10 MPa pore-pressure step diffusing along one fault the two
    formulations differ at O(h): the reference's V formulation takes the
    pressure of each stage as an implicit-Euler step from the committed P
    and its secant rate, the Newton formulation interpolates P linearly over
    the step. Halving the step cap halves their gap in slip rate and slip
    (both converge to the same solution)."""
    p = networks.small_network(seed=9, n_faults=4, tol=1e-3)
    real = ~build_arrays(p).fake_mask
    gaps = []
    for hmax in (20.0, 10.0, 5.0):
        a, b = _run_capped(p, "v", hmax, 400.0), _run_capped(p, "newton", hmax, 400.0)
        Va, Vb = a.velocity(), b.velocity()
        gaps.append(np.abs(Vb - Va)[real].max() / np.abs(Va).max())
    assert gaps[0] > 0.02
    for g1, g2 in zip(gaps, gaps[1:]):
        assert 1.8 <= g1 / g2 <= 2.2, gaps


def coupled_fault(kmin=1e-16, Snk=20e6, n_el=500):
    """One 5 km fault with 50 kg/s injection and permeability coupling
    (permeability_coupling = 1): permeability grows as the pore pressure
    lowers the effective normal stress."""
    p = networks.single_fault(n_el=n_el, length=10.0 * n_el, mode="modeII", tol=1e-6, q_kgs=50.0)
    p.hyperparameter.permeability_coupling = 1
    for f in p.faults:
        f.kmin[:] = kmin
        f.Snk[:] = Snk
    return p


def test_permeability_coupling_follows_the_committed_state():
    """k* = kmin + (k - kmin) exp(|sigmaN + P| / |Snk|) at the start
    (src/initialisation.f90:256-261), then before every pressure solve
    k = (k* - kmin) exp(-|sigmaN + P| / |Snk|) + kmin from the committed state
    (src/fluid_diffusion.f90:68-70): the initial permeability is recovered,
    and after some steps the permeability at the injection has grown."""
    p = coupled_fault()
    a = build_arrays(p)
    o = Oracle(p)
    o.use_dense()
    o.compute_P(10.0)
    assert np.allclose(o.permeability(), a.permeability, rtol=1e-14, atol=0.0)
    st, _ = o.solve_steps(20)
    assert st == 0
    s = o.state()
    N = o.N
    o.compute_P(10.0)
    kstar = a.kmin + (a.permeability - a.kmin) * np.exp(np.abs(a.sigmaN + a.P) / np.abs(a.Snk))
    expect = (kstar - a.kmin) * np.exp(-np.abs(s["Y"][2 * N:] + s["P"]) / np.abs(a.Snk)) + a.kmin
    k = o.permeability()
    assert np.allclose(k, expect, rtol=1e-13, atol=0.0)
    src = int(np.argmax(s["P"]))
    assert k[src] > 1.05 * a.permeability[src]
    # the coupled run differs from the uncoupled one
    q = networks.single_fault(n_el=500, length=5000.0, mode="modeII", tol=1e-6, q_kgs=50.0)
    o2 = Oracle(q)
    o2.use_dense()
    o2.solve_steps(20)
    assert np.abs(o2.state()["P"] - s["P"]).max() > 1e-3 * np.abs(s["P"]).max()
