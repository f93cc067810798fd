"""Seeded synthetic problems with the shapes of the benchmark workloads.

* :func:`single_fault` — one straight fault (40 km, 4000 x 10 m elements),
  rate-strengthening aging law, constant-rate injection at the centre driving
  1D diffusion (diffusivity 0.1 m^2/s).
* :func:`fault_network` — seeded random network: centres uniform in a square,
  lengths log-uniform, strikes normal, 10 m elements, per-fault friction with
  lognormal noise, a pore-pressure step on one fault.

Injection rates are given in kg/s by the workload descriptions while the
reference's ``Q`` is a volume flux in m/s. The conversion used here is
``Q = q / (rho_f * A_ref)`` with ``A_ref = 4e4 m^2`` (a 40 km fault times
1 m of out-of-plane width); it maps 50 kg/s to 1.25e-6 m/s, the value of the
reference's single-fault injection script (wrapper_python/BP6QD_A.py:105).

Faults of a random network are drawn by rejection so that no two faults come
closer than ``min_gap`` (one element length by default): crossing faults put
element midpoints on top of other faults' nodes, where the kernel is singular.
"""
from __future__ import annotations

import numpy as np

from .problem import DemystiFicatioN

A_REF = 4.0e4   # m^2, kg/s -> m/s conversion area (see module docstring)
YEAR = 365.25 * 86400.0


def kgs_to_Q(q_kgs, rho=1000.0):
    return q_kgs / (rho * A_REF)


def _material(problem, mu=32e9, cs=3464.0, poisson=0.25):
    ml = problem.material_loading
    ml.mu = mu
    ml.cs = cs
    # cp/cs = sqrt(2(1-nu)/(1-2nu)) = sqrt(3) at nu = 0.25
    ml.cp = cs * np.sqrt(2.0 * (1.0 - poisson) / (1.0 - 2.0 * poisson))
    ml.Sigma11_dot = ml.Sigma12_dot = ml.Sigma22_dot = ml.Sigma31_dot = ml.Sigma32_dot = 0.0
    ml.normal_loading_dot = 0.0
    ml.shear_loading_dot = 0.0
    # diffusivity k/(phi mu_f (bf+br)) = 0.1 m^2/s with k = 1e-13
    ml.rock_comp = 0.1e-8
    ml.fluid_comp = 0.9e-8
    ml.fluid_density = 1000.0
    ml.porosity = 0.1
    ml.dyn_viscosity = 1e-3


def diffusivity(problem, permeability):
    ml = problem.material_loading
    return permeability / (ml.porosity * ml.dyn_viscosity * (ml.fluid_comp + ml.rock_comp))


def single_fault(n_el=4000, length=40e3, mode="modeII", a=0.007, b=0.005, Dc=4e-3, f0=0.6, V0=1e-6,
                 sigmaN=-50e6, V_init=1e-12, q_kgs=50.0, t_inj=(0.0, YEAR), permeability=1e-13,
                 tol=1e-8, max_it=10, name="single_fault", kernel="direct"):
    p = DemystiFicatioN(1)
    hp = p.hyperparameter
    hp.simulation_name = name
    hp.fracture_mode = mode
    hp.static_kernel = kernel
    hp.friction_law = "RateStateAging"
    hp.tol_solver = tol
    hp.freq_writing_file = 1000
    hp.max_it = max_it
    hp.stride_time = 1
    _material(p)
    f = p.faults[0]
    f.nb_element = int(n_el)
    f.a[:] = a
    f.b[:] = b
    f.Dc[:] = Dc
    f.f0[:] = f0
    f.V0[:] = V0
    f.sigmaN[:] = sigmaN
    f.V[:] = V_init
    f.theta[:] = np.log(V0 / V_init)        # steady state: theta = Dc/V
    f.P[:] = 0.0
    f.permeability[:] = permeability
    x = np.linspace(-length / 2, length / 2, n_el + 1)
    f.node[0, :] = x
    f.node[1, :] = 0.0
    if q_kgs:
        f.nb_source = 1
        f.Q[:] = kgs_to_Q(q_kgs)
        f.t_injection_beg[:] = t_inj[0]
        f.t_injection_end[:] = t_inj[1]
        mid = 0.5 * (x[1:] + x[:-1])
        f.index_injection[:] = int(np.argmin(np.abs(mid))) + 1
    return p


def crossing_pair(n_el=100, length=1000.0, angle_deg=60.0, mode="modeII", shift=0.0, P1=1e6, q_kgs=0.0,
                  permeability=1e-13, tol=1e-8, **kw):
    """Two straight faults of n_el elements (n_el even) crossing at their
    middle nodes (a fault crossing in the sense of find_fault_crossing,
    src/initialisation.f90:279-344): fault 1 along x, fault 2 at angle_deg,
    moved by ``shift`` metres along y (shift 0: the middle nodes coincide).
    Fault 1 starts at pore pressure P1, fault 2 at 0."""
    if n_el % 2:
        raise ValueError("n_el must be even (the faults cross at their middle nodes)")
    p = single_fault(n_el=n_el, length=length, mode=mode, q_kgs=q_kgs, permeability=permeability, tol=tol,
                     name="crossing_pair", **kw)
    base = p.faults[0]
    q = DemystiFicatioN(2)
    q.hyperparameter = p.hyperparameter
    q.hyperparameter.nb_fault = 2
    q.material_loading = p.material_loading
    th = np.deg2rad(angle_deg)
    s = np.linspace(-length / 2, length / 2, n_el + 1)
    for i, f in enumerate(q.faults):
        f.nb_element = n_el
        for name in ("a", "b", "Dc", "f0", "V0", "sigmaN", "V", "theta", "permeability"):
            getattr(f, name)[:] = getattr(base, name)
        f.P[:] = P1 if i == 0 else 0.0
        if i == 0:
            f.node[0, :] = s
            f.node[1, :] = 0.0
        else:
            f.node[0, :] = s * np.cos(th)
            f.node[1, :] = s * np.sin(th) + shift
    if q_kgs:
        f0 = q.faults[0]
        f0.nb_source = 1
        f0.Q[:] = base.Q
        f0.t_injection_beg[:] = base.t_injection_beg
        f0.t_injection_end[:] = base.t_injection_end
        f0.index_injection[:] = base.index_injection
    return q


def _seg_dist(p1, p2, q1, q2):
    """Minimum distance between segment p1-p2 and segments q1-q2 (arrays)."""
    def pt_seg(p, a, b):
        ab = b - a
        t = np.clip(np.einsum("ij,ij->i", p - a, ab) / np.maximum(np.einsum("ij,ij->i", ab, ab), 1e-300), 0, 1)
        return np.linalg.norm(p - (a + t[:, None] * ab), axis=1)

    P1 = np.broadcast_to(p1, q1.shape)
    P2 = np.broadcast_to(p2, q1.shape)
    d = np.minimum.reduce([pt_seg(P1, q1, q2), pt_seg(P2, q1, q2), pt_seg(q1, P1, P2), pt_seg(q2, P1, P2)])
    # proper intersection test
    def orient(a, b, c):
        return np.sign((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0]))

    o1, o2 = orient(P1, P2, q1), orient(P1, P2, q2)
    o3, o4 = orient(q1, q2, P1), orient(q1, q2, P2)
    cross = (o1 * o2 < 0) & (o3 * o4 < 0)
    d[cross] = 0.0
    return d


def fault_network(n_faults=800, box=7000.0, seed=0, length_range=(50.0, 500.0), strike_deg=(30.0, 10.0),
                  ds=10.0, a=0.010, b=0.015, noise=0.10, Dc=1e-3, f0=0.6, V0=1e-6, sigmaN=-50e6, V_init=1e-12,
                  dP=10e6, permeability=1e-13, mode="modeII", tol=1e-8, max_it=10, min_gap=None,
                  q_kgs=None, name=None, kernel="direct", v_load=0.0):
    """Seeded random fault network (see module docstring). ``v_load`` (m/s)
    adds tectonic shear loading: each fault's shear_loading_dot is
    mu * v_load / L_f (its own length as the stiffness scale of the
    equivalent slip rate), e.g. 0.06-0.6 Pa/s for 1e-9 m/s on 50-500 m faults."""
    rng = np.random.default_rng(seed)
    gap = ds if min_gap is None else min_gap
    lo, hi = np.log(length_range[0]), np.log(length_range[1])
    segs = np.zeros((0, 4))
    specs = []
    tries = 0
    while len(specs) < n_faults:
        tries += 1
        if tries > 200 * n_faults:
            raise RuntimeError("could not place the faults without overlaps; lower n_faults or min_gap")
        c = rng.uniform(0.0, box, 2)
        L = float(np.exp(rng.uniform(lo, hi)))
        th = np.deg2rad(rng.normal(strike_deg[0], strike_deg[1]))
        d = 0.5 * L * np.array([np.cos(th), np.sin(th)])
        p1, p2 = c - d, c + d
        if len(segs):
            dist = _seg_dist(p1[None, :], p2[None, :], segs[:, :2], segs[:, 2:])
            if np.any(dist < gap):
                continue
        segs = np.vstack([segs, np.concatenate([p1, p2])[None, :]])
        specs.append((p1, p2, L))
    p = DemystiFicatioN(n_faults)
    hp = p.hyperparameter
    hp.simulation_name = name or f"network_{n_faults}_seed{seed}"
    hp.fracture_mode = mode
    hp.static_kernel = kernel
    hp.friction_law = "RateStateAging"
    hp.tol_solver = tol
    hp.freq_writing_file = 1000
    hp.max_it = max_it
    hp.stride_time = 1
    _material(p)
    stepped = int(rng.integers(n_faults))
    for i, (p1, p2, L) in enumerate(specs):
        f = p.faults[i]
        n = max(1, int(round(L / ds)))
        f.nb_element = n
        t = np.linspace(0.0, 1.0, n + 1)
        f.node[0, :] = p1[0] + t * (p2[0] - p1[0])
        f.node[1, :] = p1[1] + t * (p2[1] - p1[1])
        f.a[:] = a * np.exp(rng.normal(0.0, noise))
        f.b[:] = b * np.exp(rng.normal(0.0, noise))
        f.Dc[:] = Dc
        f.f0[:] = f0
        f.V0[:] = V0
        f.sigmaN[:] = sigmaN
        f.V[:] = V_init * np.exp(rng.normal(0.0, noise, n))
        f.theta[:] = np.log(V0 / f.V)
        f.P[:] = 0.0
        f.permeability[:] = permeability
        if v_load:
            f.shear_loading_dot[:] = p.material_loading.mu * v_load / L
        if i == stepped:
            # pressure step on the first half of the chosen fault; it diffuses
            # along the fault so that dP/dt drives the friction law
            f.P[: max(1, n // 2)] = dP
        if q_kgs is not None and i == stepped:
            f.nb_source = 1
            f.Q[:] = kgs_to_Q(q_kgs)
            f.t_injection_beg[:] = 0.0
            f.t_injection_end[:] = YEAR
            f.index_injection[:] = max(1, n // 2)
    p.stepped_fault = stepped + 1
    return p


def ensemble_member(seed, n_faults=None, q_kgs=None, diffusivity=None, ref_faults=800, ref_box=7000.0, **kw):
    """One realisation of the network ensemble: 100-400 faults drawn like
    :func:`fault_network` (the box scaled to keep the fault density of 800
    faults in 7 km x 7 km), one point injection of 10-100 kg/s at the centre
    of a random fault, and a log-uniform diffusivity in 0.01-1 m^2/s."""
    rng = np.random.default_rng(10_000 + seed)
    n = int(rng.integers(100, 401)) if n_faults is None else int(n_faults)
    q = float(rng.uniform(10.0, 100.0)) if q_kgs is None else float(q_kgs)
    D = float(np.exp(rng.uniform(np.log(0.01), np.log(1.0)))) if diffusivity is None else float(diffusivity)
    box = ref_box * np.sqrt(n / ref_faults)
    # permeability giving diffusivity D with the module's fluid constants
    perm = D * 0.1 * 1e-3 * (0.9e-8 + 0.1e-8)
    p = fault_network(n_faults=n, box=box, seed=seed, dP=0.0, permeability=perm, q_kgs=q,
                      name=f"ensemble_{seed}", **kw)
    p.diffusivity = D
    return p


def ensemble(count=64, seed0=0, **kw):
    return [ensemble_member(seed0 + i, **kw) for i in range(count)]


def small_network(seed=0, n_faults=4, mode="modeII", **kw):
    """A few-fault network for exhaustive parity tests (N of a few hundred)."""
    kw.setdefault("box", 600.0)
    kw.setdefault("length_range", (40.0, 160.0))
    return fault_network(n_faults=n_faults, seed=seed, mode=mode, **kw)


def shared_geometry_ensemble(count, base=None, seed=0, noise=0.10, **kw):
    """``count`` realisations of one fault network (same faults, nodes and
    elastic constants, so one kernel matrix serves all of them): each member
    redraws the per-fault a and b (lognormal ``noise``), the initial slip
    rates and the fault that carries the pore-pressure step, from its own
    seed. ``base`` defaults to :func:`fault_network` with ``seed`` and ``kw``."""
    import copy

    if base is None:
        base = fault_network(seed=seed, **kw)
    members = []
    for m in range(count):
        rng = np.random.default_rng(100_000 + 7919 * seed + m)
        p = copy.deepcopy(base)
        p.hyperparameter.simulation_name = f"{base.hyperparameter.simulation_name}_member{m}"
        dP = max(float(np.max(f.P)) for f in base.faults)
        stepped = int(rng.integers(len(p.faults)))
        for i, f in enumerate(p.faults):
            n = f.nb_element
            f.a[:] = np.mean(f.a) * np.exp(rng.normal(0.0, noise))
            f.b[:] = np.mean(f.b) * np.exp(rng.normal(0.0, noise))
            V = np.mean(f.V) * np.exp(rng.normal(0.0, noise, n))
            f.V[:] = V
            f.theta[:] = np.log(f.V0 / V)
            f.P[:] = 0.0
            if i == stepped:
                f.P[: max(1, n // 2)] = dP
        members.append(p)
    return members
