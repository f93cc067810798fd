"""Concatenated element layout of a fault network.

Restates how the reference lays a network out in memory after reading its
``config`` (src/configuration.f90:115-300): the faults' elements are
concatenated in fault order with ONE extra "fake" element between two
consecutive faults (it joins the last node of fault f to the first node of
fault f+1), so ``nb_element = sum(n_f) + nb_fault - 1`` and
``nb_node = nb_element + 1`` (src/configuration.f90:126,136). Fake elements get
the reader's presets ``a = b = Dc = f0 = V0 = 1`` (:199-203) and zero state,
loading and permeability (the reference leaves them uninitialised; zero is
what its allocator hands back in practice and what keeps them inert).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

MODE = {"modeII": 2, "modeIII": 3}
KERNEL = {"direct": 0, "hmatrix": 1}


@dataclass
class ProblemArrays:
    N: int
    fault_nb_element: np.ndarray
    fracture_mode: int
    static_kernel: int
    node: np.ndarray            # (N+1, 2) C order == Fortran node(2, nb_node)
    a: np.ndarray
    b: np.ndarray
    Dc: np.ndarray
    f0: np.ndarray
    V0: np.ndarray
    V: np.ndarray
    theta: np.ndarray
    sigmaN: np.ndarray
    P: np.ndarray
    normal_loading_dot: np.ndarray
    shear_loading_dot: np.ndarray
    permeability: np.ndarray
    mu: float
    cp: float
    cs: float
    Sigma11_dot: float
    Sigma12_dot: float
    Sigma22_dot: float
    Sigma31_dot: float
    Sigma32_dot: float
    rock_comp: float
    fluid_comp: float
    fluid_density: float
    porosity: float
    dyn_viscosity: float
    src_fault: np.ndarray
    src_index: np.ndarray
    src_Q: np.ndarray
    src_t_beg: np.ndarray
    src_t_end: np.ndarray
    tol_solver: float
    time0: float = 0.0
    max_it: int = 10
    stride_time: int = 1
    freq_writing_file: int = 10
    simulation_name: str = "test"
    permeability_coupling: int = 0
    kmin: np.ndarray = None     # [N] (fake elements 0)
    Snk: np.ndarray = None      # [N] (fake elements 1, the reader's preset)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def fault_first(self):
        """0-based first element of each fault (mapping_fault(f,1)-1)."""
        n = self.fault_nb_element
        return np.concatenate([[0], np.cumsum(n[:-1] + 1)]).astype(np.int64)

    @property
    def fake_mask(self):
        m = np.zeros(self.N, dtype=bool)
        idx = np.cumsum(self.fault_nb_element + 1)
        idx = idx[idx <= self.N]
        m[idx - 1] = True
        return m

    def Y0(self):
        return np.concatenate([self.V, self.theta, self.sigmaN])


def _arr(x, n, name):
    a = np.asarray(x, dtype=np.float64).reshape(-1)
    if a.size == 1 and n != 1:
        a = np.full(n, float(a[0]))
    if a.size != n:
        raise ValueError(f"{name}: expected {n} values, got {a.size}")
    return a


def build_arrays(problem) -> ProblemArrays:
    """Concatenate a :class:`DemystiFicatioN` problem into reference layout."""
    hp, ml = problem.hyperparameter, problem.material_loading
    faults = problem.faults
    F = len(faults)
    if F < 1:
        raise ValueError("a problem needs at least one fault")
    nfe = np.array([int(f.nb_element) for f in faults], dtype=np.int64)
    N = int(nfe.sum() + F - 1)
    first = np.concatenate([[0], np.cumsum(nfe[:-1] + 1)]).astype(np.int64)
    node = np.zeros((N + 1, 2))
    per = {k: np.zeros(N) for k in ("a", "b", "Dc", "f0", "V0", "V", "theta", "sigmaN", "P",
                                     "normal_loading_dot", "shear_loading_dot", "permeability")}
    for k in ("a", "b", "Dc", "f0", "V0"):
        per[k][:] = 1.0
    coupling = int(getattr(hp, "permeability_coupling", 0))
    kmin, Snk = np.zeros(N), np.ones(N)   # src/configuration.f90:224-225 (Snk = 1 between faults)
    src = {"fault": [], "index": [], "Q": [], "tb": [], "te": []}
    for fi, f in enumerate(faults):
        n, s = int(f.nb_element), int(first[fi])
        nd = np.asarray(f.node, dtype=np.float64)
        if nd.shape != (2, n + 1):
            raise ValueError(f"fault {fi + 1}: node must have shape (2, {n + 1})")
        node[s:s + n + 1, :] = nd.T
        for k in per:
            per[k][s:s + n] = _arr(getattr(f, k), n, f"fault {fi + 1} {k}")
        if coupling:
            kmin[s:s + n] = _arr(getattr(f, "kmin"), n, f"fault {fi + 1} kmin")
            Snk[s:s + n] = _arr(getattr(f, "Snk"), n, f"fault {fi + 1} Snk")
        ns = int(f.nb_source)
        if ns >= 1:
            Q = _arr(f.Q, ns, "Q")
            tb = _arr(f.t_injection_beg, ns, "t_injection_beg")
            te = _arr(f.t_injection_end, ns, "t_injection_end")
            ix = np.asarray(f.index_injection, dtype=np.int64).reshape(-1)
            if ix.size == 1 and ns != 1:
                ix = np.full(ns, int(ix[0]))
            for j in range(ns):
                src["fault"].append(fi + 1)
                src["index"].append(int(ix[j]))
                src["Q"].append(Q[j])
                src["tb"].append(tb[j])
                src["te"].append(te[j])
    mode = MODE.get(hp.fracture_mode)
    if mode is None:
        raise ValueError('Please chose a fracture mode: "modeII" or "modeIII"')
    if hp.friction_law != "RateStateAging":
        raise ValueError("only the RateStateAging friction law exists in the reference")
    kern = KERNEL.get(hp.static_kernel)
    if kern is None:
        raise ValueError(f"unsupported static_kernel {hp.static_kernel!r}")
    if coupling not in (0, 1):
        raise ValueError("permeability_coupling must be 0 or 1")
    return ProblemArrays(
        N=N, fault_nb_element=nfe, fracture_mode=mode, static_kernel=kern, node=node,
        mu=float(ml.mu), cp=float(ml.cp), cs=float(ml.cs),
        Sigma11_dot=float(ml.Sigma11_dot), Sigma12_dot=float(ml.Sigma12_dot),
        Sigma22_dot=float(ml.Sigma22_dot), Sigma31_dot=float(ml.Sigma31_dot),
        Sigma32_dot=float(ml.Sigma32_dot), rock_comp=float(ml.rock_comp),
        fluid_comp=float(ml.fluid_comp), fluid_density=float(ml.fluid_density),
        porosity=float(ml.porosity), dyn_viscosity=float(ml.dyn_viscosity),
        src_fault=np.array(src["fault"], dtype=np.int64), src_index=np.array(src["index"], dtype=np.int64),
        src_Q=np.array(src["Q"], dtype=np.float64), src_t_beg=np.array(src["tb"], dtype=np.float64),
        src_t_end=np.array(src["te"], dtype=np.float64), tol_solver=float(hp.tol_solver),
        max_it=int(hp.max_it), stride_time=int(hp.stride_time),
        freq_writing_file=int(hp.freq_writing_file), simulation_name=str(hp.simulation_name),
        permeability_coupling=coupling, kmin=kmin, Snk=Snk, **per)


# ---------------------------------------------------------------------------
# ctypes mirror of include/dfn_b200.h

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int64)


class DfnProblem(ctypes.Structure):
    _fields_ = [
        ("nb_element", ctypes.c_int64), ("nb_fault", ctypes.c_int64), ("fault_nb_element", _ip),
        ("fracture_mode", ctypes.c_int32), ("static_kernel", ctypes.c_int32), ("node", _dp),
        ("a", _dp), ("b", _dp), ("Dc", _dp), ("f0", _dp), ("V0", _dp),
        ("V", _dp), ("theta", _dp), ("sigmaN", _dp), ("P", _dp),
        ("normal_loading_dot", _dp), ("shear_loading_dot", _dp), ("permeability", _dp),
        ("mu", ctypes.c_double), ("cp", ctypes.c_double), ("cs", ctypes.c_double),
        ("Sigma11_dot", ctypes.c_double), ("Sigma12_dot", ctypes.c_double), ("Sigma22_dot", ctypes.c_double),
        ("Sigma31_dot", ctypes.c_double), ("Sigma32_dot", ctypes.c_double),
        ("rock_comp", ctypes.c_double), ("fluid_comp", ctypes.c_double), ("fluid_density", ctypes.c_double),
        ("porosity", ctypes.c_double), ("dyn_viscosity", ctypes.c_double),
        ("nb_source", ctypes.c_int64), ("src_fault", _ip), ("src_index", _ip),
        ("src_Q", _dp), ("src_t_beg", _dp), ("src_t_end", _dp),
        ("tol_solver", ctypes.c_double), ("time0", ctypes.c_double),
        ("max_it", ctypes.c_int64), ("stride_time", ctypes.c_int64), ("freq_writing_file", ctypes.c_int64),
        ("permeability_coupling", ctypes.c_int64), ("kmin", _dp), ("Snk", _dp),
    ]


class DfnOptions(ctypes.Structure):
    _fields_ = [("kernel_storage", ctypes.c_int32), ("pressure_solver", ctypes.c_int32),
                ("device", ctypes.c_int32), ("max_attempts", ctypes.c_int32),
                ("gemv_impl", ctypes.c_int32), ("hmat_leaf", ctypes.c_int32), ("formulation", ctypes.c_int32),
                ("hmat_eta", ctypes.c_double), ("hmat_eps", ctypes.c_double),
                ("newton_guess", ctypes.c_int32), ("newton_maxit", ctypes.c_int32),
                ("newton_tol", ctypes.c_double), ("max_step", ctypes.c_double)]


class DfnReport(ctypes.Structure):
    _fields_ = [("it_count", ctypes.c_int64), ("attempts", ctypes.c_int64), ("rejected", ctypes.c_int64),
                ("rhs_evals", ctypes.c_int64), ("cg_iterations", ctypes.c_int64),
                ("probe_halvings", ctypes.c_int64), ("time", ctypes.c_double), ("t_try", ctypes.c_double),
                ("last_hdid", ctypes.c_double), ("status", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("stage_cg_failures", ctypes.c_int64), ("newton_solves", ctypes.c_int64),
                ("newton_iters", ctypes.c_int64), ("newton_fail", ctypes.c_int64), ("mlp_warps", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


def ptr(a, ctype=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def to_c(pa: ProblemArrays) -> DfnProblem:
    """ctypes view of the arrays (the arrays must stay alive with ``pa``)."""
    keep = []

    def d(x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        keep.append(x)
        return ptr(x)

    def i(x):
        x = np.ascontiguousarray(x, dtype=np.int64)
        if x.size == 0:
            x = np.zeros(1, dtype=np.int64)
        keep.append(x)
        return ptr(x, ctypes.c_int64)

    def dd(x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size == 0:
            x = np.zeros(1)
        keep.append(x)
        return ptr(x)

    c = DfnProblem(
        nb_element=pa.N, nb_fault=len(pa.fault_nb_element), fault_nb_element=i(pa.fault_nb_element),
        fracture_mode=pa.fracture_mode, static_kernel=pa.static_kernel, node=d(pa.node),
        a=d(pa.a), b=d(pa.b), Dc=d(pa.Dc), f0=d(pa.f0), V0=d(pa.V0), V=d(pa.V), theta=d(pa.theta),
        sigmaN=d(pa.sigmaN), P=d(pa.P), normal_loading_dot=d(pa.normal_loading_dot),
        shear_loading_dot=d(pa.shear_loading_dot), permeability=d(pa.permeability),
        mu=pa.mu, cp=pa.cp, cs=pa.cs, Sigma11_dot=pa.Sigma11_dot, Sigma12_dot=pa.Sigma12_dot,
        Sigma22_dot=pa.Sigma22_dot, Sigma31_dot=pa.Sigma31_dot, Sigma32_dot=pa.Sigma32_dot,
        rock_comp=pa.rock_comp, fluid_comp=pa.fluid_comp, fluid_density=pa.fluid_density,
        porosity=pa.porosity, dyn_viscosity=pa.dyn_viscosity, nb_source=len(pa.src_fault),
        src_fault=i(pa.src_fault), src_index=i(pa.src_index), src_Q=dd(pa.src_Q),
        src_t_beg=dd(pa.src_t_beg), src_t_end=dd(pa.src_t_end), tol_solver=pa.tol_solver,
        time0=pa.time0, max_it=pa.max_it, stride_time=pa.stride_time,
        freq_writing_file=pa.freq_writing_file, permeability_coupling=int(pa.permeability_coupling),
        kmin=d(pa.kmin if pa.kmin is not None else np.zeros(pa.N)),
        Snk=d(pa.Snk if pa.Snk is not None else np.ones(pa.N)))
    c._keep = keep
    return c
