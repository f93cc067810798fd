"""ctypes wrapper of the CPU FP64 oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference
arm of ``bench.py`` use this module, as the checker. PARITY UNPINNED: the
reference cannot be compiled here and ships no golden outputs; the oracle is
pinned by known answers instead (see tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from demystification_dfn_b200.layout import DfnProblem, ProblemArrays, build_arrays, ptr, to_c  # noqa: E402

from build import LIB, build  # noqa: E402  (oracle/build.py, same folder)

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = ctypes.CDLL(LIB)
    V = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    i64, dbl, cint = ctypes.c_int64, ctypes.c_double, ctypes.c_int
    sig = {
        "orc_create": (V, [ctypes.POINTER(DfnProblem)]),
        "orc_destroy": (None, [V]),
        "orc_set_threads": (None, [V, cint]),
        "orc_set_kernel_impl": (None, [V, cint]),
        "orc_n": (i64, [V]),
        "orc_kernel_entry": (dbl, [V, i64, i64, cint]),
        "orc_assemble_dense": (cint, [V]),
        "orc_copy_dense": (None, [V, dp, dp]),
        "orc_kernel": (None, [V, dp, dp, dp]),
        "orc_compute_P": (cint, [V, dbl, dp, dp]),
        "orc_pressure_exact": (None, [V, dbl, dp]),
        "orc_crossings": (i64, [V]),
        "orc_rhs": (cint, [V, dbl, dp, dp]),
        "orc_rkqs": (cint, [V, dp, dp, i64, dp, dbl, dbl, dp, dp, dp]),
        "orc_solve_step": (cint, [V]),
        "orc_solve_steps": (cint, [V, i64, dp]),
        "orc_get_state": (None, [V, dp, dp, dp]),
        "orc_set_state": (None, [V, dp, dp, dbl, dbl, i64]),
        "orc_get_geometry": (None, [V, dp, dp, dp, dp, dp]),
        "orc_get_loads": (None, [V, dp, dp, ctypes.POINTER(ctypes.c_ubyte)]),
        "orc_get_last_stress": (None, [V, dp, dp, dp]),
        "orc_counters": (None, [V, ctypes.POINTER(i64)]),
        "orc_hmat_build": (cint, [V, cint, dbl, dbl]),
        "orc_hmat_perm": (None, [V, ctypes.POINTER(ctypes.c_int)]),
        "orc_hmat_stats": (None, [V, ctypes.POINTER(i64)]),
        "orc_set_formulation": (cint, [V, cint, cint, cint, dbl]),
        "orc_set_max_step": (None, [V, dbl]),
        "orc_get_permeability": (None, [V, dp]),
        "orc_velocity": (None, [V, dp]),
        "orc_get_slip": (None, [V, dp]),
        "orc_set_slip": (None, [V, dp]),
        "orc_newton_counters": (None, [V, ctypes.POINTER(i64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class Oracle:
    """CPU FP64 restatement of the reference path for one problem."""

    def __init__(self, problem, threads=1, dense=False):
        self.lib = load()
        self.arrays = problem if isinstance(problem, ProblemArrays) else build_arrays(problem)
        self.N = self.arrays.N
        self._c = to_c(self.arrays)
        self.o = self.lib.orc_create(ctypes.byref(self._c))
        if not self.o:
            raise ValueError("oracle rejected the problem")
        self.lib.orc_set_threads(self.o, int(threads))
        if dense:
            self.use_dense()

    def close(self):
        if getattr(self, "o", None):
            self.lib.orc_destroy(self.o)
            self.o = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_formulation(self, form, guess="analytic", maxit=0, tol=0.0):
        """"v" (the reference's ODE) or "newton" (the library's Newton slip
        formulation restated: state [slip, psi, sigmaN0], V from the friction
        law); guess "analytic" (bounded start) or "quasistatic"."""
        st = self.lib.orc_set_formulation(self.o, {"v": 0, "newton": 1}[form],
                                          {"analytic": 0, "quasistatic": 3}[guess], int(maxit), float(tol))
        if st:
            raise ValueError(f"oracle formulation status {st}")

    def set_max_step(self, seconds):
        """Cap on the trial step after each step (0: the reference's one day)."""
        self.lib.orc_set_max_step(self.o, float(seconds))

    def permeability(self):
        """Permeability of the last pressure solve (evolving with the coupling)."""
        k = np.empty(self.N)
        self.lib.orc_get_permeability(self.o, ptr(k))
        return k

    def velocity(self):
        V = np.empty(self.N)
        self.lib.orc_velocity(self.o, ptr(V))
        return V

    def slip(self):
        """Slip: the passive integral of V (V formulation) or the state (Newton)."""
        s = np.empty(self.N)
        self.lib.orc_get_slip(self.o, ptr(s))
        return s

    def set_slip(self, slip):
        slip = np.ascontiguousarray(slip, dtype=np.float64)
        self.lib.orc_set_slip(self.o, ptr(slip))

    def newton_counters(self):
        c = (ctypes.c_int64 * 3)()
        self.lib.orc_newton_counters(self.o, c)
        return dict(zip(["solves", "iters", "fail"], list(c)))

    def set_threads(self, n):
        self.lib.orc_set_threads(self.o, int(n))

    def use_dense(self):
        if self.lib.orc_assemble_dense(self.o) != 0:
            raise MemoryError("dense kernel does not fit in host memory")
        self.lib.orc_set_kernel_impl(self.o, 1)

    def use_direct(self):
        self.lib.orc_set_kernel_impl(self.o, 0)

    def use_hmatrix(self, leaf=100, eta=3.0, eps=1e-8):
        """The reference's H-matrix (full-pivot ACA on evaluated blocks);
        returns False when an ACA needed more than 20 terms (the reference stops)."""
        return self.lib.orc_hmat_build(self.o, int(leaf), float(eta), float(eps)) == 0

    def hmat_perm(self):
        perm = np.empty(self.N, dtype=np.int32)
        self.lib.orc_hmat_perm(self.o, perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return perm

    def hmat_stats(self):
        st = (ctypes.c_int64 * 4)()
        self.lib.orc_hmat_stats(self.o, st)
        return dict(zip(["leaves", "dense_leaves", "max_rank", "clusters"], list(st)))

    def entry(self, k, l, which):
        return self.lib.orc_kernel_entry(self.o, int(k), int(l), int(which))

    def dense(self):
        N = self.N
        KT = np.empty((N, N))
        KN = np.empty((N, N)) if self.arrays.fracture_mode == 2 else None
        if self.lib.orc_assemble_dense(self.o) != 0:
            raise MemoryError
        self.lib.orc_copy_dense(self.o, ptr(KT), ptr(KN) if KN is not None else None)
        return KT, KN

    def kernel(self, slip):
        slip = np.ascontiguousarray(slip, dtype=np.float64)
        sT, sN = np.empty(self.N), np.empty(self.N)
        self.lib.orc_kernel(self.o, ptr(slip), ptr(sT), ptr(sN))
        return sT, sN

    def compute_P(self, dt):
        Pt, Pd = np.zeros(self.N), np.zeros(self.N)
        ier = self.lib.orc_compute_P(self.o, float(dt), ptr(Pt), ptr(Pd))
        return Pt, Pd, ier

    def crossings(self):
        """Fault crossings found as find_fault_crossing does."""
        return int(self.lib.orc_crossings(self.o))

    def pressure_exact(self, dt):
        Pt = np.zeros(self.N)
        self.lib.orc_pressure_exact(self.o, float(dt), ptr(Pt))
        return Pt

    def friction_law(self, x, Y):
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        Yd = np.empty_like(Y)
        self.lib.orc_rhs(self.o, float(x), ptr(Y), ptr(Yd))
        return Yd

    def rkqs(self, y, dydx, x, htry, eps, yscal):
        y = np.array(y, dtype=np.float64, copy=True)
        dydx = np.ascontiguousarray(dydx, dtype=np.float64)
        yscal = np.ascontiguousarray(yscal, dtype=np.float64)
        xx, hd, hn = ctypes.c_double(x), ctypes.c_double(), ctypes.c_double()
        st = self.lib.orc_rkqs(self.o, ptr(y), ptr(dydx), y.size, ctypes.byref(xx), float(htry), float(eps),
                               ptr(yscal), ctypes.byref(hd), ctypes.byref(hn))
        if st:
            raise RuntimeError(f"oracle rkqs status {st}")
        return y, xx.value, hd.value, hn.value

    def solve_steps(self, n):
        log = np.zeros(max(int(n), 1))
        st = self.lib.orc_solve_steps(self.o, int(n), ptr(log))
        return st, log[: int(n)]

    def state(self):
        Y, P, s = np.empty(3 * self.N), np.empty(self.N), np.empty(3)
        self.lib.orc_get_state(self.o, ptr(Y), ptr(P), ptr(s))
        return {"Y": Y, "P": P, "time": s[0], "t_try": s[1], "it_count": int(s[2])}

    def set_state(self, Y, P, time, t_try, it_count=0):
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        self.lib.orc_set_state(self.o, ptr(Y), ptr(P), float(time), float(t_try), int(it_count))

    def geometry(self):
        N = self.N
        el, ds, tn, nr, px = np.empty(2 * N), np.empty(N), np.empty(2 * N), np.empty(2 * N), np.empty(N + 1)
        self.lib.orc_get_geometry(self.o, ptr(el), ptr(ds), ptr(tn), ptr(nr), ptr(px))
        return {"element": el.reshape(N, 2), "ds": ds, "tangent": tn.reshape(N, 2), "normal": nr.reshape(N, 2),
                "permeability_x": px}

    def loads(self):
        nl, sl = np.empty(self.N), np.empty(self.N)
        fk = np.zeros(self.N, dtype=np.uint8)
        self.lib.orc_get_loads(self.o, ptr(nl), ptr(sl), fk.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
        return nl, sl, fk.astype(bool)

    def last_stress(self):
        sT, sN, Pd = np.empty(self.N), np.empty(self.N), np.empty(self.N)
        self.lib.orc_get_last_stress(self.o, ptr(sT), ptr(sN), ptr(Pd))
        return sT, sN, Pd

    def counters(self):
        c = (ctypes.c_int64 * 7)()
        self.lib.orc_counters(self.o, c)
        return dict(zip(["cg_iters", "rhs_evals", "attempts", "rejected", "halvings", "it_count", "stage_noconv"],
                        list(c)))
