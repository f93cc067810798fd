"""Many independent fault networks advanced together on one GPU.

``Ensemble`` wraps ``dfn_create_batch``: every network keeps its own state,
adaptive step size, controller and done flag (the reference's solve() loop
per network), while each kernel launch covers the whole batch, so networks
of uneven size share the GPU without per-network launches.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .layout import DfnProblem, DfnReport, ProblemArrays, build_arrays, ptr, to_c
from .simulation import make_options


class Ensemble:
    def __init__(self, problems, storage="fp64", pressure="cg", device=0, gemv="tma", max_attempts=64,
                 hmat_leaf=0, hmat_eta=0.0, hmat_eps=0.0, formulation="v", guess="analytic", newton_maxit=0,
                 newton_tol=0.0, max_step=0.0):
        self.lib = _lib.load()
        self.arrays = [p if isinstance(p, ProblemArrays) else build_arrays(p) for p in problems]
        if not self.arrays:
            raise ValueError("an ensemble needs at least one problem")
        self.B = len(self.arrays)
        self._storage = storage
        self._pressure = pressure
        opt = make_options(self.lib, storage, pressure, device, gemv, max_attempts, hmat_leaf, hmat_eta, hmat_eps,
                           formulation, guess, newton_maxit, newton_tol, max_step)
        self._cs = [to_c(a) for a in self.arrays]
        arr = (DfnProblem * self.B)(*self._cs)
        self._arr = arr
        h = ctypes.c_void_p()
        _lib.check(self.lib.dfn_create_batch(arr, self.B, ctypes.byref(opt), ctypes.byref(h)), self.lib)
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.dfn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle: int):
        _lib.check(self.lib.dfn_set_stream(self.h, ctypes.c_void_p(stream_handle)), self.lib)

    def autotune(self):
        """Time the interchangeable launch shapes (K.V copy path, short-segment
        pressure solve) on this handle's data and keep the fastest."""
        return _lib.autotune(self.lib, self.h, self._storage, self._pressure, hmat=self.arrays[0].static_kernel == 1)

    @property
    def crossing_count(self):
        """Fault crossings that couple the pressure of the networks."""
        return int(self.lib.dfn_crossing_count(self.h))

    def set_tri_shape(self, shape):
        """Short tridiagonal segments by "warp", "thread" or "tile"."""
        _lib.check(self.lib.dfn_set_tri_shape(self.h, {"warp": 0, "thread": 1, "tile": 2}[shape]), self.lib)

    def set_hmat_small_leaves(self, form):
        """H-matrix handles: whole low-rank leaves of at most 32 KiB by one
        "warp" each (the default) or one "cta" each."""
        _lib.check(self.lib.dfn_set_hmat_small_leaves(self.h, {"warp": 0, "cta": 1}[form]), self.lib)

    def set_cg_form(self, form):
        """CG pressure solves by "cta" (one CTA per system, global memory),
        "cluster" (a thread-block cluster per system, shared memory),
        "cta_smem" (one CTA per system, shared memory) or "default"."""
        code = {"default": -1, "cta": 0, "cluster": 1, "cta_smem": 2}[form]
        _lib.check(self.lib.dfn_set_cg_form(self.h, code), self.lib)

    def set_graphs(self, enable: bool):
        """Replay the solve loop's rounds as a CUDA graph (default) or launch
        every kernel on its own; results are identical."""
        _lib.check(self.lib.dfn_set_graphs(self.h, 1 if enable else 0), self.lib)

    @property
    def kernel_bytes(self):
        return int(self.lib.dfn_kernel_bytes(self.h))

    @property
    def launches(self):
        return int(self.lib.dfn_launch_count(self.h))

    @property
    def n_elements(self):
        return [a.N for a in self.arrays]

    def kernel(self, slips):
        """K.V of every network: list of slip vectors in, lists of shear and
        normal stress rates out (dfn_kernel_batch)."""
        v = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64) for s in slips]))
        if len(v) != sum(self.n_elements):
            raise ValueError("one slip vector per network, of its nb_element")
        sT, sN = np.empty_like(v), np.empty_like(v)
        _lib.check(self.lib.dfn_kernel_batch(self.h, ptr(v), ptr(sT), ptr(sN)), self.lib)
        cut = np.cumsum(self.n_elements)[:-1]
        return np.split(sT, cut), np.split(sN, cut)

    def solve(self, n_steps=0, t_end=0.0, check=True):
        """Advance every network by n_steps accepted steps, or to time t_end."""
        reps = (DfnReport * self.B)()
        st = self.lib.dfn_solve_batch(self.h, int(n_steps), float(t_end), reps)
        if check:
            _lib.check(st, self.lib)
        return [r.as_dict() for r in reps]

    def state(self, i):
        N = self.arrays[i].N
        Y, P = np.empty(3 * N), np.empty(N)
        t, tt, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _lib.check(self.lib.dfn_get_state_instance(self.h, int(i), ptr(Y), ptr(P), ctypes.byref(t),
                                                   ctypes.byref(tt), ctypes.byref(it)), self.lib)
        return {"Y": Y, "P": P, "time": t.value, "t_try": tt.value, "it_count": it.value}

    def slip(self, i):
        """Slip (m) of network i (see Simulation.slip)."""
        out = np.empty(self.arrays[i].N)
        _lib.check(self.lib.dfn_get_slip(self.h, int(i), ptr(out)), self.lib)
        return out

    def report(self, i):
        rep = DfnReport()
        _lib.check(self.lib.dfn_get_report(self.h, int(i), ctypes.byref(rep)), self.lib)
        return rep.as_dict()

    def set_mlp(self, weights):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        _lib.check(self.lib.dfn_set_mlp(self.h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self.lib)

    def set_mlp_gate(self, rel):
        """Evaluate the learned guess only where the analytic start's
        relative residual exceeds rel (dfn_set_mlp_gate)."""
        _lib.check(self.lib.dfn_set_mlp_gate(self.h, float(rel)), self.lib)

    def record(self, capacity):
        _lib.check(self.lib.dfn_record(self.h, int(capacity)), self.lib)

    def record_read(self, max_samples):
        x = np.empty((int(max_samples), 7), dtype=np.float32)
        t = np.empty(int(max_samples), dtype=np.float32)
        n = ctypes.c_int64()
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check(self.lib.dfn_record_read(self.h, x.ctypes.data_as(fp), t.ctypes.data_as(fp), int(max_samples),
                                            ctypes.byref(n)), self.lib)
        return x[:n.value], t[:n.value]

    def time_kernel(self, reps=10):
        ms = ctypes.c_double()
        _lib.check(self.lib.dfn_time_kernel(self.h, int(reps), ctypes.byref(ms)), self.lib)
        return ms.value

    def profile_kv(self, enable=True):
        _lib.check(self.lib.dfn_profile_kv(self.h, 1 if enable else 0), self.lib)

    def profile_kv_read(self):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _lib.check(self.lib.dfn_profile_kv_read(self.h, ctypes.byref(ms), ctypes.byref(n)), self.lib)
        return ms.value, n.value
