"""Host-side driver over the C ABI, mirroring the reference's operator API.

``Simulation`` owns one device handle and exposes the reference's internal
operators with their names, argument meaning and error behaviour:

* ``kernel(slip)``             kernel_ptr (src/variables.f90:17-26)
* ``compute_P(dt)``            compute_P (src/fluid_diffusion.f90:24), returns ier
* ``friction_law(x, Y)``       fric_law_ptr (src/variables.f90:9-14)
* ``rkqs(...)``                rkqs (src/ode_solver/ode_bs.f90:125)
* ``solve(...)``               solve (src/solver.f90:42-206) with save_data /
                               write_data into ``output%07d`` files

All arithmetic runs in libdfn_b200 on the GPU; this module only moves
arrays across the ABI.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .layout import DfnOptions, DfnReport, ProblemArrays, build_arrays, ptr, to_c

STORAGE = {"fp64": 0, "fp32": 1, "bf16x2": 2, "bf16x2_tc": 3, "fp64_shared": 4}
PRESSURE = {"cg": 0, "tridiag": 1, "cg_exact": 2}
GEMV = {"tma": 0, "ldg": 1, "tc_persistent": 0, "tc_ring_deep": 1, "tc_ring_2stage": 2}


FORMULATION = {"v": 0, "newton": 1}
GUESS = {"analytic": 0, "mlp": 1, "warm": 2, "quasistatic": 3}


def make_options(lib, storage="fp64", pressure="cg", device=0, gemv="tma", max_attempts=64, hmat_leaf=0,
                 hmat_eta=0.0, hmat_eps=0.0, formulation="v", guess="analytic", newton_maxit=0, newton_tol=0.0,
                 max_step=0.0):
    """dfn_options; the H-matrix parameters default (0) to the reference's
    nleaf=100, eta=3, eps_ACA=1e-8 (src/variables.f90:122-124); max_step 0
    is the reference's one-day cap on the trial step."""
    opt = DfnOptions()
    lib.dfn_default_options(ctypes.byref(opt))
    opt.formulation = FORMULATION[formulation]
    opt.newton_guess = GUESS[guess]
    opt.newton_maxit = int(newton_maxit)
    opt.newton_tol = float(newton_tol)
    opt.kernel_storage = STORAGE[storage]
    opt.pressure_solver = PRESSURE[pressure]
    opt.device = int(device)
    opt.gemv_impl = GEMV[gemv]
    opt.max_attempts = int(max_attempts)
    opt.hmat_leaf = int(hmat_leaf)
    opt.hmat_eta = float(hmat_eta)
    opt.hmat_eps = float(hmat_eps)
    opt.max_step = float(max_step)
    return opt


class Simulation:
    def __init__(self, problem, storage="fp64", pressure="cg", device=0, gemv="tma", max_attempts=64,
                 hmat_leaf=0, hmat_eta=0.0, hmat_eps=0.0, formulation="v", guess="analytic", newton_maxit=0,
                 newton_tol=0.0, max_step=0.0):
        self.lib = _lib.load()
        self.arrays = problem if isinstance(problem, ProblemArrays) else build_arrays(problem)
        self.N = self.arrays.N
        opt = make_options(self.lib, storage, pressure, device, gemv, max_attempts, hmat_leaf, hmat_eta, hmat_eps,
                           formulation, guess, newton_maxit, newton_tol, max_step)
        self.formulation = formulation
        self._storage = storage
        self._pressure = pressure
        self.options = {"storage": storage, "pressure": pressure, "gemv": gemv}
        self._c = to_c(self.arrays)
        h = ctypes.c_void_p()
        _lib.check(self.lib.dfn_create(ctypes.byref(self._c), ctypes.byref(opt), ctypes.byref(h)), self.lib)
        self.h = h

    # -- lifecycle ---------------------------------------------------------
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
        return _lib.autotune(self.lib, self.h, self._storage, self._pressure, hmat=self.arrays.static_kernel == 1)

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

    def set_hmat_grids(self, dense_ctas=0, warp_ctas=0):
        """H-matrix handles: CTAs of the dense-row and small-leaf kernels
        (0: one per task; n: a persistent grid of n CTAs). Identical results."""
        _lib.check(self.lib.dfn_set_hmat_grids(self.h, int(dense_ctas), int(warp_ctas)), self.lib)

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

    def set_wait_limit(self, polls):
        """Polls of the bounded waits of the TMA K.V pipeline before a kernel
        gives up (None: the default); the next call then raises DfnError
        with status 10 (DFN_ERR_TIMEOUT)."""
        _lib.check(self.lib.dfn_set_wait_limit(self.h, -1 if polls is None else int(polls)), self.lib)

    @property
    def kernel_bytes(self):
        return int(self.lib.dfn_kernel_bytes(self.h))

    @property
    def launches(self):
        return int(self.lib.dfn_launch_count(self.h))

    # -- operators ---------------------------------------------------------
    def kernel(self, slip):
        slip = np.ascontiguousarray(slip, dtype=np.float64)
        if slip.shape != (self.N,):
            raise ValueError("slip must have nb_element entries")
        sT = np.empty(self.N)
        sN = np.empty(self.N)
        _lib.check(self.lib.dfn_kernel(self.h, ptr(slip), ptr(sT), ptr(sN)), self.lib)
        return sT, sN

    def compute_P(self, dt):
        Pt = np.zeros(self.N)
        Pd = np.zeros(self.N)
        ier = ctypes.c_int32(0)
        _lib.check(self.lib.dfn_compute_P(self.h, float(dt), ptr(Pt), ptr(Pd), ctypes.byref(ier)), self.lib)
        return Pt, Pd, int(ier.value)

    def friction_law(self, x, Y):
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        if Y.shape != (3 * self.N,):
            raise ValueError("Y must have 3*nb_element entries")
        Yd = np.empty_like(Y)
        _lib.check(self.lib.dfn_friction_law(self.h, float(x), Y.size, ptr(Y), ptr(Yd)), self.lib)
        return Yd

    def rkqs(self, y, dydx, x, htry, eps, yscal):
        y = np.array(y, dtype=np.float64, copy=True)
        dydx = np.ascontiguousarray(dydx, dtype=np.float64)
        yscal = np.ascontiguousarray(yscal, dtype=np.float64)
        xx = ctypes.c_double(x)
        hdid = ctypes.c_double(0)
        hnext = ctypes.c_double(0)
        _lib.check(self.lib.dfn_rkqs(self.h, ptr(y), ptr(dydx), y.size, ctypes.byref(xx), float(htry), float(eps),
                                     ptr(yscal), ctypes.byref(hdid), ctypes.byref(hnext)), self.lib)
        return y, xx.value, hdid.value, hnext.value

    # -- driver ------------------------------------------------------------
    def solve_steps(self, n):
        rep = DfnReport()
        st = self.lib.dfn_solve_steps(self.h, int(n), ctypes.byref(rep))
        _lib.check(st, self.lib)
        return rep.as_dict()

    def state(self):
        Y = np.empty(3 * self.N)
        P = np.empty(self.N)
        t = ctypes.c_double()
        tt = ctypes.c_double()
        it = ctypes.c_int64()
        _lib.check(self.lib.dfn_get_state(self.h, ptr(Y), ptr(P), ctypes.byref(t), ctypes.byref(tt),
                                          ctypes.byref(it)), self.lib)
        return {"Y": Y, "P": P, "time": t.value, "t_try": tt.value, "it_count": it.value}

    def set_state(self, Y, P, time, t_try, it_count=0):
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        _lib.check(self.lib.dfn_set_state(self.h, ptr(Y), ptr(P), float(time), float(t_try), int(it_count)),
                   self.lib)

    def snapshot(self):
        out = {k: np.empty(self.N) for k in ("V", "theta", "P", "tractionTel", "tractionNel", "permeability")}
        t = ctypes.c_double()
        _lib.check(self.lib.dfn_get_snapshot(self.h, ptr(out["V"]), ptr(out["theta"]), ptr(out["P"]),
                                             ptr(out["tractionTel"]), ptr(out["tractionNel"]),
                                             ptr(out["permeability"]), ctypes.byref(t)), self.lib)
        out["time"] = t.value
        return out

    def time_kernel(self, reps=20):
        ms = ctypes.c_double()
        _lib.check(self.lib.dfn_time_kernel(self.h, int(reps), ctypes.byref(ms)), self.lib)
        return ms.value

    # -- learned Newton guess ------------------------------------------------
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

    def report(self):
        rep = DfnReport()
        _lib.check(self.lib.dfn_get_report(self.h, 0, ctypes.byref(rep)), self.lib)
        return rep.as_dict()

    def slip(self):
        """Slip (m): the integral of V in the V formulation (a passive
        component of the RK stages), the state in the Newton formulation."""
        out = np.empty(self.N)
        _lib.check(self.lib.dfn_get_slip(self.h, 0, ptr(out)), self.lib)
        return out

    def set_slip(self, slip):
        slip = np.ascontiguousarray(slip, dtype=np.float64)
        _lib.check(self.lib.dfn_set_slip(self.h, 0, ptr(slip)), self.lib)

    def velocity(self):
        V = np.empty(self.N)
        _lib.check(self.lib.dfn_velocity(self.h, ptr(V)), self.lib)
        return V

    def solve_to(self, t_end):
        """Advance to simulated time t_end (the last step lands on it)."""
        reps = (DfnReport * 1)()
        _lib.check(self.lib.dfn_solve_batch(self.h, 0, float(t_end), reps), self.lib)
        return reps[0].as_dict()

    def hmat_stats(self):
        st = (ctypes.c_int64 * 8)()
        _lib.check(self.lib.dfn_hmat_stats(self.h, st), self.lib)
        keys = ["leaves", "dense_leaves", "lowrank_leaves", "max_rank", "mean_rank_x1000", "values",
                "dense_values", "lowrank_values"]
        return dict(zip(keys, list(st)))

    def hmat_perm(self):
        perm = np.empty(self.N, dtype=np.int32)
        _lib.check(self.lib.dfn_hmat_perm(self.h, perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))), self.lib)
        return perm

    def profile_kv(self, enable=True):
        _lib.check(self.lib.dfn_profile_kv(self.h, 1 if enable else 0), self.lib)

    def profile_kv_read(self):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _lib.check(self.lib.dfn_profile_kv_read(self.h, ctypes.byref(ms), ctypes.byref(n)), self.lib)
        return ms.value, n.value

    def step_host(self, Y, P, time, t_try, out):
        """One accepted step with host buffers on both sides (dfn_step_host)."""
        rep = DfnReport()
        st = self.lib.dfn_step_host(self.h, ptr(Y), ptr(P), float(time), float(t_try), ptr(out[0]), ptr(out[1]),
                                    ptr(out[2]), ptr(out[3]), ptr(out[4]), ctypes.byref(rep))
        _lib.check(st, self.lib)
        return rep

    def solve(self, max_it=None, output_dir=None, stride_time=None, freq_writing_file=None, callback=None):
        """The solve() loop (src/solver.f90:59-201) with its output schedule.

        A snapshot is saved when ``(it_count-1) % stride_time == 0``
        (save_data, :211-222); every ``freq_writing_file`` saved snapshots an
        ``output%07d`` file named after it_count is written (write_data,
        :190-193, :227-317), and a last file at the end (:201). Returns the list
        of saved snapshots when ``output_dir`` is None.
        """
        a = self.arrays
        max_it = a.max_it if max_it is None else int(max_it)
        stride = a.stride_time if stride_time is None else int(stride_time)
        freq = a.freq_writing_file if freq_writing_file is None else int(freq_writing_file)
        saved, buf = [], []
        it = self.state()["it_count"]
        while True:
            st = self.lib.dfn_solve_steps(self.h, 1, ctypes.byref(rep := DfnReport()))
            it = rep.it_count
            if st not in (0, 3):
                _lib.check(st, self.lib)
            if (it - 1) % stride == 0:
                snap = self.snapshot()
                buf.append(snap)
                if callback:
                    callback(it, snap)
            if st == 3:
                # sigmaN > 0: the reference prints and stops (src/solver.f90:412-418)
                # after the stop/write checks of this step
                self._flush(buf, it, freq, output_dir, saved, force=True)
                raise _lib.DfnError(3, f"it_count={it}")
            if it >= max_it:
                break
            if len(buf) == freq:
                self._flush(buf, it, freq, output_dir, saved)
        self._flush(buf, it, freq, output_dir, saved, force=True)
        return saved

    def _flush(self, buf, it, freq, output_dir, saved, force=False):
        if not buf:
            return
        if output_dir is None:
            saved.extend(buf)
        else:
            from .hdf5 import write_output

            os.makedirs(output_dir, exist_ok=True)
            # rows past the saved ones repeat the previous file's, as the
            # reference's persistent save arrays do
            self._ring = write_output(os.path.join(output_dir, "output%07d" % it), buf, freq, self.N,
                                      stale=getattr(self, "_ring", None))
        buf.clear()
