"""ctypes binding of ``libdfn_b200.so`` (the C ABI of include/dfn_b200.h).

The library is loaded from the package's ``_build`` folder. There is no
fallback: if the library is missing or cannot be loaded this module raises.
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB
from .layout import DfnOptions, DfnProblem, DfnReport

_lib = None

STATUS = {
    0: "ok", 1: "pressure CG did not converge", 2: "stepsize underflow in rkqs",
    3: "normal traction became extensional", 4: "non-finite value", 5: "invalid argument",
    6: "CUDA error", 7: "unsupported", 8: "too many rejected attempts", 9: "device allocation failed",
    10: "a bounded device wait expired",
}

EXPORTS = [
    "dfn_abi_version", "dfn_problem_struct_size", "dfn_options_struct_size", "dfn_report_struct_size",
    "dfn_status_string", "dfn_last_error", "dfn_default_options", "dfn_create", "dfn_destroy",
    "dfn_set_stream", "dfn_nb_element", "dfn_kernel_bytes", "dfn_kernel", "dfn_compute_P",
    "dfn_friction_law", "dfn_rkqs", "dfn_solve_steps", "dfn_step_host", "dfn_get_state", "dfn_set_state",
    "dfn_get_snapshot", "dfn_kernel_device", "dfn_time_kernel", "dfn_launch_count", "dfn_profile_kv",
    "dfn_profile_kv_read",
]


class DfnError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, 'status ' + str(status))}" + (f": {msg}" if msg else ""))


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise ImportError(f"{LIB} is missing; build it with `python -m demystification_dfn_b200.build`")
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    sig = {
        "dfn_abi_version": (i32, []),
        "dfn_problem_struct_size": (i64, []),
        "dfn_options_struct_size": (i64, []),
        "dfn_report_struct_size": (i64, []),
        "dfn_status_string": (ctypes.c_char_p, [i32]),
        "dfn_last_error": (ctypes.c_char_p, []),
        "dfn_default_options": (None, [ctypes.POINTER(DfnOptions)]),
        "dfn_create": (i32, [ctypes.POINTER(DfnProblem), ctypes.POINTER(DfnOptions), ctypes.POINTER(P)]),
        "dfn_destroy": (i32, [P]),
        "dfn_set_stream": (i32, [P, P]),
        "dfn_nb_element": (i64, [P]),
        "dfn_kernel_bytes": (i64, [P]),
        "dfn_kernel": (i32, [P, dp, dp, dp]),
        "dfn_compute_P": (i32, [P, dbl, dp, dp, ctypes.POINTER(i32)]),
        "dfn_friction_law": (i32, [P, dbl, i64, dp, dp]),
        "dfn_rkqs": (i32, [P, dp, dp, i64, dp, dbl, dbl, dp, dp, dp]),
        "dfn_solve_steps": (i32, [P, i64, ctypes.POINTER(DfnReport)]),
        "dfn_step_host": (i32, [P, dp, dp, dbl, dbl, dp, dp, dp, dp, dp, ctypes.POINTER(DfnReport)]),
        "dfn_get_state": (i32, [P, dp, dp, dp, dp, ctypes.POINTER(i64)]),
        "dfn_set_state": (i32, [P, dp, dp, dbl, dbl, i64]),
        "dfn_get_snapshot": (i32, [P, dp, dp, dp, dp, dp, dp, dp]),
        "dfn_kernel_device": (i32, [P, P, P, P]),
        "dfn_time_kernel": (i32, [P, i32, dp]),
        "dfn_launch_count": (i64, [P]),
        "dfn_profile_kv": (i32, [P, i32]),
        "dfn_profile_kv_read": (i32, [P, dp, ctypes.POINTER(i64)]),
        "dfn_get_report": (i32, [P, i32, ctypes.POINTER(DfnReport)]),
        "dfn_set_mlp": (i32, [P, ctypes.POINTER(ctypes.c_float)]),
        "dfn_set_mlp_gate": (i32, [P, dbl]),
        "dfn_record": (i32, [P, i64]),
        "dfn_record_read": (i32, [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), i64,
                                  ctypes.POINTER(i64)]),
        "dfn_mlp_train": (i32, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), i64,
                                ctypes.POINTER(ctypes.c_float), i32, i32, ctypes.c_float, ctypes.c_uint64,
                                ctypes.POINTER(ctypes.c_float)]),
        "dfn_mlp_loss_grad": (i32, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), i64,
                                    ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_float)]),
        "dfn_mlp_infer": (i32, [ctypes.POINTER(ctypes.c_float), i64, ctypes.POINTER(ctypes.c_float),
                                ctypes.POINTER(ctypes.c_float)]),
        "dfn_set_graphs": (i32, [P, i32]),
        "dfn_set_wait_limit": (i32, [P, i32]),
        "dfn_get_slip": (i32, [P, i32, dp]),
        "dfn_set_slip": (i32, [P, i32, dp]),
        "dfn_set_cg_form": (i32, [P, i32]),
        "dfn_set_hmat_small_leaves": (i32, [P, i32]),
        "dfn_crossing_count": (i64, [P]),
        "dfn_set_tri_shape": (i32, [P, i32]),
        "dfn_set_hmat_grids": (i32, [P, i64, i64]),
        "dfn_autotune": (i32, [P, ctypes.c_void_p]),
        "dfn_kernel_batch": (i32, [P, dp, dp, dp]),
        "dfn_velocity": (i32, [P, dp]),
        "dfn_hmat_stats": (i32, [P, ctypes.POINTER(i64)]),
        "dfn_hmat_perm": (i32, [P, ctypes.POINTER(i32)]),
        "dfn_create_batch":(i32, [ctypes.POINTER(DfnProblem), i32, ctypes.POINTER(DfnOptions), ctypes.POINTER(P)]),
        "dfn_batch_size": (i32, [P]),
        "dfn_solve_batch": (i32, [P, i64, dbl, ctypes.POINTER(DfnReport)]),
        "dfn_get_state_instance": (i32, [P, i32, dp, dp, dp, dp, ctypes.POINTER(i64)]),
        "dfn_compute_P_noalloc":(i32, [i64, dbl, dbl, P, P, P, dbl, dbl, dbl, dbl, dbl, i64, P, P, P, P, P, P,
                                        P, ctypes.POINTER(i32), P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.dfn_problem_struct_size() != ctypes.sizeof(DfnProblem):
        raise ImportError("dfn_problem layout mismatch between the library and layout.py")
    if lib.dfn_options_struct_size() != ctypes.sizeof(DfnOptions):
        raise ImportError("dfn_options layout mismatch between the library and layout.py")
    if lib.dfn_report_struct_size() != ctypes.sizeof(DfnReport):
        raise ImportError("dfn_report layout mismatch between the library and layout.py")
    _lib = lib
    return lib


def check(status, lib=None):
    if status != 0:
        lib = lib or load()
        raise DfnError(status, (lib.dfn_last_error() or b"").decode())
    return status


class DfnTuning(ctypes.Structure):
    _fields_ = [("gemv_impl", ctypes.c_int32), ("tri_thread", ctypes.c_int32), ("ms", ctypes.c_double * 6),
                ("cg_cluster", ctypes.c_int32), ("cg_cluster_ctas", ctypes.c_int32),
                ("hm_dense_grid", ctypes.c_int64), ("hm_warp_grid", ctypes.c_int64)]


def autotune(lib, h, storage, pressure, hmat=False):
    """dfn_autotune on handle h; names the K.V shapes of the handle's storage
    and the pressure shapes of its solver."""
    t = DfnTuning()
    check(lib.dfn_autotune(h, ctypes.byref(t)), lib)
    extra = {}
    if storage == "bf16x2_tc":
        names = ("tc_persistent", "tc_ring_deep", "tc_ring_2stage")
        ms = {"kv_tc_persistent": t.ms[0], "kv_tc_ring_deep": t.ms[1], "kv_tc_ring_2stage": t.ms[4]}
    elif hmat:
        names = ("tma", "ldg")
        ms = {"kv_hmat_best": t.ms[0], "kv_hmat_one_cta_per_task": t.ms[1]}
        extra = {"hm_dense_grid": int(t.hm_dense_grid), "hm_warp_grid": int(t.hm_warp_grid)}
    else:
        names = ("tma", "ldg")
        ms = {"kv_tma": t.ms[0], "kv_ldg": t.ms[1]}
    if pressure == "cg":
        ms["pressure_cg_cta"] = t.ms[2]
        ms["pressure_cg_cluster"] = t.ms[3]
        ms["pressure_cg_cta_smem"] = t.ms[5]
    else:
        ms["pressure_warp"] = t.ms[2]
        ms["pressure_thread"] = t.ms[3]
        ms["pressure_tile"] = t.ms[5]
    return {"gemv_impl": names[t.gemv_impl], "short_segments": ("warp", "thread", "tile")[t.tri_thread],
            "cg_form": ("cta", "cluster", "cta_smem")[t.cg_cluster], "cg_cluster_ctas": int(t.cg_cluster_ctas),
            "ms": ms, **extra}
