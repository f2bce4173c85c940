"""ctypes binding of libgapk.so (include/gapk.h).

The library is loaded from gap_b200/lib/ (built in-tree by gap_b200.csrc.build).  Loading
never falls back to anything: a missing library raises.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libgapk.so")

GAPK_OK = 0
PREC_FP64, PREC_FP32 = 0, 1
POLICY_REFERENCE, POLICY_NEWTON, POLICY_CLAMPED = 0, 1, 2
JAC_REFERENCE, JAC_EXACT = 0, 1
ORDER_MINDEG, ORDER_NATURAL = 0, 1
YBUS_REFERENCE, YBUS_TAPS = 0, 1
DELTA_REFERENCE, DELTA_FIXED, DELTA_FIXED_TAPS = 0, 1, 2
SCEN_CONVERGED, SCEN_MAXITER, SCEN_SINGULAR, SCEN_NONFINITE = 0, 1, 2, 3

EXPORTS = [
    "gapk_last_error", "gapk_version", "gapk_device_count",
    "gapk_ybus_create", "gapk_ybus_destroy", "gapk_ybus_nnz", "gapk_ybus_pattern",
    "gapk_ybus_assemble", "gapk_ybus_apply_changes", "gapk_ybus_delta_create",
    "gapk_ybus_delta_destroy", "gapk_ybus_delta_apply",
    "gapk_nr_plan_create", "gapk_nr_plan_destroy", "gapk_nr_plan_get_info",
    "gapk_nr_plan_export",
    "gapk_nr_batch_create", "gapk_nr_batch_destroy", "gapk_nr_batch_device_bytes",
    "gapk_nr_solve", "gapk_nr_last_loop_count", "gapk_nr_mix_create", "gapk_nr_mix_destroy",
    "gapk_nr_mix_solve",
    "gapk_nr_stage_load", "gapk_nr_stage_mismatch", "gapk_nr_stage_jacobian",
    "gapk_nr_stage_factor", "gapk_nr_stage_solve", "gapk_nr_stage_get_correction",
    "gapk_nr_stage_get_mismatch", "gapk_nr_stage_kernel", "gapk_nr_solve_noalloc",
    "gapk_nr_step", "gapk_nr_get_state", "gapk_nr_get_outputs", "gapk_nr_level_trace_size",
    "gapk_nr_set_level_trace", "gapk_nr_dense_trace_panels", "gapk_nr_batch_lanes",
    "gapk_nr_batch_device_error", "gapk_nr_batch_set_wait_test",
    "gapk_splu_create", "gapk_splu_destroy", "gapk_splu_size", "gapk_splu_factorize",
    "gapk_splu_solve", "gapk_nr_adjoint", "gapk_nr_adjoint_branch", "gapk_branch_flows",
]


class PlanOptions(C.Structure):
    _fields_ = [("jacobian_mode", C.c_int), ("ordering", C.c_int), ("dense_min", C.c_int)]


class PlanInfo(C.Structure):
    _fields_ = [("n_bus", C.c_int), ("n_block", C.c_int), ("n_pq", C.c_int),
                ("n_pv", C.c_int), ("n_slack", C.c_int), ("n_vars", C.c_int),
                ("nnz_y", C.c_int), ("nnz_l_blocks", C.c_int), ("n_slots", C.c_int),
                ("n_a_blocks", C.c_int), ("n_levels", C.c_int), ("n_pairs", C.c_int64),
                ("n_rows_pairs", C.c_int64), ("max_level_width", C.c_int),
                ("n_tail", C.c_int), ("n_schur_pairs", C.c_int64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BatchOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("y_shared", C.c_int), ("lanes", C.c_int),
                ("threads", C.c_int), ("use_graph", C.c_int), ("dense_fused", C.c_int),
                ("dense_fma", C.c_int)]


class Inputs(C.Structure):
    _fields_ = [("d_y", C.c_void_p), ("d_s_spec", C.c_void_p), ("d_v_init", C.c_void_p),
                ("d_u_pu", C.c_void_p), ("tolerance", C.c_double),
                ("max_iterations", C.c_int), ("policy", C.c_int), ("refine", C.c_int),
                ("refine_below", C.c_double), ("reuse_below", C.c_double),
                ("v_init_shared", C.c_int)]


class Outputs(C.Structure):
    _fields_ = [("d_v", C.c_void_p), ("d_iterations", C.c_void_p), ("d_status", C.c_void_p),
                ("d_final_mismatch", C.c_void_p)]


_lib = None


class GapkError(RuntimeError):
    pass


def lib():
    """The loaded libgapk.so.  Raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GapkError(f"{LIB_PATH} missing: build it with python -m gap_b200.csrc.build")
        L = C.CDLL(LIB_PATH)
        L.gapk_last_error.restype = C.c_char_p
        L.gapk_nr_plan_export.restype = C.c_int64
        L.gapk_nr_batch_device_bytes.restype = C.c_int64
        L.gapk_nr_level_trace_size.restype = C.c_int64
        L.gapk_nr_set_level_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        for name in ("gapk_ybus_create", "gapk_nr_plan_create", "gapk_nr_batch_create"):
            getattr(L, name).restype = C.c_int
        L.gapk_ybus_assemble.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64,
                                         C.c_void_p, C.c_int64, C.c_int, C.c_double,
                                         C.c_void_p, C.c_int64, C.c_void_p]
        L.gapk_ybus_delta_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                            C.c_void_p, C.c_int64, C.c_void_p]
        L.gapk_ybus_apply_changes.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                              C.c_void_p, C.c_void_p]
        L.gapk_nr_mix_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.gapk_branch_flows.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int64, C.c_void_p, C.c_double,
                                         C.c_double, C.c_void_p, C.c_void_p, C.c_int,
                                         C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def check(rc):
    if rc != GAPK_OK:
        raise GapkError(f"gapk error {rc}: {lib().gapk_last_error().decode()}")
    return rc


def iptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)
