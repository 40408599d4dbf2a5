"""ctypes binding of ``libglu_b200.so`` (the C ABI in ``include/glu_b200.h``).

The library is built in-tree (``python -m glu_public_b200.build``).  There is no fallback: if the
library is missing or a call fails, an exception says so.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libglu_b200.so")

GLU_OK = 0
INST_ZERO_PIVOT, INST_NAN_PIVOT, INST_PERTURBED, INST_TIMEOUT = 1, 2, 4, 8

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
vp = C.c_void_p


class GluError(RuntimeError):
    def __init__(self, status: int, what: str):
        lib = _lib
        msg = lib.glu_status_string(status).decode() if lib else str(status)
        detail = lib.glu_last_error().decode() if lib else ""
        super().__init__(f"{what}: {msg} ({status}): {detail}")
        self.status = status


class Options(C.Structure):
    _fields_ = [("dense_threshold", C.c_double), ("dense_min", C.c_int32), ("panel", C.c_int32),
                ("sparse_warps_per_col", C.c_int32), ("sparse_cols_per_warp", C.c_int32),
                ("gemm_variant", C.c_int32), ("deterministic", C.c_int32), ("device", C.c_int32),
                ("hub_min_frac", C.c_double), ("hub_max", C.c_int32),
                ("front_min_w", C.c_int32), ("front_min_flops", C.c_double),
                ("update_depth", C.c_int32), ("sparse_persistent", C.c_int32),
                ("level_wait_ms", C.c_double), ("wide_level_cols", C.c_int32),
                ("narrow_col_work", C.c_int32), ("sparse_block", C.c_int32),
                ("front_batch", C.c_int32),
                ("sparse_col_lanes", C.c_int32), ("level_warps_per_sm", C.c_int32)]


_lib = None

# exported symbols of the C ABI, in declaration order of include/glu_b200.h
EXPORTS = [
    "glu_options_default", "glu_status_string", "glu_last_error",
    "glu_symbolic_create", "glu_symbolic_sizes", "glu_symbolic_order", "glu_symbolic_get",
    "glu_symbolic_positions",
    "glu_symbolic_destroy", "glu_symbolic_save", "glu_symbolic_load", "glu_plan_create",
    "glu_plan_set_ingest",
    "glu_plan_ingest_from_nicslu", "glu_plan_set_solve_maps", "glu_plan_stat",
    "glu_plan_destroy", "glu_batch_create", "glu_batch_slots_per_instance",
    "glu_batch_create_external", "glu_batch_destroy", "glu_load_values", "glu_load_lu_values",
    "glu_refactor", "glu_refactor_timed", "glu_autotune", "glu_batch_status", "glu_solve",
    "glu_plan_set_original_pattern", "glu_residual", "glu_residual_noalloc", "glu_refine",
    "glu_grad_a",
    "glu_get_lu", "glu_graph_capture", "glu_graph_launch", "glu_group_capture",
    "glu_group_launch", "glu_group_launch_count", "glu_group_destroy",
    "glu_debug_refactor_unreachable_barrier", "glu_batch_launch_count", "glu_debug_gemm_sub",
]


def lib():
    """Loads the library once; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m glu_public_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.glu_options_default.argtypes = [C.POINTER(Options)]
    L.glu_options_default.restype = None
    L.glu_status_string.argtypes = [C.c_int]
    L.glu_status_string.restype = C.c_char_p
    L.glu_last_error.argtypes = []
    L.glu_last_error.restype = C.c_char_p
    L.glu_symbolic_create.argtypes = [C.c_uint32, u32p, u32p, C.POINTER(vp)]
    L.glu_symbolic_sizes.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]
    L.glu_symbolic_order.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.glu_symbolic_get.argtypes = [vp, u32p, u32p, u32p, u32p, u32p, u32p, i32p, i32p]
    L.glu_symbolic_positions.argtypes = [vp, u32p, u32p, i64p]
    L.glu_symbolic_destroy.argtypes = [vp]
    L.glu_symbolic_destroy.restype = None
    L.glu_symbolic_save.argtypes = [vp, C.c_char_p]
    L.glu_symbolic_load.argtypes = [C.c_char_p, C.c_uint32, vp, vp, C.POINTER(vp)]
    L.glu_plan_create.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, u32p, u32p, u32p, u32p,
                                  C.c_int32, i32p, i32p, C.POINTER(Options), C.POINTER(vp)]
    L.glu_plan_set_ingest.argtypes = [vp, C.c_uint64, i64p, vp]
    L.glu_plan_ingest_from_nicslu.argtypes = [vp, C.c_uint32, u32p, u32p, u32p, u32p, vp, vp]
    L.glu_plan_set_solve_maps.argtypes = [vp, u32p, u32p, vp, vp]
    L.glu_plan_stat.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
    L.glu_plan_destroy.argtypes = [vp]
    L.glu_batch_create.argtypes = [vp, C.c_int32, C.POINTER(vp)]
    L.glu_batch_slots_per_instance.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.glu_batch_create_external.argtypes = [vp, C.c_int32, vp, C.POINTER(vp)]
    L.glu_batch_destroy.argtypes = [vp]
    L.glu_load_values.argtypes = [vp, C.c_int32, C.c_int32, vp, vp]
    L.glu_load_lu_values.argtypes = [vp, C.c_int32, C.c_int32, vp, vp]
    L.glu_refactor.argtypes = [vp, C.c_double, vp]
    L.glu_batch_status.argtypes = [vp, i32p, vp]
    L.glu_refactor_timed.argtypes = [vp, C.c_double, vp, f64p, i64p]
    L.glu_autotune.argtypes = [vp, C.c_int32, vp, C.c_int32, C.POINTER(Options),
                               C.POINTER(C.c_double), vp]
    L.glu_solve.argtypes = [vp, C.c_int32, vp, vp, C.c_int, vp]
    L.glu_plan_set_original_pattern.argtypes = [vp, C.c_uint64, u32p, u32p]
    L.glu_residual.argtypes = [vp, C.c_int32, vp, vp, vp, C.c_int, vp, vp]
    L.glu_residual_noalloc.argtypes = [vp, C.c_int32, vp, vp, vp, C.c_int, vp, vp]
    L.glu_refine.argtypes = [vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_int, vp, vp]
    L.glu_grad_a.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
    L.glu_get_lu.argtypes = [vp, C.c_int32, vp, vp]
    L.glu_graph_capture.argtypes = [vp, vp, C.c_int32, vp, vp, C.c_double, C.c_int32, vp]
    L.glu_graph_launch.argtypes = [vp, vp]
    L.glu_batch_launch_count.argtypes = [vp, C.POINTER(C.c_int64)]
    L.glu_debug_refactor_unreachable_barrier.argtypes = [vp, C.c_double, vp]
    L.glu_group_capture.argtypes = [C.c_int32, C.POINTER(vp), C.POINTER(vp), C.POINTER(C.c_int32),
                                    C.POINTER(vp), C.POINTER(vp), C.c_double, C.c_int32, vp,
                                    C.POINTER(vp)]
    L.glu_group_launch.argtypes = [vp, vp]
    L.glu_group_launch_count.argtypes = [vp, C.POINTER(C.c_int64)]
    L.glu_group_destroy.argtypes = [vp]
    L.glu_debug_gemm_sub.argtypes = [C.c_int32, C.c_int32, C.c_int32, vp, C.c_int32, vp,
                                     C.c_int32, vp, C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                     C.c_int64, C.c_int32, vp]
    _lib = L
    return L


def check(status: int, what: str) -> None:
    if status != GLU_OK:
        raise GluError(status, what)


def default_options(**kw) -> Options:
    o = Options()
    lib().glu_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
