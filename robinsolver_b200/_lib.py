"""ctypes binding of librobin_b200.so (the C-ABI declared in include/robin_b200.h).

The library is loaded from this package directory.  There is no fallback: if the shared
library is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librobin_b200.so"

RB_OK = 0
RB_ERR_INVALID = -1
RB_ERR_DOMAIN = -2
RB_ERR_BNDRY_PARAMS = -3
RB_ERR_NOT_FACTORED = -4
RB_ERR_DIM_MISMATCH = -5
RB_ERR_GEOMETRY = -6
RB_ERR_UNSUPPORTED = -7
RB_ERR_CUDA = -8
RB_ERR_OUT_OF_MEMORY = -9
RB_ERR_NUMERIC = -10
RB_ERR_NO_SOLUTION = -11

RB_PREC_FP64 = 0
RB_PREC_MIXED = 1

RB_POINTS_POTENTIAL = 0
RB_POINTS_SOURCE = 1
RB_POINTS_BOUNDARY = 2
RB_POINTS_SOLUTION = 3

RB_FLAG_SKIP_ROOT_RTR = 1
RB_FLAG_VERBOSE = 2
RB_FLAG_NO_GRAPHS = 4
RB_FLAG_MERGE_DS = 8
RB_FLAG_ASYNC_FACTOR = 16
RB_FLAG_MIXED_INT8_TOP = 32
RB_FIELD_BUMP_POTENTIAL = 0
RB_FIELD_POINT_SOURCE = 1
RB_FIELD_PLANE_WAVE = 2

# every entry point include/robin_b200.h declares
EXPORTS = [
    "rb_tree_create", "rb_tree_destroy", "rb_last_error", "rb_tree_info", "rb_tree_sample_points",
    "rb_tree_factor", "rb_tree_factor_device", "rb_tree_solve", "rb_tree_solve_device",
    "rb_get_solution", "rb_get_solution_device", "rb_get_solution_async", "rb_tree_sync", "rb_tree_times",
    "rb_tree_stream",
    "rb_tree_set_timing", "rb_tree_stage_times", "rb_tree_clear_stage_times", "rb_tree_level_shape", "rb_tree_get_rtr", "rb_tree_launch_counts",
    "rb_leaf_rtr_noalloc",
    "rb_tree_sample_device", "rb_check_solution", "rb_check_solution_device", "rb_tree_save", "rb_tree_load",
    "rb_tree_set_refinement", "rb_tree_refine_info",
    "rb_server_create", "rb_server_destroy", "rb_server_last_error", "rb_server_now", "rb_server_add_tree",
    "rb_server_tree_info", "rb_server_submit_factor", "rb_server_submit_solve", "rb_server_wait", "rb_server_get_stats",
    "rb_forest_create", "rb_forest_destroy", "rb_forest_last_error", "rb_forest_factor", "rb_forest_info",
    "rb_forest_tuning", "rb_gemm_engine_name",
]


class rb_geom(C.Structure):
    _fields_ = [
        ("d", C.c_int32),
        ("L", C.c_int32),
        ("domain", C.c_double * 6),
        ("h_tgt", C.c_double),
        ("kb", C.c_double),
        ("bndry_params", C.c_double * 8),
        ("ordering", C.c_int32),
        ("flags", C.c_int32),
        ("device_budget", C.c_int64),
    ]


class rb_info(C.Structure):
    _fields_ = [
        ("nleaves", C.c_int32),
        ("leaf_a", C.c_int32),
        ("leaf_b", C.c_int32),
        ("leaf_n", C.c_int32),
        ("leaf_nb", C.c_int32),
        ("root_nb", C.c_int32),
        ("root_a", C.c_int32),
        ("root_b", C.c_int32),
        ("h_last", C.c_double * 3),
        ("n_interior", C.c_int64),
        ("device_bytes", C.c_int64),
        ("factored", C.c_int32),
        ("nrhs", C.c_int32),
        ("d", C.c_int32),
        ("leaf_c", C.c_int32),
        ("root_c", C.c_int32),
        ("reserved", C.c_int32),
    ]


class rb_server_opts(C.Structure):
    _fields_ = [
        ("device_budget", C.c_int64),
        ("max_batch_rhs", C.c_int32),
        ("precision", C.c_int32),
        ("tol", C.c_double),
    ]


class rb_server_stats(C.Structure):
    _fields_ = [
        ("solves", C.c_int64), ("rhs", C.c_int64), ("factors", C.c_int64), ("batches", C.c_int64),
        ("failed", C.c_int64),
        ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
        ("factor_p50_ms", C.c_double), ("factor_max_ms", C.c_double),
        ("reserved_bytes", C.c_int64),
    ]


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m robinsolver_b200.build`")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    sig = {
        "rb_tree_create": (C.c_int, [C.POINTER(rb_geom), C.POINTER(P)]),
        "rb_tree_destroy": (C.c_int, [P]),
        "rb_last_error": (C.c_char_p, [P]),
        "rb_tree_info": (C.c_int, [P, C.POINTER(rb_info)]),
        "rb_tree_sample_points": (C.c_int, [P, C.c_int, D]),
        "rb_tree_factor": (C.c_int, [P, D, C.c_int]),
        "rb_tree_factor_device": (C.c_int, [P, P, C.c_int, C.c_int]),
        "rb_tree_solve": (C.c_int, [P, C.c_int, D, D]),
        "rb_tree_solve_device": (C.c_int, [P, C.c_int, P, P, C.c_int]),
        "rb_get_solution": (C.c_int, [P, C.c_int, D, D]),
        "rb_get_solution_device": (C.c_int, [P, P, C.c_int]),
        "rb_get_solution_async": (C.c_int, [P, C.c_int, D, D]),
        "rb_tree_sync": (C.c_int, [P]),
        "rb_tree_times": (C.c_int, [P, D, D]),
        "rb_tree_stream": (P, [P]),
        "rb_tree_set_timing": (C.c_int, [P, C.c_int]),
        "rb_tree_stage_times": (C.c_int, [P, D, D, C.POINTER(C.c_char_p), C.c_int]),
        "rb_tree_clear_stage_times": (C.c_int, [P]),
        "rb_tree_level_shape": (C.c_int, [P, C.c_int, C.POINTER(C.c_int32)]),
        "rb_tree_get_rtr": (C.c_int, [P, C.c_int, C.c_int, D]),
        "rb_tree_launch_counts": (C.c_int, [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "rb_leaf_rtr_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_double, P, P, C.c_int, P, P]),
        "rb_tree_sample_device": (C.c_int, [P, C.c_int, C.c_int, D, P, P, C.c_int]),
        "rb_check_solution": (C.c_int, [P, C.c_int, D, C.c_int, C.c_int, D]),
        "rb_check_solution_device": (C.c_int, [P, C.c_int, P, C.c_int, C.c_int, D]),
        "rb_tree_save": (C.c_int, [P, C.c_char_p]),
        "rb_tree_load": (C.c_int, [C.c_char_p, C.POINTER(P)]),
        "rb_tree_set_refinement": (C.c_int, [P, C.c_double, C.c_int]),
        "rb_tree_refine_info": (C.c_int, [P, C.POINTER(C.c_int32), D, D, D]),
        "rb_server_create": (C.c_int, [C.POINTER(rb_server_opts), C.POINTER(P)]),
        "rb_server_destroy": (C.c_int, [P]),
        "rb_server_last_error": (C.c_char_p, [P]),
        "rb_server_now": (C.c_double, [P]),
        "rb_server_add_tree": (C.c_int, [P, C.POINTER(rb_geom), C.POINTER(C.c_int32)]),
        "rb_server_tree_info": (C.c_int, [P, C.c_int32, C.POINTER(rb_info)]),
        "rb_server_submit_factor": (C.c_int, [P, C.c_int32, D, C.c_int, D, C.c_double, C.POINTER(C.c_int64)]),
        "rb_server_submit_solve": (C.c_int, [P, C.c_int32, C.c_int, C.c_int, D, P, P, P, C.c_double,
                                             C.POINTER(C.c_int64)]),
        "rb_server_wait": (C.c_int, [P, C.c_int64, C.c_double]),
        "rb_server_get_stats": (C.c_int, [P, C.POINTER(rb_server_stats), C.c_int]),
        "rb_forest_create": (C.c_int, [C.POINTER(P), C.c_int, C.POINTER(P)]),
        "rb_forest_destroy": (C.c_int, [P]),
        "rb_forest_last_error": (C.c_char_p, [P]),
        "rb_forest_factor": (C.c_int, [P, C.POINTER(P), C.c_int]),
        "rb_forest_info": (C.c_int, [P, D, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
        "rb_forest_tuning": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32), D,
                                       C.c_int]),
        "rb_gemm_engine_name": (C.c_char_p, [C.c_int]),
        # test hooks of the GEMM engines (rb_testing.cpp), not part of the drop-in boundary
        "rb_test_zgemm": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_longlong, C.c_longlong, P,
                                    C.c_longlong, C.c_longlong, P, C.c_longlong, C.c_longlong, C.c_double,
                                    C.c_double, C.c_double, C.c_double, C.c_int]),
        "rb_test_zgemm_timed": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_longlong, C.c_longlong, P,
                                          C.c_longlong, C.c_longlong, P, C.c_longlong, C.c_longlong, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, D]),
        # test hook of the batched Gauss-Jordan inversion (rb_testing.cpp)
        "rb_test_zinvert": (C.c_int, [C.c_int, C.c_int, P, C.c_longlong, C.c_longlong, C.c_int, D]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error(handle=None) -> str:
    msg = lib.rb_last_error(handle)
    return msg.decode() if msg else ""


def dptr(a):
    """double* of a contiguous numpy array (float64 or complex128)."""
    return a.ctypes.data_as(C.POINTER(C.c_double))
