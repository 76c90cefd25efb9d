"""ctypes binding of libtkb200.so (declared in include/tkb200.h).

The library is built in-tree by `tensorkit_b200._build.build()`; loading fails loudly
when it is missing — there is no CPU fallback for device tensors.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

LIBDIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib")
LIBPATH = os.path.join(LIBDIR, "libtkb200.so")

TKB_MAX_IND = 8
TKB_OK, TKB_ERR_ARG, TKB_ERR_SIZE, TKB_ERR_OOM, TKB_ERR_CUDA, TKB_ERR_TIMEOUT, \
    TKB_ERR_UNSUPPORTED = range(7)
TKB_F64, TKB_C128 = 0, 1
TKB_PLAIN, TKB_SPLIT_INT8 = 0, 1
TKB_OP_N, TKB_OP_T, TKB_OP_C = 0, 1, 2
TKB_NORM2, TKB_INNER, TKB_TRACE = 0, 1, 2

EXPORTS = [
    "tkb_version", "tkb_ctx_create", "tkb_ctx_destroy", "tkb_ctx_set_stream",
    "tkb_ctx_synchronize", "tkb_selftest_bounded_wait", "tkb_ctx_launch_count", "tkb_last_error",
    "tkb_table_create",
    "tkb_table_destroy", "tkb_table_info", "tkb_treetransform", "tkb_trace_table_create",
    "tkb_trace_table_destroy", "tkb_tracetransform", "tkb_gemm_plan_create", "tkb_gemm_plan_create_tuned",
    "tkb_gemm_plan_destroy", "tkb_gemm_plan_info", "tkb_gemm_plan_slices", "tkb_grouped_gemm",
    "tkb_rplan_create",
    "tkb_rplan_destroy", "tkb_reduce", "tkb_reduce_async", "tkb_reduce_noalloc",
    "tkb_graph_begin", "tkb_graph_end",
    "tkb_graph_launch", "tkb_graph_destroy",
]


class tkb_scalar(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class tkb_table_desc(C.Structure):
    _fields_ = [
        ("nind", C.c_int32), ("perm", C.c_int32 * TKB_MAX_IND), ("ngroups", C.c_int64),
        ("group_src_ptr", C.c_void_p), ("group_dst_ptr", C.c_void_p), ("coeff_ptr", C.c_void_p),
        ("coeffs", C.c_void_p), ("sizes", C.c_void_p), ("src_strides", C.c_void_p),
        ("src_offsets", C.c_void_p), ("dst_strides", C.c_void_p), ("dst_offsets", C.c_void_p),
        ("src_len", C.c_int64), ("dst_len", C.c_int64),
    ]


class tkb_trace_desc(C.Structure):
    _fields_ = [
        ("nfree", C.c_int32), ("ntrace", C.c_int32), ("ngroups", C.c_int64),
        ("group_entry_ptr", C.c_void_p), ("sizes", C.c_void_p), ("dst_strides", C.c_void_p),
        ("dst_offsets", C.c_void_p), ("src_strides", C.c_void_p), ("trace_sizes", C.c_void_p),
        ("trace_strides", C.c_void_p), ("src_offsets", C.c_void_p), ("coeffs", C.c_void_p),
        ("src_len", C.c_int64), ("dst_len", C.c_int64),
    ]


class tkb_gemm_desc(C.Structure):
    _fields_ = [
        ("nblocks", C.c_int64), ("m", C.c_void_p), ("n", C.c_void_p), ("k", C.c_void_p),
        ("offA", C.c_void_p), ("offB", C.c_void_p), ("offC", C.c_void_p),
        ("lda", C.c_void_p), ("ldb", C.c_void_p), ("ldc", C.c_void_p),
        ("opA", C.c_void_p), ("opB", C.c_void_p),
        ("lenA", C.c_int64), ("lenB", C.c_int64), ("lenC", C.c_int64),
        ("dtype", C.c_int32), ("precision", C.c_int32), ("slices", C.c_int32),
    ]


class tkb_gemm_tuning(C.Structure):
    _fields_ = [("max_pieces", C.c_int32), ("min_piece_steps", C.c_int32)]


class TKBError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libtkb200 error {code}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()


def _declare(lib):
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int32, C.c_double
    P = C.POINTER
    sig = {
        "tkb_version": ([], C.c_int),
        "tkb_ctx_create": ([C.c_int, vp, C.c_size_t, P(vp)], C.c_int),
        "tkb_ctx_destroy": ([vp], C.c_int),
        "tkb_ctx_set_stream": ([vp, vp], C.c_int),
        "tkb_ctx_synchronize": ([vp], C.c_int),
        "tkb_selftest_bounded_wait": ([vp, i64], C.c_int),
        "tkb_ctx_launch_count": ([vp, P(i64)], C.c_int),
        "tkb_last_error": ([vp], C.c_char_p),
        "tkb_table_create": ([vp, P(tkb_table_desc), P(vp)], C.c_int),
        "tkb_table_destroy": ([vp], C.c_int),
        "tkb_table_info": ([vp, P(i64), P(i64), P(i64)], C.c_int),
        "tkb_treetransform": ([vp, vp, C.c_int, vp, vp, tkb_scalar, tkb_scalar, C.c_int], C.c_int),
        "tkb_trace_table_create": ([vp, P(tkb_trace_desc), P(vp)], C.c_int),
        "tkb_trace_table_destroy": ([vp], C.c_int),
        "tkb_tracetransform": ([vp, vp, C.c_int, vp, vp, tkb_scalar, tkb_scalar, C.c_int], C.c_int),
        "tkb_gemm_plan_create": ([vp, P(tkb_gemm_desc), P(vp)], C.c_int),
        "tkb_gemm_plan_create_tuned": ([vp, P(tkb_gemm_desc), P(tkb_gemm_tuning), P(vp)], C.c_int),
        "tkb_gemm_plan_destroy": ([vp], C.c_int),
        "tkb_gemm_plan_info": ([vp, P(dbl), P(i32)], C.c_int),
        "tkb_gemm_plan_slices": ([vp, vp, vp, i64], C.c_int),
        "tkb_grouped_gemm": ([vp, vp, vp, vp, vp, tkb_scalar, tkb_scalar], C.c_int),
        "tkb_rplan_create": ([vp, i64, vp, vp, vp, vp, i64, P(vp)], C.c_int),
        "tkb_rplan_destroy": ([vp], C.c_int),
        "tkb_reduce": ([vp, vp, C.c_int, C.c_int, vp, vp, P(dbl)], C.c_int),
        "tkb_reduce_async": ([vp, vp, C.c_int, C.c_int, vp, vp, vp], C.c_int),
        "tkb_reduce_noalloc": ([C.c_int, vp, C.c_int, C.c_int, vp, vp, i64, i64, vp, vp, vp, vp,
                                P(dbl)], C.c_int),
        "tkb_graph_begin": ([vp], C.c_int),
        "tkb_graph_end": ([vp, P(vp)], C.c_int),
        "tkb_graph_launch": ([vp, vp], C.c_int),
        "tkb_graph_destroy": ([vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


def load(path: str = LIBPATH):
    """Load the shared library (idempotent)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise ImportError(
                    f"libtkb200.so not found at {path}; build it with tensorkit_b200._build.build()")
            _lib = _declare(C.CDLL(path))
        return _lib


def check(code, ctx=None):
    if code != TKB_OK:
        lib = load()
        msg = lib.tkb_last_error(ctx)
        raise TKBError(code, msg.decode() if msg else "")


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)
