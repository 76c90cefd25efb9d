"""Device context, precision settings and the per-structure caches of device tables/plans.

One `Context` per CUDA device wraps a libtkb200 context bound to a dedicated torch CUDA
stream (capturable in CUDA graphs). Device tables (flattened tree transformers) and grouped
GEMM plans are cached per structure, the counterpart of TensorKit's `@cached` treebraider
(src/tensors/treetransformers.jl:156-167, LRU size `src/auxiliary/caches.jl:19`).
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from collections import OrderedDict
from contextlib import contextmanager

import numpy as np

from . import _lib as L

__all__ = ["Context", "get_context", "precision", "set_precision", "B200Backend",
           "DeviceTable", "GemmPlan", "ReducePlan", "launch_count"]

_DEFAULT_CACHE = 10_000


class _Settings(threading.local):
    def __init__(self):
        self.precision = os.environ.get("TKB_PRECISION", "plain")   # "plain" | "split" | "auto"
        self.slices = int(os.environ.get("TKB_SLICES", "0"))        # 0 = automatic


_settings = _Settings()


def precision():
    return _settings.precision, _settings.slices


def set_precision(mode: str, slices: int = 0):
    if mode not in ("plain", "split", "auto"):
        raise ValueError("precision must be 'plain', 'split' or 'auto'")
    _settings.precision = mode
    _settings.slices = int(slices)


@contextmanager
def using_precision(mode: str, slices: int = 0):
    old = (_settings.precision, _settings.slices)
    set_precision(mode, slices)
    try:
        yield
    finally:
        _settings.precision, _settings.slices = old


class B200Backend:
    """Marker passed as `backend=` (TensorOperations' AbstractBackend analogue,
    src/TensorKit.jl:117); selects the libtkb200 path, with an optional precision."""

    def __init__(self, precision: str | None = None, slices: int = 0):
        self.precision = precision
        self.slices = slices


class _LRU(OrderedDict):
    def __init__(self, maxsize, on_evict=None):
        super().__init__()
        self.maxsize = maxsize
        self.on_evict = on_evict

    def get_or(self, key, make):
        if key in self:
            self.move_to_end(key)
            return self[key]
        v = make()
        self[key] = v
        if len(self) > self.maxsize:
            _, old = self.popitem(last=False)
            if self.on_evict:
                self.on_evict(old)
        return v


class DeviceTable:
    """A flattened transformer uploaded to the device."""

    def __init__(self, ctx: "Context", flat, src_len, dst_len):
        self.ctx = ctx
        self.flat = flat
        d = L.tkb_table_desc()
        d.nind = flat.nind
        for k in range(flat.nind):
            d.perm[k] = int(flat.perm[k])
        d.ngroups = flat.ngroups
        self._keep = [flat.group_src_ptr, flat.group_dst_ptr, flat.coeff_ptr, flat.coeffs,
                      np.ascontiguousarray(flat.sizes), np.ascontiguousarray(flat.src_strides),
                      flat.src_offsets, np.ascontiguousarray(flat.dst_strides), flat.dst_offsets]
        (d.group_src_ptr, d.group_dst_ptr, d.coeff_ptr, d.coeffs, d.sizes, d.src_strides,
         d.src_offsets, d.dst_strides, d.dst_offsets) = [L.ptr(a) for a in self._keep]
        d.src_len = int(src_len)
        d.dst_len = int(dst_len)
        h = C.c_void_p()
        L.check(ctx.lib.tkb_table_create(ctx.handle, C.byref(d), C.byref(h)), ctx.handle)
        self.handle = h
        nt, er, ew = C.c_int64(), C.c_int64(), C.c_int64()
        L.check(ctx.lib.tkb_table_info(h, C.byref(nt), C.byref(er), C.byref(ew)))
        self.ntasks, self.elems_read, self.elems_written = nt.value, er.value, ew.value

    def free(self):
        if self.handle:
            self.ctx.lib.tkb_table_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GemmPlan:
    def __init__(self, ctx: "Context", blocks, lens, dtype_code, precision_code, slices, tuning=None):
        """blocks: list of (m, n, k, offA, offB, offC, lda, ldb, ldc, opA, opB); tuning:
        (max_pieces, min_piece_steps) of the split-K decomposition, or None for the default."""
        self.ctx = ctx
        nb = len(blocks)
        arr = np.array(blocks, dtype=np.int64).reshape(nb, 11) if nb else np.zeros((0, 11), np.int64)
        cols = [np.ascontiguousarray(arr[:, i]) for i in range(9)]
        ops = [np.ascontiguousarray(arr[:, 9].astype(np.int32)), np.ascontiguousarray(arr[:, 10].astype(np.int32))]
        self._keep = cols + ops
        d = L.tkb_gemm_desc()
        d.nblocks = nb
        (d.m, d.n, d.k, d.offA, d.offB, d.offC, d.lda, d.ldb, d.ldc) = [L.ptr(c) for c in cols]
        d.opA, d.opB = L.ptr(ops[0]), L.ptr(ops[1])
        d.lenA, d.lenB, d.lenC = [int(x) for x in lens]
        d.dtype = dtype_code
        d.precision = precision_code
        d.slices = slices
        h = C.c_void_p()
        if tuning is None:
            L.check(ctx.lib.tkb_gemm_plan_create(ctx.handle, C.byref(d), C.byref(h)), ctx.handle)
        else:
            tn = L.tkb_gemm_tuning(int(tuning[0]), int(tuning[1]))
            L.check(ctx.lib.tkb_gemm_plan_create_tuned(ctx.handle, C.byref(d), C.byref(tn), C.byref(h)),
                    ctx.handle)
        self.handle = h
        self.tuning = tuning
        fl, sl = C.c_double(), C.c_int32()
        L.check(ctx.lib.tkb_gemm_plan_info(h, C.byref(fl), C.byref(sl)))
        self.flops, self.slices = fl.value, sl.value
        self.blocks = arr
        self.is_complex = dtype_code == L.TKB_C128

    def last_slices(self):
        """(slice count per block of the last launch, tiles the error check sent to FP64).
        Per block: 3..7 slices, 0 = the block ran in FP64, -1 = no products (k = 0, skinny
        block or plain precision). Waits for the library stream."""
        nb = len(self.blocks)
        out = np.zeros(nb + 1, dtype=np.int32)
        L.check(self.ctx.lib.tkb_gemm_plan_slices(self.ctx.handle, self.handle, L.ptr(out), nb + 1),
                self.ctx.handle)
        return out[:nb].tolist(), int(out[nb])

    def free(self):
        if self.handle:
            self.ctx.lib.tkb_gemm_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class ReducePlan:
    def __init__(self, ctx: "Context", segs, length):
        """segs: list of (offset, count, stride, weight)."""
        self.ctx = ctx
        n = len(segs)
        off = np.array([s[0] for s in segs], np.int64)
        cnt = np.array([s[1] for s in segs], np.int64)
        st = np.array([s[2] for s in segs], np.int64)
        w = np.array([s[3] for s in segs], np.float64)
        self._keep = (off, cnt, st, w)
        h = C.c_void_p()
        L.check(ctx.lib.tkb_rplan_create(ctx.handle, n, L.ptr(off), L.ptr(cnt), L.ptr(st), L.ptr(w),
                                         int(length), C.byref(h)), ctx.handle)
        self.handle = h

    def free(self):
        if self.handle:
            self.ctx.lib.tkb_rplan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """libtkb200 context on one device with its own torch stream."""

    def __init__(self, device: int = 0, workspace_bytes: int = 64 << 20):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("the B200 path needs a CUDA device; no CPU fallback exists")
        self.lib = L.load()
        self.device = device
        self.torch_device = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(device=self.torch_device)
        h = C.c_void_p()
        L.check(self.lib.tkb_ctx_create(device, C.c_void_p(self.stream.cuda_stream),
                                        workspace_bytes, C.byref(h)))
        self.handle = h
        self.tables = _LRU(_DEFAULT_CACHE, lambda t: t.free())
        self.plans = _LRU(_DEFAULT_CACHE, lambda p: p.free())
        self.rplans = _LRU(_DEFAULT_CACHE, lambda p: p.free())

    def synchronize(self):
        L.check(self.lib.tkb_ctx_synchronize(self.handle), self.handle)

    def launch_count(self) -> int:
        v = C.c_int64()
        L.check(self.lib.tkb_ctx_launch_count(self.handle, C.byref(v)))
        return v.value

    def empty_caches(self):
        for cache in (self.tables, self.plans, self.rplans):
            for v in cache.values():
                v.free()
            cache.clear()


_contexts: dict = {}
_ctx_lock = threading.Lock()


def get_context(device: int | None = None) -> Context:
    import torch
    if device is None:
        device = torch.cuda.current_device() if torch.cuda.is_available() else 0
    with _ctx_lock:
        c = _contexts.get(device)
        if c is None:
            c = Context(device)
            _contexts[device] = c
        return c


def launch_count(device: int | None = None) -> int:
    return get_context(device).launch_count()


def empty_globalcaches():
    """Counterpart of TensorKit.empty_globalcaches! (src/auxiliary/caches.jl:2-5)."""
    from . import structure, treetransformers, fusiontrees
    structure.sectorstructure.cache_clear()
    structure.degeneracystructure.cache_clear()
    structure.fusionblocks.cache_clear()
    treetransformers._TRANSFORMER_CACHE.clear()
    fusiontrees._FSBRAID_CACHE.clear()
    for c in _contexts.values():
        c.empty_caches()
