"""Partial traces on device tensors: TensorKit's `trace_permute!` and `TO.tensortrace!`.

Follows `src/tensors/tensoroperations.jl` (bosonic sectors):
- `TO.tensortrace!(C, A, p, q, conjA, α, β)` (`:83-98`) realises conj(A) through the lazy
  adjoint and `adjointtensorindices`, then calls `trace_permute!`;
- `trace_permute!(tdst, tsrc, (p₁, p₂), (q₁, q₂), α, β)` (`:212-244`) checks the spaces
  (`space(tdst) == select(space(tsrc), (p₁, p₂))`, `space(tsrc, q₁[i]) == dual(space(tsrc,
  q₂[i]))`) and runs `_trace_permute!` (`:246-296`): β scales the destination, every source
  tree pair (or fusion block, with its recoupling matrix U) is permuted to ((p₁, q₁),
  (p₂, q₂)), both trees are split after the kept legs, pairs whose split-off trees differ
  are dropped, the others contribute coeff·dim(g.coupled)/dim(g.uncoupled[1]) times the
  dense partial trace of the source sub-block. Twists are trivial for bosonic sectors.

All of that recoupling is resolved on the host once per structure into a trace table
(grouped by destination sub-block) and executed by one libtkb200 launch
(`tkb_tracetransform`).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .backend import get_context
from .fusiontrees import braid as _braid_trees
from .fusiontrees import split
from .spaces import SpaceMismatch
from .structure import fusionblocks, sectorstructure, subblockstructure
from .tensor import AdjointTensorMap, TensorMap, new_tensor
from .treetransformers import _adjoint_subblocks

__all__ = ["trace_permute_", "trace_permute", "TraceFlat", "build_trace_table", "TraceTable"]


class TraceFlat:
    """Host form of a trace table (arrays as in `tkb_trace_desc`)."""

    def __init__(self, nfree, ntrace, group_entry_ptr, sizes, dst_strides, dst_offsets,
                 src_strides, trace_sizes, trace_strides, src_offsets, coeffs):
        self.nfree, self.ntrace = int(nfree), int(ntrace)
        as64 = lambda a: np.ascontiguousarray(a, dtype=np.int64)
        self.group_entry_ptr = as64(group_entry_ptr)
        self.sizes = as64(sizes)
        self.dst_strides = as64(dst_strides)
        self.dst_offsets = as64(dst_offsets)
        self.src_strides = as64(src_strides)
        self.trace_sizes = as64(trace_sizes)
        self.trace_strides = as64(trace_strides)
        self.src_offsets = as64(src_offsets)
        self.coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)

    @property
    def ngroups(self):
        return len(self.group_entry_ptr) - 1


def build_trace_table(Vsrc, p, q, src_adjoint_of=None) -> TraceFlat:
    """Flatten trace_permute!(·, tsrc, p, q) for a source of space Vsrc (a lazy adjoint of a
    tensor of space `src_adjoint_of` when given)."""
    p1, p2 = tuple(p[0]), tuple(p[1])
    q1, q2 = tuple(q[0]), tuple(q[1])
    N1, N2 = len(p1), len(p2)
    Vdst = Vsrc.select((p1, p2))
    fts_src = subblockstructure(Vsrc) if src_adjoint_of is None else _adjoint_subblocks(src_adjoint_of)
    fts_dst = subblockstructure(Vdst)
    r = (p1 + q1, p2 + q2)
    n1, n = Vsrc.numout(), Vsrc.numind()
    levels = (tuple(range(1, n1 + 1)), tuple(range(n1 + 1, n + 1)))
    contrib: dict = {}

    def add(pair, f1p, f2p, x):
        h1, g1 = split(f1p, N1)
        h2, g2 = split(f2p, N2)
        if g1 != g2:
            return
        x = x * g1.coupled.dim() / g1.uncoupled[0].dim()
        contrib.setdefault((h1, h2), []).append((pair, x))

    if Vsrc.unit().fusionstyle == "unique":
        for pair in sectorstructure(Vsrc).fusiontrees:
            (f1p, f2p), x = _braid_trees(pair, r, levels)
            if x != 0.0:
                add(pair, f1p, f2p, x)
    else:
        for blk in fusionblocks(Vsrc):
            dst, U = _braid_trees(blk, r, levels)
            for i, pair in enumerate(blk.trees):
                for j, (f1p, f2p) in enumerate(dst.trees):
                    x = float(U[j, i])
                    if x != 0.0:
                        add(pair, f1p, f2p, x)
    free = p1 + p2
    gptr, sizes, dstr, doff = [0], [], [], []
    sstr, tsz, tstr, soff, coef = [], [], [], [], []
    for pair in sectorstructure(Vdst).fusiontrees:
        dsz, dst_st, off = fts_dst[pair]
        sizes.extend(dsz)
        dstr.extend(dst_st)
        doff.append(off)
        for spair, x in contrib.get(pair, ()):
            ssz, sst, so = fts_src[spair]
            sstr.extend(sst[k - 1] for k in free)
            tsz.extend(ssz[a - 1] for a in q1)
            tstr.extend(sst[a - 1] + sst[b - 1] for a, b in zip(q1, q2))
            soff.append(so)
            coef.append(x)
        gptr.append(len(soff))
    return TraceFlat(N1 + N2, len(q1), gptr, sizes, dstr, doff, sstr, tsz, tstr, soff, coef)


class TraceTable:
    """A trace table uploaded to the device."""

    def __init__(self, ctx, flat: TraceFlat, src_len, dst_len):
        self.ctx = ctx
        self.flat = flat
        d = L.tkb_trace_desc()
        d.nfree, d.ntrace, d.ngroups = flat.nfree, flat.ntrace, flat.ngroups
        self._keep = [flat.group_entry_ptr, flat.sizes, flat.dst_strides, flat.dst_offsets,
                      flat.src_strides, flat.trace_sizes, flat.trace_strides, flat.src_offsets,
                      flat.coeffs]
        (d.group_entry_ptr, d.sizes, d.dst_strides, d.dst_offsets, d.src_strides, d.trace_sizes,
         d.trace_strides, d.src_offsets, d.coeffs) = [L.ptr(a) for a in self._keep]
        d.src_len, d.dst_len = int(src_len), int(dst_len)
        h = C.c_void_p()
        L.check(ctx.lib.tkb_trace_table_create(ctx.handle, C.byref(d), C.byref(h)), ctx.handle)
        self.handle = h

    def free(self):
        if self.handle:
            self.ctx.lib.tkb_trace_table_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _norm(p):
    return (tuple(int(i) for i in p[0]), tuple(int(i) for i in p[1]))


def trace_permute_(tdst: TensorMap, tsrc, p, q, alpha=1.0, beta=0.0):
    """tdst = β·tdst + α·(tsrc permuted by p with the leg pairs q traced)."""
    from .indexmanipulations import _check_device, _scalar, _sync_in, _sync_out, dtype_code
    from . import indexmanipulations as IM
    p, q = _norm(p), _norm(q)
    if len(q[0]) != len(q[1]):
        raise ValueError("number of trace indices does not match")
    if len(q[0]) == 0:
        return IM.permute_(tdst, tsrc, p, alpha, beta)
    W = tsrc.space
    if tdst.space != W.select(p):
        raise SpaceMismatch(f"trace: tsrc = {W}, tdst = {tdst.space}, p = {p}")
    if any(W[a] != W[b].dual() for a, b in zip(q[0], q[1])):
        raise SpaceMismatch(f"trace: tsrc = {W}, q = {q}")
    _check_device(tdst, tsrc)
    if tdst.data.dtype != tsrc.data.dtype:
        raise TypeError("source and destination must share their scalar type")
    ctx = get_context(tdst.data.device.index)
    parent = tsrc.parent.space if isinstance(tsrc, AdjointTensorMap) else None
    src_len = parent.dim() if parent is not None else W.dim()
    key = ("trace", tdst.space, W, p, q, parent)
    table = ctx.tables.get_or(key, lambda: TraceTable(ctx, build_trace_table(W, p, q, parent),
                                                      src_len, tdst.space.dim()))
    conj = 1 if (isinstance(tsrc, AdjointTensorMap) and tsrc.is_complex()) else 0
    if IM.LAUNCH_LOG is not None:
        IM.LAUNCH_LOG.append(("trace", table, tdst, tsrc, complex(alpha), complex(beta), conj))
    _sync_in(ctx, tdst, tsrc)
    L.check(ctx.lib.tkb_tracetransform(ctx.handle, table.handle, dtype_code(tdst.data),
                                       C.c_void_p(tdst.data.data_ptr()),
                                       C.c_void_p(tsrc.data.data_ptr()),
                                       _scalar(alpha), _scalar(beta), conj), ctx.handle)
    _sync_out(ctx, tdst)
    return tdst


def trace_permute(tsrc, p, q, alpha=1.0):
    """New tensor α·(tsrc permuted by p with the leg pairs q traced)."""
    p = _norm(p)
    tdst = new_tensor(tsrc.space.select(p), tsrc.data.dtype, tsrc.data.device)
    return trace_permute_(tdst, tsrc, p, q, alpha, 0.0)
