"""permute / braid / transpose / add_transform! on device tensors.

Follows `src/tensors/indexmanipulations.jl`:
- `permute!(tdst, tsrc, p, α, β)` = `braid!` with levels 1..N (`:217-225`);
- `permute(t, p; copy)` shares data when p is the identity (`:242-258`);
- `braid!` builds (or fetches) the cached transformer and calls `add_transform!`
  (`:304-318`, `:557-580`);
- `add_transform_kernel!` (`:658-726`) is one libtkb200 launch over every sub-block.

A lazy adjoint source (`AdjointTensorMap`) is read from its parent's data with complex
conjugation; its transformer is built over the adjoint space and addresses the parent's
sub-blocks (`src/tensors/adjoint.jl:47-51`).

Bosonic sectors only (U1, SU2, U1⊠SU2): twists are trivial (`:42-43`) and `transpose`
equals `permute` for a cyclic permutation, so both go through the braid tables.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from .backend import DeviceTable, get_context
from .spaces import SpaceMismatch
from .tensor import AdjointTensorMap, TensorMap, new_tensor
from .treetransformers import flatten_transformer, treebraider, treeflipper, treetransposer

__all__ = ["permute", "permute_", "braid", "braid_", "add_transform_", "transpose",
           "transpose_", "repartition", "device_table", "dtype_code"]


# every device launch issued while this list is installed is recorded (used to re-time
# individual kernels of a network)
LAUNCH_LOG: list | None = None


def relaunch(entry):
    """Re-issue one recorded launch with the same operands (for kernel timing)."""
    ctx = entry[1].ctx
    if entry[0] in ("transform", "trace"):
        _, table, tdst, tsrc, a, b, conj = entry
        fn = ctx.lib.tkb_treetransform if entry[0] == "transform" else ctx.lib.tkb_tracetransform
        L.check(fn(ctx.handle, table.handle, dtype_code(tdst.data), C.c_void_p(tdst.data.data_ptr()),
                   C.c_void_p(tsrc.data.data_ptr()), _scalar(a), _scalar(b), conj), ctx.handle)
    else:
        _, plan, tC, tA, tB, a, b = entry
        L.check(ctx.lib.tkb_grouped_gemm(ctx.handle, plan.handle, C.c_void_p(tC.data.data_ptr()),
                                         C.c_void_p(tA.data.data_ptr()), C.c_void_p(tB.data.data_ptr()),
                                         _scalar(a), _scalar(b)), ctx.handle)


def dtype_code(t):
    import torch
    if t.dtype == torch.float64:
        return L.TKB_F64
    if t.dtype == torch.complex128:
        return L.TKB_C128
    raise TypeError(f"unsupported dtype {t.dtype}; the path computes in float64/complex128")


def _scalar(x):
    x = complex(x)
    return L.tkb_scalar(x.real, x.imag)


def _norm_p(p):
    return (tuple(int(i) for i in p[0]), tuple(int(i) for i in p[1]))


def device_table(ctx, tdst_space, tsrc, p, levels, planar=False):
    """The device table of braid!(…, p, levels), or of transpose!(…, p) with `planar`."""
    parent_space = tsrc.parent.space if isinstance(tsrc, AdjointTensorMap) else None
    src_len = tsrc.parent.space.dim() if parent_space is not None else tsrc.space.dim()
    key = ("transpose" if planar else "braid", tdst_space, tsrc.space, p, levels, parent_space)

    def make():
        if planar:
            tr = treetransposer(tdst_space, tsrc.space, p, parent_space)
        else:
            tr = treebraider(tdst_space, tsrc.space, p, levels, parent_space)
        flat = flatten_transformer(tr, p)
        return DeviceTable(ctx, flat, src_len, tdst_space.dim())

    return ctx.tables.get_or(key, make)


def _check_device(*ts):
    for t in ts:
        if not t.data.is_cuda:
            raise RuntimeError("the B200 path needs CUDA tensors (no CPU fallback)")


def add_transform_(tdst: TensorMap, tsrc, p, table: DeviceTable, alpha=1.0, beta=0.0):
    """tdst = β·tdst + α·transform(tsrc)."""
    _check_device(tdst, tsrc)
    ctx = table.ctx
    if tdst.data.dtype != tsrc.data.dtype:
        raise TypeError("source and destination must share their scalar type")
    code = dtype_code(tdst.data)
    conj = 1 if (isinstance(tsrc, AdjointTensorMap) and tsrc.is_complex()) else 0
    if LAUNCH_LOG is not None:
        LAUNCH_LOG.append(("transform", table, tdst, tsrc, complex(alpha), complex(beta), conj))
    _sync_in(ctx, tdst, tsrc)
    L.check(ctx.lib.tkb_treetransform(ctx.handle, table.handle, code,
                                      C.c_void_p(tdst.data.data_ptr()),
                                      C.c_void_p(tsrc.data.data_ptr()),
                                      _scalar(alpha), _scalar(beta), conj), ctx.handle)
    _sync_out(ctx, tdst)
    return tdst


def _sync_in(ctx, *ts):
    """Order the library stream after the torch current stream (data producers)."""
    import torch
    cur = torch.cuda.current_stream(ctx.torch_device)
    if cur.cuda_stream != ctx.stream.cuda_stream:
        ctx.stream.wait_stream(cur)


def _sync_out(ctx, *ts):
    import torch
    cur = torch.cuda.current_stream(ctx.torch_device)
    if cur.cuda_stream != ctx.stream.cuda_stream:
        cur.wait_stream(ctx.stream)
        for t in ts:
            t.data.record_stream(ctx.stream)


def braid_(tdst: TensorMap, tsrc, p, levels, alpha=1.0, beta=0.0):
    p = _norm_p(p)
    if tsrc.space.permute(p) != tdst.space:
        raise SpaceMismatch(f"tsrc = {tsrc.space}, tdst = {tdst.space}, p = {p}")
    lv = tuple(levels)
    l1 = tuple(lv[i - 1] for i in tsrc.codomainind())
    l2 = tuple(lv[i - 1] for i in tsrc.domainind())
    ctx = get_context(tdst.data.device.index)
    table = device_table(ctx, tdst.space, tsrc, p, (l1, l2))
    return add_transform_(tdst, tsrc, p, table, alpha, beta)


def permute_(tdst: TensorMap, tsrc, p, alpha=1.0, beta=0.0):
    """tdst = β·tdst + α·permute(tsrc, p) (p = (p₁, p₂), 1-based)."""
    return braid_(tdst, tsrc, p, tuple(range(1, tsrc.numind() + 1)), alpha, beta)


def permute(t, p, copy=False):
    p = _norm_p(p)
    if not copy and isinstance(t, TensorMap) and p == (t.codomainind(), t.domainind()):
        return t
    if not copy and isinstance(t, AdjointTensorMap):
        # adjointtensorindex: i ≤ numout(t) ↦ numin(t) + i, else i - numout(t)
        adj = lambda i: t.numin() + i if i <= t.numout() else i - t.numout()
        if (tuple(map(adj, p[1])), tuple(map(adj, p[0]))) == (t.parent.codomainind(),
                                                               t.parent.domainind()):
            return t
    dst = new_tensor(t.space.permute(p), t.data.dtype, t.data.device)
    return permute_(dst, t, p, 1.0, 0.0)


def braid(t, p, levels, copy=False):
    p = _norm_p(p)
    if not copy and isinstance(t, TensorMap) and p == (t.codomainind(), t.domainind()):
        return t
    dst = new_tensor(t.space.permute(p), t.data.dtype, t.data.device)
    return braid_(dst, t, p, levels, 1.0, 0.0)


def transpose_(tdst, tsrc, p, alpha=1.0, beta=0.0):
    """tdst = β·tdst + α·transpose(tsrc, p): a cyclic (planar) permutation, whose trees move by
    folds, bends and rotations only (`src/tensors/indexmanipulations.jl:378-391`)."""
    from .fusiontrees import linearizepermutation
    p = _norm_p(p)
    lin = linearizepermutation(p[0], p[1], tsrc.numout(), tsrc.numin())
    n = len(lin)
    if n and not all(lin[(i + 1) % n] == (lin[i] % n) + 1 for i in range(n)):
        raise ValueError(f"invalid cyclic or planar permutation p = {p}")
    if tsrc.space.permute(p) != tdst.space:
        raise SpaceMismatch(f"tsrc = {tsrc.space}, tdst = {tdst.space}, p = {p}")
    ctx = get_context(tdst.data.device.index)
    table = device_table(ctx, tdst.space, tsrc, p, None, planar=True)
    return add_transform_(tdst, tsrc, p, table, alpha, beta)


def transpose(t, p=None, copy=False):
    if p is None:
        p = (tuple(reversed(t.domainind())), tuple(reversed(t.codomainind())))
    p = _norm_p(p)
    dst = new_tensor(t.space.permute(p), t.data.dtype, t.data.device)
    return transpose_(dst, t, p)


def flip(t, I, inv=False):
    """A tensor isomorphic to t with the arrows of the legs i ∈ I (1-based) flipped:
    space(t′, i) = flip(space(t, i)), every sub-block scaled by its tree pair's flip factor;
    `flip(flip(t, I), I, inv=True)` is t (`src/tensors/indexmanipulations.jl:21-29`). One
    transform launch with the identity permutation."""
    if not isinstance(t, TensorMap):
        raise TypeError("flip takes a TensorMap (materialise a lazy adjoint first)")
    I = (int(I),) if isinstance(I, int) else tuple(int(i) for i in I)
    W = t.space.flip(I)
    dst = new_tensor(W, t.data.dtype, t.data.device)
    n1, n = t.numout(), t.numind()
    p = (tuple(range(1, n1 + 1)), tuple(range(n1 + 1, n + 1)))
    ctx = get_context(t.data.device.index)

    def make():
        flat = flatten_transformer(treeflipper(W, t.space, I, inv), p)
        return DeviceTable(ctx, flat, t.space.dim(), W.dim())

    table = ctx.tables.get_or(("flip", W, t.space, I, bool(inv)), make)
    return add_transform_(dst, t, p, table, 1.0, 0.0)


def repartition(t, N1, copy=False):
    """Move legs between codomain and domain keeping the cyclic order
    (`permutedims(a, (1..N₁, reverse(N₁+1..N)))` in dense form)."""
    N = t.numind()
    lin = list(range(1, t.numout() + 1)) + list(reversed(range(t.numout() + 1, N + 1)))
    p1 = tuple(lin[:N1])
    p2 = tuple(reversed(lin[N1:]))
    return transpose(t, (p1, p2), copy)
