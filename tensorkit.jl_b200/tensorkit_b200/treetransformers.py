"""Tree transformers: the per-structure recipe of a permute/braid, flattened into tables.

Restates `src/tensors/treetransformers.jl`:
- `AbelianTreeTransformer` (`:10-42`): one `(coeff, dst (sz,str,off), src (sz,str,off))`
  per source tree pair, in the order of `fusiontrees(Vsrc)`, unsorted;
- `GenericTreeTransformer` (`:44-120`): one `(U, (sz_dst, [(str,off)...]),
  (sz_src, [(str,off)...]))` per source fusion block, then sorted by the weight
  `length(U) * prod(sz_dst)` in decreasing order (stable sort, `:186-205`);
- `treebraider` (`:156-167`) is cached per `(Vdst, Vsrc, p, levels)`.

`FlatTable` is the device-table form handed to the C-ABI (`tkb_table_create`): every
transformer becomes a list of groups (a unique-fusion entry is a group with one tree on
each side and U = [[coeff]]), each with a source size tuple, per-tree strides/offsets
and a dense row-major U (rows = destination trees, columns = source trees).
"""
from __future__ import annotations

import numpy as np

from .fusiontrees import braid as _braid_trees
from .fusiontrees import FusionTreeBlock
from .fusiontrees import flip as _flip_pair
from .fusiontrees import fstranspose as _fstranspose
from .structure import fusionblocks, sectorstructure, subblockstructure

__all__ = ["AbelianTreeTransformer", "GenericTreeTransformer", "treebraider", "treetransposer", "treeflipper",
           "FlatTable",
           "flatten_transformer"]


class AbelianTreeTransformer:
    __slots__ = ("data",)

    def __init__(self, data):
        self.data = data


class GenericTreeTransformer:
    __slots__ = ("data",)

    def __init__(self, data):
        self.data = data


def _is_unique(W):
    u = W.unit()
    return u.fusionstyle == "unique"


def _adjoint_subblocks(Wparent):
    """Sub-block structure of adjoint(t) expressed in the parent's data vector: the tree
    pair (f₁, f₂) of the adjoint is the parent's (f₂, f₁) with its dims reordered
    (domain legs first), read with complex conjugation (`src/tensors/adjoint.jl:47-51`)."""
    n1 = Wparent.numout()
    sbs = subblockstructure(Wparent)
    out = {}
    for (f1, f2), (sz, st, off) in sbs.items():
        perm = tuple(range(n1, len(sz))) + tuple(range(n1))
        out[(f2, f1)] = (tuple(sz[k] for k in perm), tuple(st[k] for k in perm), off)
    return out


def build_transformer(Vdst, Vsrc, p, levels, src_adjoint_of=None, planar=False):
    """Build the transformer for braid!(tdst, tsrc, p, levels), or with `planar` for
    transpose!(tdst, tsrc, p) (trees moved by fstranspose, levels unused); `src_adjoint_of` is
    the parent HomSpace when the source is a lazy adjoint (then Vsrc == adjoint(parent))."""
    if planar:
        def move(x):
            return _fstranspose(x, p[0], p[1])
    else:
        def move(x):
            return _braid_trees(x, p, levels)
    if Vsrc.permute(p) != Vdst:
        from .spaces import SpaceMismatch
        raise SpaceMismatch("Incompatible spaces for permuting.")
    if src_adjoint_of is None:
        fts_src = subblockstructure(Vsrc)
    else:
        fts_src = _adjoint_subblocks(src_adjoint_of)
    fts_dst = subblockstructure(Vdst)
    if _is_unique(Vsrc):
        data = []
        for pair in sectorstructure(Vsrc).fusiontrees:
            pdst, coeff = move(pair)
            data.append((coeff, fts_dst[pdst], fts_src[pair]))
        return AbelianTreeTransformer(data)
    data = []
    for blk in fusionblocks(Vsrc):
        dst, U = move(blk)
        sz_src = fts_src[blk.trees[0]][0]
        sz_dst = fts_dst[dst.trees[0]][0]
        ss = [(fts_src[t][1], fts_src[t][2]) for t in blk.trees]
        sd = [(fts_dst[t][1], fts_dst[t][2]) for t in dst.trees]
        data.append((U, (sz_dst, sd), (sz_src, ss)))
    # stable sort by decreasing weight length(U) * prod(sz_dst); the lazy-adjoint source
    # goes through the closure transformer of the reference, which keeps block order
    if src_adjoint_of is None:
        data.sort(key=lambda e: -(e[0].size * int(np.prod(e[1][0]))))
    return GenericTreeTransformer(data)


_TRANSFORMER_CACHE: dict = {}


def treebraider(Vdst, Vsrc, p, levels, src_adjoint_of=None):
    key = (Vdst, Vsrc, tuple(map(tuple, p)), tuple(map(tuple, levels)), src_adjoint_of)
    t = _TRANSFORMER_CACHE.get(key)
    if t is None:
        t = build_transformer(Vdst, Vsrc, p, levels, src_adjoint_of)
        if len(_TRANSFORMER_CACHE) > 10000:
            _TRANSFORMER_CACHE.clear()
        _TRANSFORMER_CACHE[key] = t
    return t


def treetransposer(Vdst, Vsrc, p, src_adjoint_of=None):
    """Transformer of transpose!(tdst, tsrc, p): the trees move by fstranspose (folds, bends
    and cyclic rotations, no braiding), cached per `(Vdst, Vsrc, p)`
    (`src/tensors/treetransformers.jl:175-180`)."""
    key = ("transpose", Vdst, Vsrc, tuple(map(tuple, p)), src_adjoint_of)
    t = _TRANSFORMER_CACHE.get(key)
    if t is None:
        t = build_transformer(Vdst, Vsrc, p, ((), ()), src_adjoint_of, planar=True)
        if len(_TRANSFORMER_CACHE) > 10000:
            _TRANSFORMER_CACHE.clear()
        _TRANSFORMER_CACHE[key] = t
    return t


def treeflipper(Vdst, Vsrc, I, inv=False):
    """Transformer of flip(t, I): every tree pair goes to the same pair with the duality flags
    of the legs I toggled, scaled by the flip factor, under the identity permutation
    (`src/tensors/indexmanipulations.jl:21-29`), cached per `(Vdst, Vsrc, I, inv)`."""
    I = tuple(int(i) for i in I)
    key = ("flip", Vdst, Vsrc, I, bool(inv))
    t = _TRANSFORMER_CACHE.get(key)
    if t is not None:
        return t
    fts_src = subblockstructure(Vsrc)
    fts_dst = subblockstructure(Vdst)
    if _is_unique(Vsrc):
        data = []
        for pair in sectorstructure(Vsrc).fusiontrees:
            pdst, coeff = _flip_pair(pair, I, inv)
            data.append((coeff, fts_dst[pdst], fts_src[pair]))
        t = AbelianTreeTransformer(data)
    else:
        n1 = Vsrc.numout()
        data = []
        for blk in fusionblocks(Vsrc):
            d1 = tuple((not d) if k + 1 in I else d for k, d in enumerate(blk.isdual[0]))
            d2 = tuple((not d) if n1 + k + 1 in I else d for k, d in enumerate(blk.isdual[1]))
            dst = FusionTreeBlock(blk.uncoupled, (d1, d2), blk.trees[0][0].coupled.unit())
            U = np.zeros((len(dst), len(blk)))
            for col, pair in enumerate(blk.trees):
                pdst, coeff = _flip_pair(pair, I, inv)
                U[dst.index[pdst], col] = coeff
            sz_src = fts_src[blk.trees[0]][0]
            sz_dst = fts_dst[dst.trees[0]][0]
            ss = [(fts_src[x][1], fts_src[x][2]) for x in blk.trees]
            sd = [(fts_dst[x][1], fts_dst[x][2]) for x in dst.trees]
            data.append((U, (sz_dst, sd), (sz_src, ss)))
        data.sort(key=lambda e: -(e[0].size * int(np.prod(e[1][0]))))
        t = GenericTreeTransformer(data)
    if len(_TRANSFORMER_CACHE) > 10000:
        _TRANSFORMER_CACHE.clear()
    _TRANSFORMER_CACHE[key] = t
    return t


class FlatTable:
    """Flattened transformer (all arrays int64 / float64, 0-based offsets).

    nind: N; perm[k] (0-based) is the source dim that becomes destination dim k.
    group_src_ptr / group_dst_ptr: prefix sums of trees per group on each side;
    coeff_ptr: prefix sums of rows*cols; sizes: (ngroups, N) source sizes;
    src_strides/dst_strides: (ntrees, N); src_offsets/dst_offsets: (ntrees,)."""

    def __init__(self, nind, perm, group_src_ptr, group_dst_ptr, coeff_ptr, coeffs, sizes,
                 src_strides, src_offsets, dst_strides, dst_offsets):
        self.nind = int(nind)
        self.perm = np.asarray(perm, dtype=np.int64)
        self.group_src_ptr = np.ascontiguousarray(group_src_ptr, dtype=np.int64)
        self.group_dst_ptr = np.ascontiguousarray(group_dst_ptr, dtype=np.int64)
        self.coeff_ptr = np.ascontiguousarray(coeff_ptr, dtype=np.int64)
        self.coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int64).reshape(-1, self.nind)
        self.src_strides = np.ascontiguousarray(src_strides, dtype=np.int64).reshape(-1, self.nind)
        self.src_offsets = np.ascontiguousarray(src_offsets, dtype=np.int64)
        self.dst_strides = np.ascontiguousarray(dst_strides, dtype=np.int64).reshape(-1, self.nind)
        self.dst_offsets = np.ascontiguousarray(dst_offsets, dtype=np.int64)

    @property
    def ngroups(self):
        return len(self.group_src_ptr) - 1

    def nbytes_moved(self, elsize, beta_nonzero=False):
        """Algorithmic bytes: read every source element once, write every destination
        element once (and read it when β ≠ 0)."""
        n_src = 0
        n_dst = 0
        for g in range(self.ngroups):
            vol = int(np.prod(self.sizes[g]))
            n_src += vol * int(self.group_src_ptr[g + 1] - self.group_src_ptr[g])
            n_dst += vol * int(self.group_dst_ptr[g + 1] - self.group_dst_ptr[g])
        return elsize * (n_src + n_dst * (2 if beta_nonzero else 1))


def flatten_transformer(tr, p) -> FlatTable:
    p1, p2 = p
    flat = tuple(p1) + tuple(p2)
    N = len(flat)
    perm = [x - 1 for x in flat]
    gs, gd, cp, coeffs, sizes, sst, sof, dst_, dof = [0], [0], [0], [], [], [], [], [], []
    if isinstance(tr, AbelianTreeTransformer):
        for coeff, (szd, std, offd), (szs, sts, offs) in tr.data:
            gs.append(gs[-1] + 1)
            gd.append(gd[-1] + 1)
            cp.append(cp[-1] + 1)
            coeffs.append(float(coeff))
            sizes.append(szs)
            sst.append(sts)
            sof.append(offs)
            dst_.append(std)
            dof.append(offd)
    else:
        for U, (szd, sd), (szs, ss) in tr.data:
            rows, cols = U.shape
            gs.append(gs[-1] + cols)
            gd.append(gd[-1] + rows)
            cp.append(cp[-1] + rows * cols)
            coeffs.extend(np.asarray(U, dtype=np.float64).reshape(-1).tolist())
            sizes.append(szs)
            for st, off in ss:
                sst.append(st)
                sof.append(off)
            for st, off in sd:
                dst_.append(st)
                dof.append(off)
    if N == 0:
        sizes = np.zeros((len(gs) - 1, 0))
    return FlatTable(N, perm, gs, gd, cp, coeffs, sizes, sst, sof, dst_, dof)
