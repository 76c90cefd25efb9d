"""Block and sub-block layout of a TensorMap's flat data vector.

Restates `src/spaces/structure.jl`:
- `sectorstructure` (`:41-72`): coupled sectors in `_blocksectors` order; for each coupled
  sector c, the domain trees in iteration order (outer) × codomain trees (inner);
- `degeneracystructure` (`:114-188`): block c is a contiguous column-major
  (d₁(c), d₂(c)) matrix; the sub-block of tree pair (f₁, f₂) is the window at row offset
  Σ(preceding codomain trees) and column offset Σ(preceding domain trees), reshaped to the
  uncoupled degeneracy dims (d₁s..., d₂s...) with strides (1, d₁s₁, d₁s₁d₁s₂, ...,
  B, B·d₂s₁, ...) where B = d₁(c) is the block's leading dimension.
- `fusionblocks` (`src/spaces/homspace.jl:178-188`): trees grouped by uncoupled sectors,
  domain sectors outer, codomain sectors inner.

Strides of size-1 dimensions are the natural cumulative products (a size-1 dimension
never changes an address).
"""
from __future__ import annotations

from functools import lru_cache

from .fusiontrees import FusionTreeBlock

__all__ = ["SectorStructure", "DegeneracyStructure", "sectorstructure", "degeneracystructure",
           "fusionblocks", "subblockstructure", "blockstructure"]


class SectorStructure:
    __slots__ = ("blocksectors", "fusiontrees", "index")

    def __init__(self, blocksectors, trees):
        self.blocksectors = blocksectors
        self.fusiontrees = trees
        self.index = {t: i for i, t in enumerate(trees)}


class DegeneracyStructure:
    """totaldim; per block ((d₁, d₂), (start, stop)) 0-based half-open; per tree pair
    (sizes, strides, offset) with a 0-based offset."""
    __slots__ = ("totaldim", "blockstructure", "subblockstructure")

    def __init__(self, totaldim, blockstructure, subblockstructure):
        self.totaldim = totaldim
        self.blockstructure = blockstructure
        self.subblockstructure = subblockstructure


@lru_cache(maxsize=10000)
def sectorstructure(W) -> SectorStructure:
    cod, dom = W.codomain, W.domain
    bs = []
    trees = []
    for c in W._blocksectors():
        bs.append(c)
        ftrees1 = cod.fusiontrees(c)
        for f2 in dom.fusiontrees(c):
            for f1 in ftrees1:
                trees.append((f1, f2))
    return SectorStructure(bs, trees)


def _prod(xs):
    r = 1
    for x in xs:
        r *= x
    return r


@lru_cache(maxsize=10000)
def degeneracystructure(W) -> DegeneracyStructure:
    cod, dom = W.codomain, W.domain
    ss = sectorstructure(W)
    treelist = ss.fusiontrees
    L = len(treelist)
    subs = []
    blocks = []
    blockoffset = 0
    ti = 0
    while ti < L:
        f1, f2 = treelist[ti]
        c = f1.coupled
        split = []
        off1 = 0
        for i in range(ti, L):
            g1, g2 = treelist[i]
            if g2 != f2:
                break
            d1s = cod.dims(g1.uncoupled)
            off1 += _prod(d1s)
            split.append(d1s)
        bd1 = off1
        n1 = len(split)
        off2 = 0
        n2 = 0
        for i in range(ti, L, n1):
            g1, g2 = treelist[i]
            if g2.coupled != c:
                break
            n2 += 1
            d2s = dom.dims(g2.uncoupled)
            d2 = _prod(d2s)
            o1 = 0
            for d1s in split:
                d1 = _prod(d1s)
                tot = blockoffset + off2 * bd1 + o1
                sz = tuple(d1s) + tuple(d2s)
                assert all(x > 0 for x in sz)
                st = []
                s = 1
                for x in d1s:
                    st.append(s)
                    s *= x
                s = bd1
                for x in d2s:
                    st.append(s)
                    s *= x
                subs.append((sz, tuple(st), tot))
                o1 += d1
            off2 += d2
        bd2 = off2
        blocks.append(((bd1, bd2), (blockoffset, blockoffset + bd1 * bd2)))
        blockoffset += bd1 * bd2
        ti += n1 * n2
        # sanity: the loop above consumed exactly the trees of block c
    assert len(subs) == L
    return DegeneracyStructure(blockoffset, blocks, subs)


def subblockstructure(W) -> dict:
    ss = sectorstructure(W)
    ds = degeneracystructure(W)
    return dict(zip(ss.fusiontrees, ds.subblockstructure))


def blockstructure(W) -> dict:
    ss = sectorstructure(W)
    ds = degeneracystructure(W)
    return dict(zip(ss.blocksectors, ds.blockstructure))


@lru_cache(maxsize=10000)
def fusionblocks(W):
    u = W.unit()
    isdual = (tuple(v.isdual() for v in W.codomain), tuple(v.isdual() for v in W.domain))
    out = []
    for dom_unc in W.domain.sectors():
        for cod_unc in W.codomain.sectors():
            blk = FusionTreeBlock((cod_unc, dom_unc), isdual, u)
            if len(blk):
                out.append(blk)
    return tuple(out)
