"""Fusion trees, fusion-tree blocks and the recoupling moves of the permute/braid path.

Follows, for multiplicity-free sectors (U1, SU2, U1⊠SU2):
- `FusionTree` / `FusionTreeBlock` (`src/fusiontrees/fusiontrees.jl:22-157`);
- the deterministic iteration order (`src/fusiontrees/iterator.jl:98-226`);
- `bendright` / `bendleft` and `repartition` (`src/fusiontrees/duality_manipulations.jl:33-194`,
  `:460-505`);
- `multi_Fmove` / `multi_Fmove_inv` (`src/fusiontrees/basic_manipulations.jl:191-440`), `foldright` /
  `foldleft`, `cycleclockwise` / `cycleanticlockwise` and `fstranspose`
  (`src/fusiontrees/duality_manipulations.jl:220-426`, `:534-562`);
- `artin_braid` for single trees (`src/fusiontrees/braiding_manipulations.jl:18-79`) and for
  blocks (`:81-198`), `braid` of a unique-fusion tree (`:215-251`), `fsbraid` (`:304-340`);
- `linearizepermutation` and `permutation2swaps` (`src/auxiliary/auxiliary.jl:1-28`).

Unique fusion (U1) uses single tree pairs and scalar coefficients; multiplicity-free
non-abelian fusion (SU2, U1⊠SU2) uses FusionTreeBlocks and recoupling matrices U with
`U = U_tmp @ U` accumulated in the reference's order.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np

from .sectors import (Asymbol, Bsymbol, Fsymbol, Nsymbol, Rsymbol, frobenius_schur_phase,
                      invsqrtdim, otimes_many, sqrtdim)

__all__ = ["FusionTree", "FusionTreeBlock", "fusiontrees", "bendright", "bendleft", "split",
           "repartition", "artin_braid", "braid", "permute", "linearizepermutation",
           "permutation2swaps", "multi_Fmove", "multi_Fmove_inv", "foldright", "foldleft",
           "cycleclockwise", "cycleanticlockwise", "fstranspose", "flip"]


class FusionTree:
    """Splitting tree: coupled → uncoupled[0] ⊗ ... ⊗ uncoupled[N-1] (multiplicity-free)."""
    __slots__ = ("uncoupled", "coupled", "isdual", "innerlines", "_h")

    def __init__(self, uncoupled, coupled, isdual, innerlines=()):
        self.uncoupled = tuple(uncoupled)
        self.coupled = coupled
        self.isdual = tuple(bool(x) for x in isdual)
        self.innerlines = tuple(innerlines)
        self._h = hash((self.uncoupled, self.coupled, self.isdual, self.innerlines))

    def key(self):
        return (self.uncoupled, self.coupled, self.isdual, self.innerlines)

    def __eq__(self, o):
        return isinstance(o, FusionTree) and self.key() == o.key()

    def __hash__(self):
        return self._h

    def __len__(self):
        return len(self.uncoupled)

    def __repr__(self):
        return (f"FusionTree({self.uncoupled}, {self.coupled}, {self.isdual}, "
                f"{self.innerlines})")


def _abelian_inner(uncoupled):
    """Inner lines of a unique-fusion tree: successive fusion products from the left."""
    n = len(uncoupled)
    if n <= 2:
        return ()
    inner = []
    acc = uncoupled[0].otimes(uncoupled[1])[0]
    inner.append(acc)
    for k in range(2, n - 1):
        acc = acc.otimes(uncoupled[k])[0]
        inner.append(acc)
    return tuple(inner)


def _iter_trees(lists, c):
    """Yield (uncoupled, innerlines) in the reference iteration order: the last leg's sector
    varies slowest, then the inner line, then recursively the front legs."""
    n = len(lists)
    if n == 0:
        if c.isunit():
            yield (), ()
        return
    if n == 1:
        if c in lists[0]:
            yield (c,), ()
        return
    if n == 2:
        for b in lists[1]:
            for a in lists[0]:
                if Nsymbol(a, b, c):
                    yield (a, b), ()
        return
    for b in lists[-1]:
        for a in c.otimes(b.dual()):
            for rest_out, rest_lines in _iter_trees(lists[:-1], a):
                yield rest_out + (b,), rest_lines + (a,)


def fusiontrees(uncoupled_lists, coupled, isdual):
    """All fusion trees with uncoupled sectors drawn from `uncoupled_lists[i]`."""
    isdual = tuple(bool(x) for x in isdual)
    return [FusionTree(out, coupled, isdual, lines)
            for out, lines in _iter_trees(tuple(tuple(l) for l in uncoupled_lists), coupled)]


@lru_cache(maxsize=100000)
def _trees_single(uncoupled, coupled, isdual):
    return tuple(fusiontrees(tuple((s,) for s in uncoupled), coupled, isdual))


class FusionTreeBlock:
    """All tree pairs (f₁, f₂) sharing the same uncoupled sectors and duality flags."""
    __slots__ = ("trees", "uncoupled", "isdual", "index", "_h")

    def __init__(self, uncoupled, isdual, unit, trees=None):
        u1, u2 = tuple(uncoupled[0]), tuple(uncoupled[1])
        d1, d2 = tuple(bool(x) for x in isdual[0]), tuple(bool(x) for x in isdual[1])
        self.uncoupled = (u1, u2)
        self.isdual = (d1, d2)
        if trees is None:
            trees = []
            n1, n2 = len(u1), len(u2)
            if n1 == 0 and n2 == 0:
                f = FusionTree((), unit, (), ())
                trees.append((f, f))
            else:
                if n1 == 0:
                    cs = [c for c in otimes_many(u2, unit) if c.isunit()]
                elif n2 == 0:
                    cs = [c for c in otimes_many(u1, unit) if c.isunit()]
                else:
                    s2 = set(otimes_many(u2, unit))
                    cs = [c for c in otimes_many(u1, unit) if c in s2]
                cs.sort(key=lambda c: c.sortkey())
                for c in cs:
                    for f2 in _trees_single(u2, c, d2):
                        for f1 in _trees_single(u1, c, d1):
                            trees.append((f1, f2))
        self.trees = trees
        self.index = {t: i for i, t in enumerate(trees)}
        self._h = hash((self.uncoupled, self.isdual))

    def __len__(self):
        return len(self.trees)

    def __eq__(self, o):
        return isinstance(o, FusionTreeBlock) and self.trees == o.trees

    def __hash__(self):
        return self._h

    def numout(self):
        return len(self.uncoupled[0])

    def numin(self):
        return len(self.uncoupled[1])


def _unit_of(src):
    f1, f2 = src.trees[0] if isinstance(src, FusionTreeBlock) else src
    return f1.coupled.unit()


# ------------------------------------------------------------------------------------
# bending (B-moves)
# ------------------------------------------------------------------------------------
def _bendright_treepair(f1, f2):
    n1, n2 = len(f1), len(f2)
    c = f1.coupled
    if n1 == 1:
        a = c.unit()
    elif n1 == 2:
        a = f1.uncoupled[0]
    else:
        a = f1.innerlines[-1]
    b = f1.uncoupled[n1 - 1]
    f1n = FusionTree(f1.uncoupled[:-1], a, f1.isdual[:-1], f1.innerlines[:-1] if n1 > 2 else ())
    f2n = FusionTree(f2.uncoupled + (b.dual(),), a, f2.isdual + (not f1.isdual[n1 - 1],),
                     (f2.innerlines + (c,)) if n2 > 1 else ())
    return (a, b, c), (f1n, f2n)


def _bend_coeff(a, b, c, isdual_b):
    coeff0 = sqrtdim(c) * invsqrtdim(a)
    if isdual_b:
        coeff0 = coeff0 * frobenius_schur_phase(b.dual())
    return coeff0 * Bsymbol(a, b, c)


def bendright(src):
    """Bend the last splitting leg to the fusion side (`duality_manipulations.jl:52-118`)."""
    if not isinstance(src, FusionTreeBlock):
        f1, f2 = src
        (a, b, c), pair = _bendright_treepair(f1, f2)
        return pair, _bend_coeff(a, b, c, f1.isdual[-1])
    u1, u2 = src.uncoupled
    d1, d2 = src.isdual
    unit = _unit_of(src)
    dst = FusionTreeBlock((u1[:-1], u2 + (u1[-1].dual(),)), (d1[:-1], d2 + (not d1[-1],)), unit)
    U = np.zeros((len(dst), len(src)))
    for col, (f1, f2) in enumerate(src.trees):
        (a, b, c), pair = _bendright_treepair(f1, f2)
        U[dst.index[pair], col] = _bend_coeff(a, b, c, f1.isdual[-1])
    return dst, U


def bendleft(src):
    """Bend the last fusion leg to the splitting side (`duality_manipulations.jl:120-194`)."""
    if not isinstance(src, FusionTreeBlock):
        f1, f2 = src
        (a, b, c), (f2n, f1n) = _bendright_treepair(f2, f1)
        return (f1n, f2n), _bend_coeff(a, b, c, f2.isdual[-1])  # real: conj is identity
    u1, u2 = src.uncoupled
    d1, d2 = src.isdual
    unit = _unit_of(src)
    dst = FusionTreeBlock((u1 + (u2[-1].dual(),), u2[:-1]), (d1 + (not d2[-1],), d2[:-1]), unit)
    U = np.zeros((len(dst), len(src)))
    for col, (f1, f2) in enumerate(src.trees):
        (a, b, c), (f2n, f1n) = _bendright_treepair(f2, f1)
        U[dst.index[(f1n, f2n)], col] = _bend_coeff(a, b, c, f2.isdual[-1])
    return dst, U


def split(f, M):
    """(f₁, f₂) with f₁ the first M uncoupled legs of f fused to the line c₁ between them and
    the rest, and f₂ = (c₁, remaining legs) → f.coupled
    (`src/fusiontrees/basic_manipulations.jl:30-52`)."""
    N = len(f.uncoupled)
    if not 0 <= M <= N or N == 0:
        raise ValueError("split: M must lie in 0..N (N ≥ 1)")
    ext = (f.uncoupled[0],) + tuple(f.innerlines) + (f.coupled,)
    c1 = f.coupled.unit() if M == 0 else ext[M - 1]
    f1 = FusionTree(f.uncoupled[:M], c1, f.isdual[:M], f.innerlines[:max(0, M - 2)])
    f2 = FusionTree((c1,) + f.uncoupled[M:], f.coupled, (False,) + f.isdual[M:],
                    ext[M:M + max(0, N - M - 1)])
    return f1, f2


def repartition(src, N):
    """Bend legs until the splitting side has N legs (`duality_manipulations.jl:460-505`)."""
    if isinstance(src, FusionTreeBlock):
        n1 = src.numout()
        n = n1 - N
        if n == 0:
            return src, np.eye(len(src))
        f = bendright if n > 0 else bendleft
        dst, U = f(src)
        for _ in range(abs(n) - 1):
            dst, Ut = f(dst)
            U = Ut @ U
        return dst, U
    f1, f2 = src
    n = len(f1) - N
    if n == 0:
        return src, 1.0
    f = bendright if n > 0 else bendleft
    dst, coeff = f(src)
    for _ in range(abs(n) - 1):
        dst, ct = f(dst)
        coeff = ct * coeff
    return dst, coeff


# ------------------------------------------------------------------------------------
# folding, cyclic permutations and transpose
# ------------------------------------------------------------------------------------
def _extend(T, u, isdual_u, coupled):
    """T with one more leg u on the right, the old coupled line fused with u to `coupled`."""
    inner = (T.innerlines + (T.coupled,)) if len(T.uncoupled) >= 2 else ()
    return FusionTree(T.uncoupled + (u,), coupled, T.isdual + (isdual_u,), inner)


def multi_Fmove(f):
    """Recouple the splitting tree f so that its first leg a meets the coupled line last:
    a list of (f′, coeff), f′ the trees of the other legs (coupled b, a ⊗ b → f.coupled on
    top). One F-move per further leg, from the left: after legs 0..k-1 the state is
    (a ⊗ T → e) with e the coupling of those legs in f; adding leg k (fused to d in f) gives
    Σ_b′ [F^{a b u}_d]^e_{b′} a ⊗ (T ⊗ u → b′) → d (`basic_manipulations.jl:191-322`)."""
    N = len(f.uncoupled)
    if N == 0:
        raise ValueError("multi_Fmove requires at least one uncoupled sector")
    c = f.coupled
    if N == 1:
        return [(FusionTree((), c.unit(), (), ()), 1.0)]
    a = f.uncoupled[0]
    ext = tuple(f.innerlines) + (c,)  # ext[k-2]: the line the first k legs fuse to in f
    u1 = f.uncoupled[1]
    states = [(FusionTree((u1,), u1, (f.isdual[1],), ()), 1.0)]
    for k in range(2, N):
        e, d, u = ext[k - 2], ext[k - 1], f.uncoupled[k]
        nxt = []
        for T, cf in states:
            b = T.coupled
            for b2 in b.otimes(u):
                if not Nsymbol(a, b2, d):
                    continue
                F = Fsymbol(a, b, u, d, e, b2)
                if F != 0.0:
                    nxt.append((_extend(T, u, f.isdual[k], b2), cf * F))
        states = nxt
    return states


def multi_Fmove_inv(a, c, f, isduala=False):
    """Fuse a new first leg a (duality flag isduala) with the splitting tree f (coupled b) to
    c, expanded in standard trees of (a, f's legs) → c: a list of (tree, coeff). The last leg
    v of f is peeled off with the inverse F-move a ⊗ (b′ ⊗ v → b) → c = Σ_e [F^{a b′ v}_c]^e_b
    (a ⊗ b′ → e) ⊗ v → c (F is orthogonal for these sectors), then the rest recursively
    (`basic_manipulations.jl:353-440`)."""
    b = f.coupled
    if not Nsymbol(a, b, c):
        raise ValueError(f"cannot fuse sectors {a} and {b} to {c}")
    N = len(f.uncoupled)
    if N == 0:
        return [(FusionTree((a,), c, (isduala,), ()), 1.0)]
    if N == 1:
        return [(FusionTree((a, f.uncoupled[0]), c, (isduala, f.isdual[0]), ()), 1.0)]
    v = f.uncoupled[-1]
    bp = f.innerlines[-1] if N > 2 else f.uncoupled[0]
    fp = FusionTree(f.uncoupled[:-1], bp, f.isdual[:-1], f.innerlines[:-1] if N > 2 else ())
    out = []
    for e in a.otimes(bp):
        if not Nsymbol(e, v, c):
            continue
        F = Fsymbol(a, bp, v, c, e, b)
        if F == 0.0:
            continue
        for S, cf in multi_Fmove_inv(a, e, fp, isduala):
            out.append((_extend(S, v, f.isdual[-1], c), cf * F))
    return out


def _fold_terms(fa, fo, right):
    """Terms of folding the first leg a of the tree fa (splitting side for foldright, fusion
    side for foldleft) onto the other tree fo: ((f₁′, f₂′), coeff) pairs with coefficient
    √d_c/√d_b · A^{ab}_c · (multi_Fmove coefficient) · (multi_Fmove_inv coefficient), times
    χ_a when a is a dual leg (`duality_manipulations.jl:220-236`, `:319-325`)."""
    a, isduala, c = fa.uncoupled[0], fa.isdual[0], fa.coupled
    ka = frobenius_schur_phase(a)
    acc = {}
    for fap, ca in multi_Fmove(fa):
        b = fap.coupled
        A = Asymbol(a, b, c)
        if A == 0.0:
            continue
        c0 = sqrtdim(c) * invsqrtdim(b) * A * ca
        for fop, co in multi_Fmove_inv(a.dual(), b, fo, not isduala):
            coeff = c0 * co * (ka if isduala else 1.0)
            key = (fap, fop) if right else (fop, fap)
            acc[key] = acc.get(key, 0.0) + coeff
    return acc


def _fold(src, right):
    if not isinstance(src, FusionTreeBlock):
        f1, f2 = src
        acc = _fold_terms(f1, f2, True) if right else _fold_terms(f2, f1, False)
        if len(acc) != 1:
            raise ValueError("folding a tree pair needs unique fusion; use a FusionTreeBlock")
        (pair, coeff), = acc.items()
        return pair, coeff
    u1, u2 = src.uncoupled
    d1, d2 = src.isdual
    unit = (u1 + u2)[0].unit()
    if right:
        if not u1:
            raise ValueError("foldright needs a splitting leg")
        dst = FusionTreeBlock((u1[1:], (u1[0].dual(),) + u2), (d1[1:], (not d1[0],) + d2), unit)
    else:
        if not u2:
            raise ValueError("foldleft needs a fusion leg")
        dst = FusionTreeBlock(((u2[0].dual(),) + u1, u2[1:]), ((not d2[0],) + d1, d2[1:]), unit)
    U = np.zeros((len(dst), len(src)))
    for col, (f1, f2) in enumerate(src.trees):
        acc = _fold_terms(f1, f2, True) if right else _fold_terms(f2, f1, False)
        for pair, coeff in acc.items():
            U[dst.index[pair], col] += coeff
    return dst, U


def foldright(src):
    """Fold the first splitting leg a to the fusion side (it becomes the first fusion leg,
    dualised): (dst, U) for a block, (pair, coeff) for a unique-fusion tree pair
    (`duality_manipulations.jl:220-290`)."""
    return _fold(src, True)


def foldleft(src):
    """Fold the first fusion leg to the splitting side (`duality_manipulations.jl:316-376`)."""
    return _fold(src, False)


def _compose(first, second):
    (tmp, U1) = first
    dst, U2 = second(tmp)
    return dst, (U2 @ U1 if isinstance(U1, np.ndarray) else U2 * U1)


def _numout(src):
    return src.numout() if isinstance(src, FusionTreeBlock) else len(src[0])


def _numin(src):
    return src.numin() if isinstance(src, FusionTreeBlock) else len(src[1])


def cycleclockwise(src):
    """Fold the first splitting leg to the fusion side and bend the last fusion leg back: the
    legs rotate one step clockwise at fixed (N₁, N₂) (`duality_manipulations.jl:402-411`)."""
    if _numout(src) > 0:
        return _compose(foldright(src), bendleft)
    return _compose(bendleft(src), foldright)


def cycleanticlockwise(src):
    """Bend the last splitting leg to the fusion side and fold the first fusion leg back
    (`duality_manipulations.jl:433-442`)."""
    if _numin(src) > 0:
        return _compose(foldleft(src), bendright)
    return _compose(bendright(src), foldleft)


def fstranspose(src, p1, p2):
    """Planar (cyclic) permutation (p₁, p₂), 1-based, as a repartition followed by cyclic
    rotations, the shorter way round (`duality_manipulations.jl:534-562`)."""
    p1, p2 = tuple(p1), tuple(p2)
    N1 = len(p1)
    N = N1 + len(p2)
    p = linearizepermutation(p1, p2, _numout(src), _numin(src))
    dst, U = repartition(src, N1)
    if len(p) == 0:
        return dst, U
    i1 = p.index(1) + 1
    if i1 == 1:
        return dst, U
    Nhalf = N >> 1
    while 1 < i1 <= Nhalf:
        dst, U = _compose((dst, U), cycleanticlockwise)
        i1 -= 1
    while Nhalf < i1:
        dst, U = _compose((dst, U), cycleclockwise)
        i1 = (i1 % N) + 1
    return dst, U


def _flip_tree(f, i, factor_if):
    isd = list(f.isdual)
    fac = frobenius_schur_phase(f.uncoupled[i]) if factor_if(isd[i]) else 1.0
    isd[i] = not isd[i]
    return FusionTree(f.uncoupled, f.coupled, isd, f.innerlines), fac


def flip(pair, I, inv=False):
    """Flip the duality flags of the legs I (1-based, splitting legs first) of a tree pair:
    ((f₁′, f₂′), factor). For bosonic sectors (θ = 1) each flipped leg a contributes χ_a when
    it was dual (χ_a when it was not, with `inv`), else 1; the labels stay
    (`src/fusiontrees/braiding_manipulations.jl:388-436`)."""
    f1, f2 = pair
    n1 = len(f1.uncoupled)
    factor = 1.0
    for i in I:
        if not 1 <= i <= n1 + len(f2.uncoupled):
            raise IndexError(f"flip: leg {i} out of range")
        if i <= n1:
            f1, fac = _flip_tree(f1, i - 1, (lambda d: not d) if inv else (lambda d: d))
        else:
            f2, fac = _flip_tree(f2, i - n1 - 1, (lambda d: not d) if inv else (lambda d: d))
        factor *= fac
    return (f1, f2), factor


# ------------------------------------------------------------------------------------
# braiding
# ------------------------------------------------------------------------------------
def linearizepermutation(p1, p2, n1, n2):
    """1-based linearisation of (p₁, p₂) onto a single splitting tree (`auxiliary.jl:1-11`)."""
    q1 = tuple((n2 + 2 * n1 + 1 - x) if x > n1 else x for x in p1)
    q2 = tuple((n2 + 2 * n1 + 1 - x) if x > n1 else x for x in reversed(p2))
    return q1 + q2


def permutation2swaps(perm):
    """Bubble decomposition of a 1-based permutation into adjacent swaps (`auxiliary.jl:13-28`)."""
    p = list(perm)
    N = len(p)
    swaps = []
    for k in range(1, N):
        swaps.extend(range(p[k - 1] - 1, k - 1, -1))
        for l in range(k + 1, N + 1):
            if p[l - 1] < p[k - 1]:
                p[l - 1] += 1
        p[k - 1] = k
    return swaps


def _artin_braid_block(src, i, inv):
    """Elementary braid of legs i, i+1 (1-based) on a block with N₂ = 0."""
    u = src.uncoupled[0]
    N = len(u)
    if not 1 <= i < N:
        raise ValueError(f"Cannot swap outputs i={i} and i+1 out of only {N} outputs")
    dflag = src.isdual[0]
    a, b = u[i - 1], u[i]
    un = list(u)
    un[i - 1], un[i] = b, a
    un = tuple(un)
    dn = list(dflag)
    dn[i - 1], dn[i] = dflag[i], dflag[i - 1]
    dn = tuple(dn)
    unit = _unit_of(src)
    coupled_n = unit
    dst = FusionTreeBlock((un, ()), (dn, ()), unit)
    U = np.zeros((len(dst), len(src)))
    if a.isunit() or b.isunit():
        for col, (f, f2) in enumerate(src.trees):
            inner = f.innerlines
            ext = (u[0],) + inner + (coupled_n,)
            innern = inner
            if i > 1:
                innern = list(inner)
                innern[i - 2] = ext[i] if a.isunit() else ext[i - 2]
                innern = tuple(innern)
            fn = FusionTree(un, coupled_n, dn, innern)
            U[dst.index[(fn, f2)], col] = 1.0
        return dst, U
    for col, (f, f2) in enumerate(src.trees):
        inner = f.innerlines
        ext = (u[0],) + inner + (coupled_n,)
        if i == 1:
            c = inner[0] if N > 2 else coupled_n
            R = Rsymbol(b, a, c) if inv else Rsymbol(a, b, c)
            fn = FusionTree(un, coupled_n, dn, inner)
            U[dst.index[(fn, f2)], col] = R
            continue
        bb, dd = u[i - 1], u[i]
        aa, cc, ee = ext[i - 2], ext[i - 1], ext[i]
        s2 = set(ee.otimes(bb.dual()))
        for cp in aa.otimes(dd):
            if cp not in s2:
                continue
            if inv:
                coeff = (Rsymbol(dd, cc, ee) * Fsymbol(dd, aa, bb, ee, cp, cc)) * Rsymbol(dd, aa, cp)
            else:
                coeff = Rsymbol(cc, dd, ee) * (Fsymbol(dd, aa, bb, ee, cp, cc) * Rsymbol(aa, dd, cp))
            if coeff == 0:
                continue
            innern = list(inner)
            innern[i - 2] = cp
            fn = FusionTree(un, coupled_n, dn, tuple(innern))
            U[dst.index[(fn, f2)], col] = coeff
    return dst, U


def artin_braid(src, i, inv=False):
    if isinstance(src, FusionTreeBlock):
        return _artin_braid_block(src, i, inv)
    raise NotImplementedError("single-tree artin_braid is only used through braid()")


def _braid_unique_tree(f, p):
    """Braid of a unique-fusion splitting tree with symmetric braiding: coefficient is the
    product of R-symbols of every crossing pair (`braiding_manipulations.jl:226-242`)."""
    N = len(f)
    coeff = 1.0
    for i in range(N):
        for j in range(i):
            if p[j] > p[i]:
                a, b = f.uncoupled[p[j] - 1], f.uncoupled[p[i] - 1]
                coeff = coeff * Rsymbol(a, b, a.otimes(b)[0])
    un = tuple(f.uncoupled[k - 1] for k in p)
    dn = tuple(f.isdual[k - 1] for k in p)
    return FusionTree(un, f.coupled, dn, _abelian_inner(un)), coeff


def _fsbraid_pair(pair, p1, p2, l1, l2):
    f1, f2 = pair
    n1s, n2s = len(f1), len(f2)
    p = linearizepermutation(p1, p2, n1s, n2s)
    (f, f0), coeff1 = repartition((f1, f2), n1s + n2s)
    fp, coeff2 = _braid_unique_tree(f, p)
    (g1, g2), coeff3 = repartition((fp, f0), len(p1))
    return (g1, g2), coeff1 * coeff2 * coeff3


def _fsbraid_block(src, p1, p2, l1, l2):
    N1 = len(p1)
    N2 = len(p2)
    p = linearizepermutation(p1, p2, src.numout(), src.numin())
    levels = list(l1) + list(reversed(l2))
    dst, U = repartition(src, src.numout() + src.numin())
    for s in permutation2swaps(p):
        inv = levels[s - 1] > levels[s]
        dst, Ut = _artin_braid_block(dst, s, inv)
        U = Ut @ U
        levels[s - 1], levels[s] = levels[s], levels[s - 1]
    if N2 == 0:
        return dst, U
    dst, Ut = repartition(dst, N1)
    U = Ut @ U
    return dst, U


_FSBRAID_CACHE: dict = {}


def braid(src, p, levels):
    """Braid a tree pair (unique fusion) or a FusionTreeBlock; p = (p₁, p₂) 1-based,
    levels = (levels₁, levels₂)."""
    p1, p2 = tuple(p[0]), tuple(p[1])
    l1, l2 = tuple(levels[0]), tuple(levels[1])
    if isinstance(src, FusionTreeBlock):
        key = (src.uncoupled, src.isdual, p1, p2, l1, l2)
        hit = _FSBRAID_CACHE.get(key)
        if hit is None:
            hit = _fsbraid_block(src, p1, p2, l1, l2)
            if len(_FSBRAID_CACHE) > 10000:
                _FSBRAID_CACHE.clear()
            _FSBRAID_CACHE[key] = hit
        return hit
    return _fsbraid_pair(src, p1, p2, l1, l2)


def permute(src, p):
    """Permute = braid with levels 1..N (`braiding_manipulations.jl:356-361`)."""
    if isinstance(src, FusionTreeBlock):
        n1, n2 = src.numout(), src.numin()
    else:
        n1, n2 = len(src[0]), len(src[1])
    l1 = tuple(range(1, n1 + 1))
    l2 = tuple(range(n1 + 1, n1 + n2 + 1))
    return braid(src, p, (l1, l2))
