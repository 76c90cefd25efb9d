"""CPU oracle for the symmetric-contraction path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may import
this package, and only as the checker or the timed CPU baseline; the product never calls it.

A plain restatement of the reference algorithm in numpy (pure-Python fusion-tree algebra,
numpy/BLAS for the block arithmetic), written independently of the product's host code:
sectors are tuples, fusion trees are tuples, recoupling moves act on dictionaries of tree
pairs {pair: coefficient} one tree pair at a time.

Parity status: the reference (Julia) cannot run in this environment and ships no golden
vectors. This restatement is pinned by the reference's own test identities instead
(oracle/dense.py): dense conversion through Clebsch–Gordan fusion tensors commutes with
permute (test/tensors/indexmanipulations.jl:77-99), contraction equals the dense contraction
(test/tensors/contractions.jl:78-92), norm/dot are invariant under every permutation
(test/tensors/indexmanipulations.jl:55-75). SU(2) symbols are exact (sympy) rounded once.

Reference citations (TensorKit.jl v0.17.1):
  sectors/symbols  docs/src/man/sectors.md:243-264, 350-400; docs/src/appendix/categories.md:590-593
  tree iteration   src/fusiontrees/iterator.jl:98-226
  structure        src/spaces/structure.jl:41-196, src/spaces/homspace.jl:94-126,178-188,
                   src/spaces/productspace.jl:147-183, src/spaces/gradedspace.jl:92-110,180-187
  bend / braid     src/fusiontrees/duality_manipulations.jl:33-194,460-505;
                   src/fusiontrees/braiding_manipulations.jl:18-79,215-251,304-361
  permutation aux  src/auxiliary/auxiliary.jl:1-28
  transformers     src/tensors/treetransformers.jl:16-120,186-205
  add_transform    src/tensors/indexmanipulations.jl:658-726
  mul/norm/tr      src/tensors/linalg.jl:257-282,319-370; inner src/tensors/vectorinterface.jl:114-130
  contract         src/tensors/tensoroperations.jl:130-161,318-462
  trace            src/tensors/tensoroperations.jl:212-296, src/fusiontrees/basic_manipulations.jl:30-52
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

# ============================================================================================
# sectors: ('U1', 2q) | ('SU2', 2j) | ('P', (s1, s2, ...))
# ============================================================================================


def U1(q):
    return ("U1", int(round(2 * q)))


def SU2(j):
    return ("SU2", int(round(2 * j)))


def P(*parts):
    return ("P", tuple(parts))


def unit(s):
    if s[0] == "P":
        return ("P", tuple(unit(x) for x in s[1]))
    return (s[0], 0)


def dual(s):
    if s[0] == "U1":
        return ("U1", -s[1])
    if s[0] == "SU2":
        return s
    return ("P", tuple(dual(x) for x in s[1]))


def qdim(s):
    if s[0] == "U1":
        return 1
    if s[0] == "SU2":
        return s[1] + 1
    r = 1
    for x in s[1]:
        r *= qdim(x)
    return r


def unique(s):
    if s[0] == "U1":
        return True
    if s[0] == "SU2":
        return False
    return all(unique(x) for x in s[1])


def order_key(s):
    if s[0] == "U1":
        return (abs(s[1]), 1 if s[1] < 0 else 0)
    if s[0] == "SU2":
        return (s[1],)
    return tuple(order_key(x) for x in s[1])


def fuse(a, b):
    """Fusion outputs in the reference iteration order."""
    if a[0] == "U1":
        return [("U1", a[1] + b[1])]
    if a[0] == "SU2":
        return [("SU2", t) for t in range(abs(a[1] - b[1]), a[1] + b[1] + 1, 2)]
    comps = [fuse(x, y) for x, y in zip(a[1], b[1])]
    res = []  # Iterators.product order: first component varies fastest
    idx = [0] * len(comps)
    while True:
        res.append(("P", tuple(comps[k][idx[k]] for k in range(len(comps)))))
        k = 0
        while k < len(comps):
            idx[k] += 1
            if idx[k] < len(comps[k]):
                break
            idx[k] = 0
            k += 1
        if k == len(comps):
            return res


def Nsym(a, b, c):
    if a[0] == "U1":
        return int(a[1] + b[1] == c[1])
    if a[0] == "SU2":
        return int(abs(a[1] - b[1]) <= c[1] <= a[1] + b[1] and (a[1] + b[1] + c[1]) % 2 == 0)
    r = 1
    for x, y, z in zip(a[1], b[1], c[1]):
        r *= Nsym(x, y, z)
    return r


@lru_cache(maxsize=None)
def _racahW_float(s1, s2, s3, s4, s5, s6):
    """float(racahW(s1, s2, s4, s3, s5, s6)) from sympy's exact 6j (twice-spin args):
    racahW(j1,j2,J,j3,J12,J23) = (-1)^(j1+j2+j3+J) {j1 j2 J12; j3 J J23}."""
    from sympy import Rational
    from sympy.physics.wigner import wigner_6j
    h = lambda x: Rational(x, 2)
    val = wigner_6j(h(s1), h(s2), h(s5), h(s3), h(s4), h(s6))
    ph = (s1 + s2 + s3 + s4) // 2
    val = -val if ph % 2 else val
    return float(val.evalf(50))


@lru_cache(maxsize=None)
def Fsym(a, b, c, d, e, f):
    if a[0] == "U1":
        return 1.0 if (Nsym(a, b, e) and Nsym(e, c, d) and Nsym(b, c, f) and Nsym(a, f, d)) else 0.0
    if a[0] == "SU2":
        s = (a[1], b[1], c[1], d[1], e[1], f[1])
        if all(x == 0 for x in s):
            return 1.0
        if not (Nsym(a, b, e) and Nsym(e, c, d) and Nsym(b, c, f) and Nsym(a, f, d)):
            return 0.0
        return (math.sqrt(e[1] + 1) * math.sqrt(f[1] + 1)) * _racahW_float(*s)
    r = 1.0
    for comp in zip(a[1], b[1], c[1], d[1], e[1], f[1]):
        r = r * Fsym(*comp)
    return r


def Rsym(a, b, c):
    if a[0] == "U1":
        return float(Nsym(a, b, c))
    if a[0] == "SU2":
        if not Nsym(a, b, c):
            return 0.0
        return 1.0 if ((a[1] + b[1] - c[1]) // 2) % 2 == 0 else -1.0
    r = 1.0
    for comp in zip(a[1], b[1], c[1]):
        r = r * Rsym(*comp)
    return r


def fsphase(a):
    if a[0] == "U1":
        return 1.0
    if a[0] == "SU2":
        return -1.0 if a[1] % 2 else 1.0
    r = 1.0
    for x in a[1]:
        r = r * fsphase(x)
    return r


def sqrtd(a):
    return 1.0 if unique(a) else math.sqrt(qdim(a))


def isqrtd(a):
    return 1.0 if unique(a) else 1.0 / math.sqrt(qdim(a))


def Bsym(a, b, c):
    if unique(a):
        return float(Nsym(a, b, c))
    return (sqrtd(a) * sqrtd(b) * isqrtd(c)) * Fsym(a, b, dual(b), a, c, unit(a))


def fuse_all(secs, u):
    if not secs:
        return [u]
    acc = [secs[0]]
    for s in secs[1:]:
        nxt = []
        for a in acc:
            for c in fuse(a, s):
                if c not in nxt:
                    nxt.append(c)
        acc = nxt
    return acc


# ============================================================================================
# spaces: Space(dict sector->deg, dual)  ; HomSpace = (codomain list, domain list)
# ============================================================================================
class Space:
    def __init__(self, degs, dual=False):
        self.degs = {s: int(d) for s, d in degs.items() if int(d) > 0}
        self.dual = bool(dual)
        self.keys = sorted(self.degs, key=order_key)

    def sectors(self):
        return [dual(s) for s in self.keys] if self.dual else list(self.keys)

    def deg(self, c):
        return self.degs.get(dual(c) if self.dual else c, 0)

    def dim(self):
        return sum(qdim(s) * self.deg(s) for s in self.sectors())

    def flipdual(self):
        return Space(self.degs, not self.dual)

    def axes(self, c):
        off = 0
        for s in self.sectors():
            if s == c:
                break
            off += qdim(s) * self.deg(s)
        return range(off, off + qdim(c) * self.deg(c))

    def key(self):
        return (tuple((s, self.degs[s]) for s in self.keys), self.dual)

    def __eq__(self, o):
        return isinstance(o, Space) and self.key() == o.key()

    def __hash__(self):
        return hash(self.key())

    def __repr__(self):
        return f"Space({self.degs}{', dual' if self.dual else ''})"


class Hom:
    """cod ← dom; `u` (the unit sector) is carried explicitly so that spaces without legs
    (scalars) keep their sector type."""

    def __init__(self, cod, dom, u=None):
        self.cod = tuple(cod)
        self.dom = tuple(dom)
        if u is None:
            u = unit((self.cod + self.dom)[0].keys[0])
        self.u = u

    def n1(self):
        return len(self.cod)

    def n2(self):
        return len(self.dom)

    def leg(self, i):  # 1-based
        return self.cod[i - 1] if i <= len(self.cod) else self.dom[i - 1 - len(self.cod)].flipdual()

    def select(self, p):
        return Hom([self.leg(i) for i in p[0]], [self.leg(i).flipdual() for i in p[1]], self.u)

    def adjoint(self):
        return Hom(self.dom, self.cod, self.u)

    def __eq__(self, o):
        return self.cod == o.cod and self.dom == o.dom and self.u == o.u

    def __hash__(self):
        return hash((self.cod, self.dom, self.u))

    def unit(self):
        return self.u


def _product(lists):
    """Iterators.product order: first list fastest."""
    res = []
    if any(len(l) == 0 for l in lists):
        return res
    idx = [0] * len(lists)
    while True:
        res.append(tuple(lists[k][idx[k]] for k in range(len(lists))))
        k = 0
        while k < len(lists):
            idx[k] += 1
            if idx[k] < len(lists[k]):
                break
            idx[k] = 0
            k += 1
        if k == len(lists):
            return res


# fusion trees: (uncoupled tuple, coupled, isdual tuple, inner tuple)
def trees(lists, c, isdual):
    """Trees in reference order (last leg slowest, then its inner line, then the front)."""
    def rec(ls, cc):
        n = len(ls)
        if n == 0:
            if cc == unit(cc):
                yield (), ()
            return
        if n == 1:
            if cc in ls[0]:
                yield (cc,), ()
            return
        if n == 2:
            for b in ls[1]:
                for a in ls[0]:
                    if Nsym(a, b, cc):
                        yield (a, b), ()
            return
        for b in ls[-1]:
            for a in fuse(cc, dual(b)):
                for ro, rl in rec(ls[:-1], a):
                    yield ro + (b,), rl + (a,)
    return [(o, c, tuple(isdual), l) for o, l in rec([list(x) for x in lists], c)]


def blocksectors_prod(spaces, u):
    if len(spaces) == 0:
        return [u]
    if len(spaces) == 1:
        return sorted(spaces[0].sectors(), key=order_key)
    out = []
    for s in _product([sp.sectors() for sp in spaces]):
        for c in fuse_all(list(s), u):
            if c not in out:
                out.append(c)
    return sorted(out, key=order_key)


def has_block(spaces, c):
    return len(trees([sp.sectors() for sp in spaces], c, [sp.dual for sp in spaces])) > 0


def coupled_sectors(W: Hom):
    u = W.unit()
    n1, n2 = W.n1(), W.n2()
    if n1 == 0 and n2 == 0:
        return [u]
    if n1 == 0:
        return [c for c in blocksectors_prod(W.dom, u) if c == u]
    if n2 == 0:
        return [c for c in blocksectors_prod(W.cod, u) if c == u]
    if n2 <= n1:
        return [c for c in blocksectors_prod(W.dom, u) if has_block(W.cod, c)]
    return [c for c in blocksectors_prod(W.cod, u) if has_block(W.dom, c)]


@lru_cache(maxsize=4096)
def layout(W: Hom):
    """(total, blocks {c: (d1, d2, off)}, subs {(f1, f2): (sizes, strides, off)}, pairs list)."""
    blocks = {}
    subs = {}
    pairs = []
    off = 0
    for c in coupled_sectors(W):
        t1 = trees([sp.sectors() for sp in W.cod], c, [sp.dual for sp in W.cod])
        t2 = trees([sp.sectors() for sp in W.dom], c, [sp.dual for sp in W.dom])
        d1s = [[sp.deg(s) for sp, s in zip(W.cod, f[0])] for f in t1]
        d2s = [[sp.deg(s) for sp, s in zip(W.dom, f[0])] for f in t2]
        D1 = sum(int(np.prod(x)) for x in d1s)
        D2 = sum(int(np.prod(x)) for x in d2s)
        blocks[c] = (D1, D2, off)
        o2 = 0
        for f2, ds2 in zip(t2, d2s):
            o1 = 0
            for f1, ds1 in zip(t1, d1s):
                st = []
                acc = 1
                for x in ds1:
                    st.append(acc)
                    acc *= x
                acc = D1
                for x in ds2:
                    st.append(acc)
                    acc *= x
                subs[(f1, f2)] = (tuple(ds1) + tuple(ds2), tuple(st), off + o2 * D1 + o1)
                pairs.append((f1, f2))
                o1 += int(np.prod(ds1))
            o2 += int(np.prod(ds2))
        off += D1 * D2
    return off, blocks, subs, pairs


# ============================================================================================
# tree-pair moves on dictionaries {(f1, f2): coeff}
# ============================================================================================
def _bendright_pair(f1, f2):
    (u1, c, d1, in1), (u2, c2, d2, in2) = f1, f2
    n1, n2 = len(u1), len(u2)
    a = unit(c) if n1 == 1 else (u1[0] if n1 == 2 else in1[-1])
    b = u1[-1]
    g1 = (u1[:-1], a, d1[:-1], in1[:-1] if n1 > 2 else ())
    g2 = (u2 + (dual(b),), a, d2 + (not d1[-1],), (in2 + (c,)) if n2 > 1 else ())
    coeff = sqrtd(c) * isqrtd(a)
    if d1[-1]:
        coeff = coeff * fsphase(dual(b))
    coeff = coeff * Bsym(a, b, c)
    return (g1, g2), coeff


def bendright(lc):
    out = {}
    for (f1, f2), x in lc.items():
        pr, cf = _bendright_pair(f1, f2)
        out[pr] = out.get(pr, 0.0) + cf * x
    return out


def bendleft(lc):
    out = {}
    for (f1, f2), x in lc.items():
        (g2, g1), cf = _bendright_pair(f2, f1)
        out[(g1, g2)] = out.get((g1, g2), 0.0) + cf * x
    return out


def repartition(lc, N):
    n1 = len(next(iter(lc))[0][0])
    n = n1 - N
    for _ in range(abs(n)):
        lc = bendright(lc) if n > 0 else bendleft(lc)
    return lc


def _artin(f, i, inv):
    """Elementary braid of legs i, i+1 (1-based) of a splitting tree coupled to the unit."""
    u, c0, dd, inner = f
    N = len(u)
    a, b = u[i - 1], u[i]
    un = u[:i - 1] + (b, a) + u[i + 1:]
    dn = dd[:i - 1] + (dd[i], dd[i - 1]) + dd[i + 1:]
    ext = (u[0],) + inner + (c0,)
    if a == unit(a) or b == unit(b):
        inn = list(inner)
        if i > 1:
            inn[i - 2] = ext[i] if a == unit(a) else ext[i - 2]
        return {(un, c0, dn, tuple(inn)): 1.0}
    if i == 1:
        c = inner[0] if N > 2 else c0
        r = Rsym(b, a, c) if inv else Rsym(a, b, c)
        return {(un, c0, dn, inner): r}
    bb, dv = u[i - 1], u[i]
    aa, cc, ee = ext[i - 2], ext[i - 1], ext[i]
    out = {}
    cands = fuse(ee, dual(bb))
    for cp in fuse(aa, dv):
        if cp not in cands:
            continue
        if inv:
            x = (Rsym(dv, cc, ee) * Fsym(dv, aa, bb, ee, cp, cc)) * Rsym(dv, aa, cp)
        else:
            x = Rsym(cc, dv, ee) * (Fsym(dv, aa, bb, ee, cp, cc) * Rsym(aa, dv, cp))
        if x == 0.0:
            continue
        inn = list(inner)
        inn[i - 2] = cp
        out[(un, c0, dn, tuple(inn))] = x
    return out


def linperm(p1, p2, n1, n2):
    q = [(n2 + 2 * n1 + 1 - x) if x > n1 else x for x in p1]
    q += [(n2 + 2 * n1 + 1 - x) if x > n1 else x for x in reversed(p2)]
    return q


def swaps_of(perm):
    p = list(perm)
    sw = []
    N = len(p)
    for k in range(1, N):
        sw += list(range(p[k - 1] - 1, k - 1, -1))
        for l in range(k + 1, N + 1):
            if p[l - 1] < p[k - 1]:
                p[l - 1] += 1
        p[k - 1] = k
    return sw


def braid_pair(pair, p1, p2, l1, l2):
    """{(f1', f2'): coeff} for one tree pair (multiplicity-free sectors)."""
    f1, f2 = pair
    n1s, n2s = len(f1[0]), len(f2[0])
    perm = linperm(p1, p2, n1s, n2s)
    levels = list(l1) + list(reversed(l2))
    lc = repartition({pair: 1.0}, n1s + n2s)
    if unique(f1[1]):
        # symmetric braiding of a unique-fusion tree: product of R over crossing pairs
        ((t, t0), x), = lc.items()
        r = 1.0
        for i in range(len(perm)):
            for j in range(i):
                if perm[j] > perm[i]:
                    aa, bb = t[0][perm[j] - 1], t[0][perm[i] - 1]
                    r = r * Rsym(aa, bb, fuse(aa, bb)[0])
        un = tuple(t[0][k - 1] for k in perm)
        dn = tuple(t[2][k - 1] for k in perm)
        inner = []
        if len(un) > 2:
            acc = fuse(un[0], un[1])[0]
            inner.append(acc)
            for k in range(2, len(un) - 1):
                acc = fuse(acc, un[k])[0]
                inner.append(acc)
        lc = {((un, t[1], dn, tuple(inner)), t0): x * r}
    else:
        for s in swaps_of(perm):
            inv = levels[s - 1] > levels[s]
            new = {}
            for (t, t0), x in lc.items():
                for tn, y in _artin(t, s, inv).items():
                    new[(tn, t0)] = new.get((tn, t0), 0.0) + y * x
            lc = new
            levels[s - 1], levels[s] = levels[s], levels[s - 1]
    # the final repartition is composed on its own and then applied (U = U_tmp * U)
    out = {}
    for pr, x in lc.items():
        for q, y in repartition({pr: 1.0}, len(p1)).items():
            out[q] = out.get(q, 0.0) + y * x
    return out


def permute_pair(pair, p):
    n1, n2 = len(pair[0][0]), len(pair[1][0])
    return braid_pair(pair, p[0], p[1], tuple(range(1, n1 + 1)), tuple(range(n1 + 1, n1 + n2 + 1)))


# ============================================================================================
# block-sparse tensors
# ============================================================================================
class BT:
    """Block-sparse tensor: Hom space + flat numpy data in the reference layout."""

    def __init__(self, W: Hom, data):
        self.W = W
        self.data = np.asarray(data)
        assert self.data.ndim == 1 and self.data.size == layout(W)[0]

    def sub(self, pair):
        sz, st, off = layout(self.W)[2][pair]
        it = self.data.itemsize
        return np.lib.stride_tricks.as_strided(self.data[off:], sz, tuple(s * it for s in st))

    def block(self, c):
        d1, d2, off = layout(self.W)[1][c]
        return self.data[off:off + d1 * d2].reshape(d2, d1).T

    def blocks(self):
        return {c: self.block(c) for c in layout(self.W)[1]}


def adjoint_sub(t: BT, pair):
    """Sub-block (f1, f2) of adjoint(t): conj(permutedims(t[f2, f1], (dom..., cod...)))."""
    f1, f2 = pair
    x = t.sub((f2, f1))
    n1 = t.W.n1()
    perm = tuple(range(n1, x.ndim)) + tuple(range(n1))
    return np.conj(np.transpose(x, perm))


def permute(t: BT, p, alpha=1.0, adjoint=False, tdst=None, beta=0.0):
    """β·tdst + α·permute(t or adjoint(t), p) via tree-pair transformation dictionaries."""
    Wsrc = t.W.adjoint() if adjoint else t.W
    Wdst = Wsrc.select(p)
    total = layout(Wdst)[0]
    out = np.zeros(total, dtype=t.data.dtype) if tdst is None else tdst.data * beta
    res = BT(Wdst, out)
    flat = list(p[0]) + list(p[1])
    axes = [k - 1 for k in flat]
    for pair in layout(Wsrc)[3]:
        src = adjoint_sub(t, pair) if adjoint else t.sub(pair)
        moved = np.transpose(src, axes)
        for dpair, x in permute_pair(pair, p).items():
            if x == 0.0:
                continue
            d = res.sub(dpair)
            d += (alpha * x) * moved
    return res


def split_tree(f, M):
    """(f₁, f₂): f₁ keeps the first M uncoupled legs and couples to the line between them and
    the rest; f₂ starts with that line (src/fusiontrees/basic_manipulations.jl:30-52)."""
    u, c, d, inner = f
    N = len(u)
    ext = (u[0],) + tuple(inner) + (c,) if N > 0 else (c,)
    c1 = unit(c) if M == 0 else ext[M - 1]
    f1 = (u[:M], c1, d[:M], tuple(inner[:max(0, M - 2)]))
    f2 = ((c1,) + u[M:], c, (False,) + d[M:], tuple(ext[M:M + max(0, N - M - 1)]))
    return f1, f2


def trace_permute(t: BT, p, q, alpha=1.0, tdst=None, beta=0.0):
    """β·tdst + α·(permute t by p, tracing the leg pairs q = (q₁, q₂)) for bosonic sectors
    (src/tensors/tensoroperations.jl:212-296): every tree pair is permuted to
    ((p₁, q₁), (p₂, q₂)); both trees are split after the kept legs, pairs whose split-off
    trees differ vanish, the others carry dim(g.coupled)/dim(g.uncoupled[1]) and a dense
    partial trace of the sub-block."""
    W = t.W
    p1, p2 = tuple(p[0]), tuple(p[1])
    q1, q2 = tuple(q[0]), tuple(q[1])
    N1, N2 = len(p1), len(p2)
    Wdst = W.select((p1, p2))
    total = layout(Wdst)[0]
    out = np.zeros(total, dtype=t.data.dtype) if tdst is None else tdst.data * beta
    res = BT(Wdst, out)
    r = (p1 + q1, p2 + q2)
    letters = "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ"
    nlegs = W.n1() + W.n2()
    sub_in = [""] * nlegs
    k = 0
    for x in p1 + p2:
        sub_in[x - 1] = letters[k]
        k += 1
    for a, b in zip(q1, q2):
        sub_in[a - 1] = sub_in[b - 1] = letters[k]
        k += 1
    spec = "".join(sub_in) + "->" + "".join(sub_in[x - 1] for x in p1 + p2)
    for pair in layout(W)[3]:
        src = t.sub(pair)
        traced = None
        for (f1p, f2p), x in permute_pair(pair, r).items():
            if x == 0.0:
                continue
            h1, g1 = split_tree(f1p, N1)
            h2, g2 = split_tree(f2p, N2)
            if g1 != g2:
                continue
            x = x * qdim(g1[1]) / qdim(g1[0][0])
            if traced is None:
                traced = np.einsum(spec, src)
            res.sub((h1, h2))[...] += (alpha * x) * traced
    return res


def mul(A: BT, B: BT, adjA=False, adjB=False):
    """Blockwise C = op(A)·op(B) (op = adjoint when flagged)."""
    WA = A.W.adjoint() if adjA else A.W
    WB = B.W.adjoint() if adjB else B.W
    assert WA.dom == WB.cod
    WC = Hom(WA.cod, WB.dom, WA.unit())
    dt = np.result_type(A.data, B.data)
    C = BT(WC, np.zeros(layout(WC)[0], dtype=dt))
    bA = A.blocks()
    bB = B.blocks()
    for c in layout(WC)[1]:
        if c in bA and c in bB:
            a = bA[c].conj().T if adjA else bA[c]
            b = bB[c].conj().T if adjB else bB[c]
            C.block(c)[...] = a @ b
    return C


def norm(t: BT):
    return math.sqrt(sum(qdim(c) * float(np.vdot(b, b).real) for c, b in t.blocks().items()))


def inner(x: BT, y: BT):
    return sum(qdim(c) * np.vdot(x.block(c), y.block(c)) for c in layout(x.W)[1])


def tr(t: BT):
    return sum(qdim(c) * np.trace(b) for c, b in t.blocks().items())


def contract(A: BT, la, conjA, B: BT, lb, conjB, out_cod, out_dom):
    """Pairwise contraction over shared labels: permute both operands into GEMM form,
    blockwise multiply, permute into (out_cod; out_dom)."""
    contracted = [l for l in la if l in lb]
    openA = [l for l in la if l not in lb]
    openB = [l for l in lb if l not in la]

    def legs(t, conj):
        return t.W.n2() if conj else t.W.n1()
    # an adjoint's leg i corresponds to the parent's adjointtensorindex(i); labels refer to
    # the parent legs, so map them into adjoint positions
    def pos(t, conj, labels, l):
        i = labels.index(l) + 1
        if not conj:
            return i
        n1, n2 = t.W.n1(), t.W.n2()
        return n2 + i if i <= n1 else i - n1
    pA = (tuple(pos(A, conjA, la, l) for l in openA), tuple(pos(A, conjA, la, l) for l in contracted))
    pB = (tuple(pos(B, conjB, lb, l) for l in contracted), tuple(pos(B, conjB, lb, l) for l in openB))
    An = permute(A, pA, adjoint=conjA)
    Bn = permute(B, pB, adjoint=conjB)
    Cn = mul(An, Bn)
    outl = openA + openB
    pC = (tuple(outl.index(l) + 1 for l in out_cod), tuple(outl.index(l) + 1 for l in out_dom))
    return permute(Cn, pC)


def network(expr_factors, lhs, tensors):
    """Left-to-right pairwise evaluation of an @tensor network.
    expr_factors: [(name, labels, conj)], lhs: (cod labels, dom labels)."""
    name, labels, conj = expr_factors[0]
    cur, curl, curc = tensors[name], list(labels), conj
    for k in range(1, len(expr_factors)):
        nb, lb, cb = expr_factors[k]
        B = tensors[nb]
        lbl = list(lb)
        openA = [l for l in curl if l not in lbl]
        openB = [l for l in lbl if l not in curl]
        if k == len(expr_factors) - 1:
            cod, dom = list(lhs[0]), list(lhs[1])
        else:
            cod, dom = openA, openB
        cur = contract(cur, curl, curc, B, lbl, cb, cod, dom)
        curl, curc = cod + dom, False
    return cur


def randn(W: Hom, seed, complex_=False):
    n = layout(W)[0]
    rng = np.random.Generator(np.random.PCG64(seed))
    if not complex_:
        return BT(W, rng.standard_normal(n))
    x = rng.standard_normal(2 * n).reshape(n, 2)
    return BT(W, (x[:, 0] + 1j * x[:, 1]) / math.sqrt(2.0))


# ============================================================================================
# flattened transformer tables (for the bit-exact table comparison)
# ============================================================================================
def transformer_table(Wsrc: Hom, p, adjoint_parent=None):
    """Per source tree pair (in source order): (src (sz, str, off), [(dst (sz, str, off), coeff)])."""
    Wdst = Wsrc.select(p)
    Ld = layout(Wdst)[2]
    if adjoint_parent is None:
        Ls = layout(Wsrc)[2]
        srcs = {pr: Ls[pr] for pr in layout(Wsrc)[3]}
    else:
        Lp = layout(adjoint_parent)[2]
        n1 = adjoint_parent.n1()
        srcs = {}
        for (f1, f2), (sz, st, off) in Lp.items():
            perm = list(range(n1, len(sz))) + list(range(n1))
            srcs[(f2, f1)] = (tuple(sz[k] for k in perm), tuple(st[k] for k in perm), off)
    out = []
    for pr in layout(Wsrc)[3]:
        d = permute_pair(pr, p)
        out.append((srcs[pr], [(Ld[q], x) for q, x in d.items() if x != 0.0]))
    return out
