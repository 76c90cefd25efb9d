"""Dense conversion through fusion tensors — TEST INFRASTRUCTURE ONLY (pins oracle/core.py).

Restates the reference's dense check path, which its own tests use as ground truth:
- `fusiontensor` of sectors / trees / tree pairs (src/fusiontrees/fusiontrees.jl:278-341),
  with the Z isomorphism of a dual leg Z = sqrt(d_c)·conj(C^{c̄ c}_1) (`:282-291`);
- `convert(Array, t)` (src/tensors/abstracttensor.jl:733-751): A[axes(f₁), axes(f₂)] +=
  kron(t[f₁, f₂], F(f₁, f₂));
- `project_symmetric!` (src/tensors/abstracttensor.jl:755-792): the inverse, with 1/dim(c).
SU(2) Clebsch–Gordan coefficients are sympy's exact values (Condon–Shortley), magnetic
quantum numbers ordered m = j, j-1, ..., -j. U(1) fusion tensors are 1.
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

from .core import BT, Hom, dual, layout, qdim, unit


@lru_cache(maxsize=None)
def _cg_su2(j1, j2, j3):
    from sympy import Rational
    from sympy.physics.wigner import clebsch_gordan
    C = np.zeros((j1 + 1, j2 + 1, j3 + 1))
    h = lambda x: Rational(x, 2)
    for k1 in range(j1 + 1):
        m1 = j1 - 2 * k1
        for k2 in range(j2 + 1):
            m2 = j2 - 2 * k2
            m3 = m1 + m2
            if abs(m3) > j3:
                continue
            k3 = (j3 - m3) // 2
            C[k1, k2, k3] = float(clebsch_gordan(h(j1), h(j2), h(j3), h(m1), h(m2), h(m3)).evalf(40))
    return C


def fusiontensor3(a, b, c):
    if a[0] == "U1":
        return np.ones((1, 1, 1)) if a[1] + b[1] == c[1] else np.zeros((1, 1, 1))
    if a[0] == "SU2":
        return _cg_su2(a[1], b[1], c[1])
    out = np.ones((1, 1, 1))
    for x, y, z in zip(a[1], b[1], c[1]):
        f = fusiontensor3(x, y, z)
        s = tuple(p * q for p, q in zip(out.shape, f.shape))
        out = np.einsum("abc,def->adbecf", out, f).reshape(s)
    return out


def _zmap(c):
    """fusiontensor(FusionTree((c,), c, (true,))) = sqrt(d_c)·conj(C^{c̄ c}_1[:, :, 1])."""
    C = fusiontensor3(dual(c), c, unit(c))[:, :, 0]
    return math.sqrt(qdim(c)) * np.conj(C)


def fusiontensor_tree(f):
    unc, c, isd, inner = f
    N = len(unc)
    if N == 0:
        return np.ones(1)
    if N == 1:
        if isd[0]:
            return _zmap(c)
        return fusiontensor3(c, unit(c), c)[:, 0, :]
    if N == 2:
        a, b = unc
        X = fusiontensor3(a, b, c)
        if isd[0]:
            X = np.einsum("pa,abc->pbc", _zmap(a), X)
        if isd[1]:
            X = np.einsum("qb,abc->aqc", _zmap(b), X)
        return X
    tail = ((inner[0],) + unc[2:], c, (False,) + isd[2:], inner[1:])
    Ct = fusiontensor_tree(tail)
    C1 = fusiontensor_tree(((unc[0], unc[1]), inner[0], (isd[0], isd[1]), ()))
    return np.tensordot(C1, Ct, axes=([2], [0]))


def fusiontensor_pair(f1, f2):
    F1 = fusiontensor_tree(f1)
    F2 = fusiontensor_tree(f2)
    d1, d2 = F1.shape[:-1], F2.shape[:-1]
    M = F1.reshape(-1, F1.shape[-1]) @ np.conj(F2.reshape(-1, F2.shape[-1])).T
    return M.reshape(d1 + d2)


def _kron_nd(A, F):
    """Per-dimension Kronecker product, degeneracy index major (reference `_kron`)."""
    nd = A.ndim
    out = np.multiply.outer(A, F)  # axes: A dims then F dims
    perm = []
    for k in range(nd):
        perm += [k, nd + k]
    out = np.transpose(out, perm)
    return out.reshape(tuple(A.shape[k] * F.shape[k] for k in range(nd)))


def to_dense(t: BT):
    W = t.W
    legs = list(W.cod) + list(W.dom)
    dims = [sp.dim() for sp in legs]
    dt = np.result_type(t.data.dtype, np.float64)
    A = np.zeros(dims, dtype=dt)
    for (f1, f2) in layout(W)[3]:
        F = fusiontensor_pair(f1, f2)
        sub = t.sub((f1, f2))
        sl = tuple(slice(r.start, r.stop) for r in
                   [sp.axes(s) for sp, s in zip(W.cod, f1[0])] + [sp.axes(s) for sp, s in zip(W.dom, f2[0])])
        A[sl] += _kron_nd(np.asarray(sub), F)
    return A


def from_dense(W: Hom, A):
    total = layout(W)[0]
    data = np.zeros(total, dtype=np.result_type(A.dtype, np.float64))
    t = BT(W, data)
    for (f1, f2) in layout(W)[3]:
        F = fusiontensor_pair(f1, f2)
        sl = tuple(slice(r.start, r.stop) for r in
                   [sp.axes(s) for sp, s in zip(W.cod, f1[0])] + [sp.axes(s) for sp, s in zip(W.dom, f2[0])])
        D = A[sl]
        sub = t.sub((f1, f2))
        nd = D.ndim
        shp = []
        for k in range(nd):
            shp += [sub.shape[k], F.shape[k]]
        Dr = D.reshape(shp)
        # contract conj(F) over the multiplet indices
        letters = "abcdefghijklmnop"
        ein_d = "".join(letters[2 * k] + letters[2 * k + 1] for k in range(nd))
        ein_f = "".join(letters[2 * k + 1] for k in range(nd))
        ein_o = "".join(letters[2 * k] for k in range(nd))
        val = np.einsum(f"{ein_d},{ein_f}->{ein_o}", Dr, np.conj(F)) / qdim(f1[1])
        sub[...] = val
    return t
