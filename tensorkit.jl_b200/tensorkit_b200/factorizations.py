"""Block factorizations of device tensors with sector-aware truncation.

Follows TensorKit's factorization layer (`src/factorizations/matrixalgebrakit.jl`,
`src/factorizations/truncation.jl`): every factorization acts block by block on the coupled
sectors (`foreachblock`, `matrixalgebrakit.jl:34-49`), and the new bond space is built from the
fused codomain/domain (`initialize_output`, `matrixalgebrakit.jl:128-200`):
- `svd_compact`, `qr_compact`, `lq_compact`: V = infimum(fuse(codomain), fuse(domain));
- `eigh_full`: V = fuse(domain) (square blocks);
- `svd_trunc`, `eigh_trunc`: the same, then the kept values per sector are chosen by a
  truncation strategy over all sectors at once (`findtruncated`, `truncation.jl:158-300`), with
  the values weighted by the quantum dimension dim(c) where the strategy sums or counts them.

The per-block linear algebra runs on the device through the vendor solver (cuSOLVER via
`torch.linalg`), one batched call per distinct block shape. Singular values come in
non-increasing order per block and eigenvalues in increasing order, as from LAPACK. The
diagonal factor (S, D) is returned as a TensorMap V ← V whose blocks are diagonal, together with
the values as a `SectorVector` (sector → 1-D tensor).

The block decompositions themselves (U, S, Vᴴ of one matrix) come from MatrixAlgebraKit in the
reference; the truncation strategies' selection rules restated here are TensorKit's own
(`truncation.jl`), and `trunctol` keeps values with by(v) > atol (keep_below=False).
"""
from __future__ import annotations

import math

import numpy as np

from .spaces import GradedSpace, HomSpace, ProductSpace, SpaceMismatch
from .tensor import AdjointTensorMap, TensorMap

__all__ = ["SectorVector", "svd_compact", "svd_vals", "svd_trunc", "qr_compact", "lq_compact",
           "eigh_full", "eigh_vals", "eigh_trunc", "notrunc", "truncrank", "trunctol", "truncerror",
           "truncspace", "truncation_error"]


# ---- sector vectors ------------------------------------------------------------------------
class SectorVector(dict):
    """Values per coupled sector (sector → 1-D tensor), `SectorVector` in
    `src/tensors/sectorvector.jl`. Norms weight every sector by its quantum dimension."""

    def norm(self, p=2):
        """`norm(v, p)` = (Σ_c dim(c) Σ |v_c|^p)^(1/p) (`linalg.jl:261-276` through
        `sectorvector.jl:112-114`); p = inf: the largest |v|."""
        if p == math.inf:
            return max((float(v.abs().max()) for v in self.values() if v.numel()), default=0.0)
        if p <= 0:
            raise ValueError("norm with non-positive p is not defined")
        s = sum(c.dim() * float((v.abs() ** p).sum()) for c, v in self.items())
        return s ** (1.0 / p)


def _fuse(P: ProductSpace) -> GradedSpace:
    return GradedSpace({c: P.blockdim(c) for c in P.blocksectors()}, unit=P.unit())


def _infimum(V: GradedSpace, W: GradedSpace) -> GradedSpace:
    dims = {c: min(V.dim(c), W.dim(c)) for c in V.sectors() if c in set(W.sectors())}
    return GradedSpace(dims, unit=V.unit())


def _check(t):
    if isinstance(t, AdjointTensorMap):
        raise TypeError("factorize the parent tensor or a copy (lazy adjoints are not supported here)")
    return t


def _batched(blocks: dict, fn):
    """Apply fn to stacks of equal-shape blocks; returns {c: outputs of fn for that block}."""
    import torch
    groups: dict = {}
    for c, b in blocks.items():
        groups.setdefault(tuple(b.shape), []).append(c)
    out = {}
    for shape, cs in groups.items():
        res = fn(torch.stack([blocks[c] for c in cs]))
        for i, c in enumerate(cs):
            out[c] = tuple(r[i] for r in res)
    return out


def _new(space: HomSpace, like: TensorMap, dtype=None):
    return TensorMap.zeros(space, dtype=dtype or like.data.dtype, device=like.data.device)


def _real_dtype(t):
    import torch
    return torch.float64 if t.data.dtype in (torch.float64, torch.complex128) else torch.float32


def _diag(V: GradedSpace, vals: SectorVector, like, dtype):
    D = _new(HomSpace(ProductSpace((V,), V.unit()), ProductSpace((V,), V.unit()), V.unit()), like, dtype)
    for c in D.blocksectors():
        D.block(c).diagonal().copy_(vals[c])
    return D


# ---- SVD -----------------------------------------------------------------------------------
SVD_DRIVER = None  # cuSOLVER driver for device SVDs (None: torch's default; "gesvdj": Jacobi)


def _svd_blocks(t):
    import torch
    blocks = {c: t.block(c) for c in t.blocksectors()}
    drv = SVD_DRIVER if t.data.is_cuda else None
    return _batched(blocks, lambda x: torch.linalg.svd(x, full_matrices=False, driver=drv))


def svd_compact(t):
    """U, S, Vᴴ with t = U·S·Vᴴ per block; V = infimum(fuse(codomain), fuse(domain))."""
    t = _check(t)
    res = _svd_blocks(t)
    V = _infimum(_fuse(t.space.codomain), _fuse(t.space.domain))
    U, S, Vh, _ = _assemble_svd(t, V, {c: (u, s, vh) for c, (u, s, vh) in res.items()})
    return U, S, Vh


def _assemble_svd(t, V, parts):
    u1 = t.space.unit()
    PV = ProductSpace((V,), u1)
    U = _new(HomSpace(t.space.codomain, PV, u1), t)
    Vh = _new(HomSpace(PV, t.space.domain, u1), t)
    vals = SectorVector()
    for c, (u, s, vh) in parts.items():
        if V.dim(c) == 0:
            continue
        U.block(c).copy_(u)
        Vh.block(c).copy_(vh)
        vals[c] = s
    S = _diag(V, vals, t, _real_dtype(t))
    return U, S, Vh, vals


def svd_vals(t) -> SectorVector:
    """Singular values per coupled sector (non-increasing)."""
    import torch
    t = _check(t)
    return SectorVector({c: torch.linalg.svdvals(t.block(c)) for c in t.blocksectors()})


# ---- truncation strategies (truncation.jl) ------------------------------------------------
class _Strategy:
    def __and__(self, other):
        return _Combine(self, other, "and")

    def __or__(self, other):
        return _Combine(self, other, "or")


class notrunc(_Strategy):
    def select(self, values: SectorVector):
        return {c: np.ones(v.numel(), bool) for c, v in values.items()}


class truncrank(_Strategy):
    """Keep the `howmany` first values after sorting all sectors together by `by` (descending
    when rev), counting each value dim(c) times (`truncation.jl:171-206`)."""

    def __init__(self, howmany, by=abs, rev=True):
        self.howmany, self.by, self.rev = int(howmany), by, rev

    def select(self, values: SectorVector):
        keys = list(values.keys())
        flat = np.concatenate([values[c].detach().cpu().numpy() for c in keys]) if keys else np.zeros(0)
        owner = np.concatenate([[i] * values[c].numel() for i, c in enumerate(keys)]).astype(int) \
            if keys else np.zeros(0, int)
        key = np.array([self.by(x) for x in flat], dtype=float)
        order = np.argsort(-key if self.rev else key, kind="stable")
        keep = np.zeros(flat.size, bool)
        unique = bool(keys) and keys[0].fusionstyle == "unique"  # no weights needed
        if unique:
            keep[order[:min(self.howmany, flat.size)]] = True
        else:
            total = 0
            for i in order:
                total += keys[owner[i]].dim()
                if total > self.howmany:
                    break
                keep[i] = True
        return _split(keep, keys, values)


class trunctol(_Strategy):
    """Keep, in every sector, the values with by(v) > atol', atol' = max(atol, rtol·norm(values,
    p)) when rtol ≠ 0 (`truncation.jl:213-222`, `rtol_to_atol` at `:155`)."""

    def __init__(self, atol=0.0, rtol=0.0, p=2, by=abs, keep_below=False):
        self.atol, self.rtol, self.p, self.by, self.keep_below = float(atol), float(rtol), p, by, keep_below

    def select(self, values: SectorVector):
        atol = self.atol if self.rtol == 0 else max(self.atol, values.norm(self.p) * self.rtol)
        out = {}
        for c, v in values.items():
            k = np.array([self.by(x) for x in v.detach().cpu().numpy()], dtype=float)
            out[c] = (k <= atol) if self.keep_below else (k > atol)
        return out


class truncerror(_Strategy):
    """Discard the smallest values (by |v|, all sectors together) while the accumulated
    Σ dim(c)·|v|^p stays ≤ max(atol^p, rtol^p·norm(values, p)) (`truncation.jl:228-262`)."""

    def __init__(self, atol=0.0, rtol=0.0, p=2):
        if not (math.isfinite(p) and p > 0):
            raise ValueError(f"p-norm with p = {p} is not supported")
        self.atol, self.rtol, self.p = float(atol), float(rtol), p

    def select(self, values: SectorVector):
        p = self.p
        emax = max(self.atol ** p, self.rtol ** p * values.norm(p))
        keys = list(values.keys())
        flat = np.concatenate([values[c].detach().cpu().numpy() for c in keys]) if keys else np.zeros(0)
        w = np.concatenate([[c.dim()] * values[c].numel() for c in keys]).astype(float) if keys else np.zeros(0)
        err = np.abs(flat) ** p * w
        keep = np.ones(flat.size, bool)
        total = 0.0
        for i in np.argsort(np.abs(flat), kind="stable"):
            total += err[i]
            if total > emax:
                break
            keep[i] = False
        return _split(keep, keys, values)


class truncspace(_Strategy):
    """Keep the dim(V, c) first values of every sector c, sorted by `by` (descending when rev)
    (`truncation.jl:264-273`)."""

    def __init__(self, V: GradedSpace, by=abs, rev=True):
        if V.isdual():
            raise ValueError("truncation space should not be dual")
        self.V, self.by, self.rev = V, by, rev

    def select(self, values: SectorVector):
        out = {}
        for c, v in values.items():
            k = np.array([self.by(x) for x in v.detach().cpu().numpy()], dtype=float)
            order = np.argsort(-k if self.rev else k, kind="stable")
            m = np.zeros(v.numel(), bool)
            m[order[:min(self.V.dim(c), v.numel())]] = True
            out[c] = m
        return out


class _Combine(_Strategy):
    """Intersection (&) or union (|) of the kept sets (`truncation.jl:279-300`)."""

    def __init__(self, a, b, how):
        self.a, self.b, self.how = a, b, how

    def select(self, values):
        ka, kb = self.a.select(values), self.b.select(values)
        op = np.logical_and if self.how == "and" else np.logical_or
        return {c: op(ka[c], kb[c]) for c in values}


def _split(keep, keys, values):
    out, off = {}, 0
    for c in keys:
        n = values[c].numel()
        out[c] = keep[off:off + n]
        off += n
    return out


def truncation_error(values: SectorVector, kept: dict, p=2) -> float:
    """Norm of the discarded values (`MAK.truncation_error!`, `truncation.jl:317-323`)."""
    import torch
    rest = SectorVector()
    for c, v in values.items():
        m = torch.as_tensor(~kept[c], device=v.device)
        rest[c] = v[m] if v.numel() else v
    return rest.norm(p)


def _apply(values, strategy):
    kept = (strategy or notrunc()).select(values)
    V = GradedSpace({c: int(m.sum()) for c, m in kept.items()}, unit=next(iter(values)).unit()) \
        if values else None
    return kept, V


def svd_trunc(t, trunc=None):
    """Truncated SVD: U, S, Vᴴ restricted to the kept singular values, and the truncation error
    (the weighted norm of the discarded values). Returns (U, S, Vᴴ, err)."""
    import torch
    t = _check(t)
    res = _svd_blocks(t)
    vals = SectorVector({c: s for c, (u, s, vh) in res.items()})
    kept, V = _apply(vals, trunc)
    if V is None:
        raise ValueError("tensor has no blocks")
    parts = {}
    for c, (u, s, vh) in res.items():
        m = torch.as_tensor(kept[c], device=s.device)
        parts[c] = (u[:, m], s[m], vh[m, :])
    U, S, Vh, _ = _assemble_svd(t, V, parts)
    return U, S, Vh, truncation_error(vals, kept)


# ---- QR / LQ -------------------------------------------------------------------------------
def qr_compact(t):
    """Q, R with t = Q·R per block, Q with orthonormal columns, R upper triangular."""
    import torch
    t = _check(t)
    u1 = t.space.unit()
    V = _infimum(_fuse(t.space.codomain), _fuse(t.space.domain))
    PV = ProductSpace((V,), u1)
    Q = _new(HomSpace(t.space.codomain, PV, u1), t)
    R = _new(HomSpace(PV, t.space.domain, u1), t)
    res = _batched({c: t.block(c) for c in t.blocksectors()}, lambda x: torch.linalg.qr(x, mode="reduced"))
    for c, (q, r) in res.items():
        Q.block(c).copy_(q)
        R.block(c).copy_(r)
    return Q, R


def lq_compact(t):
    """L, Q with t = L·Q per block, Q with orthonormal rows, L lower triangular (from the QR of
    the blocks' adjoints)."""
    import torch
    t = _check(t)
    u1 = t.space.unit()
    V = _infimum(_fuse(t.space.codomain), _fuse(t.space.domain))
    PV = ProductSpace((V,), u1)
    L = _new(HomSpace(t.space.codomain, PV, u1), t)
    Q = _new(HomSpace(PV, t.space.domain, u1), t)
    res = _batched({c: t.block(c).mH for c in t.blocksectors()}, lambda x: torch.linalg.qr(x, mode="reduced"))
    for c, (q, r) in res.items():
        L.block(c).copy_(r.mH)
        Q.block(c).copy_(q.mH)
    return L, Q


# ---- Hermitian eigendecomposition -----------------------------------------------------------
def _square(t):
    if t.space.codomain != t.space.domain:
        raise SpaceMismatch(f"eigh needs a square tensor map (codomain = domain): {t.space}")


def _eigh_blocks(t):
    import torch
    return _batched({c: t.block(c) for c in t.blocksectors()}, lambda x: torch.linalg.eigh(x))


def eigh_full(t):
    """D, V with t·V = V·D per block (t Hermitian), eigenvalues in increasing order."""
    t = _check(t)
    _square(t)
    res = _eigh_blocks(t)
    VD = _fuse(t.space.domain)
    vals = SectorVector({c: w for c, (w, v) in res.items()})
    return _assemble_eigh(t, VD, {c: (w, v) for c, (w, v) in res.items()}, vals)


def _assemble_eigh(t, VD, parts, vals):
    u1 = t.space.unit()
    V = _new(HomSpace(t.space.codomain, ProductSpace((VD,), u1), u1), t)
    for c, (w, v) in parts.items():
        if VD.dim(c):
            V.block(c).copy_(v)
    D = _diag(VD, SectorVector({c: w for c, (w, v) in parts.items() if VD.dim(c)}), t, _real_dtype(t))
    return D, V


def eigh_vals(t) -> SectorVector:
    import torch
    t = _check(t)
    _square(t)
    return SectorVector({c: torch.linalg.eigvalsh(t.block(c)) for c in t.blocksectors()})


def eigh_trunc(t, trunc=None):
    """Truncated Hermitian eigendecomposition: D, V restricted to the kept eigenvalues, and the
    truncation error. Returns (D, V, err)."""
    import torch
    t = _check(t)
    _square(t)
    res = _eigh_blocks(t)
    vals = SectorVector({c: w for c, (w, v) in res.items()})
    kept, VD = _apply(vals, trunc)
    parts = {}
    for c, (w, v) in res.items():
        m = torch.as_tensor(kept[c], device=w.device)
        parts[c] = (w[m], v[:, m])
    D, V = _assemble_eigh(t, VD, parts, vals)
    return D, V, truncation_error(vals, kept)
