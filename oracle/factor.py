"""Oracle (test infrastructure only): blockwise factorizations and TensorKit's truncation rules
in numpy, the checker for the device factorizations. Nothing in the library imports this.

Blocks are the coupled-sector matrices of `oracle.core` tensors; values are dicts sector →
numpy vector. The selection rules restate `src/factorizations/truncation.jl`:
- truncrank (TruncationByOrder, `:171-206`): sort all values by `by` (descending when rev);
  unique fusion keeps the first `howmany`, otherwise walk the sorted list adding dim(c) per
  value and stop before the sum exceeds `howmany`;
- trunctol (TruncationByValue, `:213-222`): atol' = max(atol, rtol·norm(values, p)) when
  rtol ≠ 0 (`rtol_to_atol`, `:155`), keep by(v) > atol' in every sector;
- truncerror (TruncationByError, `:228-262`): ϵᵖmax = max(atol^p, rtol^p·norm(values, p));
  walk the values by increasing |v|, adding dim(c)·|v|^p, discarding while the sum ≤ ϵᵖmax;
- truncspace (`:264-273`): keep the dim(V, c) largest in sector c;
- the truncation error is the dim-weighted norm of the discarded values (`:317-323`);
- norm(values, p) = (Σ_c dim(c) Σ|v|^p)^(1/p) (`src/tensors/linalg.jl:261-276`).
The per-block SVD/QR/eigh come from numpy's LAPACK (MatrixAlgebraKit's role in the reference).
"""
import numpy as np

from . import core as O


def blocks(t):
    return t.blocks()


def svd_vals(t):
    return {c: np.linalg.svd(b, compute_uv=False) for c, b in t.blocks().items()}


def eigh_vals(t):
    return {c: np.linalg.eigvalsh(b) for c, b in t.blocks().items()}


def vnorm(values, p=2):
    return sum(O.qdim(c) * float(np.sum(np.abs(v) ** p)) for c, v in values.items()) ** (1.0 / p)


def _flat(values):
    keys = list(values)
    flat = np.concatenate([values[c] for c in keys]) if keys else np.zeros(0)
    owner = np.concatenate([[i] * len(values[c]) for i, c in enumerate(keys)]).astype(int) if keys \
        else np.zeros(0, int)
    return keys, flat, owner


def _split(keep, keys, values):
    out, off = {}, 0
    for c in keys:
        out[c] = keep[off:off + len(values[c])]
        off += len(values[c])
    return out


def truncrank(values, howmany, unique):
    keys, flat, owner = _flat(values)
    order = np.argsort(-np.abs(flat), kind="stable")
    keep = np.zeros(flat.size, bool)
    if unique:
        keep[order[:min(howmany, flat.size)]] = True
    else:
        total = 0
        for i in order:
            total += O.qdim(keys[owner[i]])
            if total > howmany:
                break
            keep[i] = True
    return _split(keep, keys, values)


def trunctol(values, atol=0.0, rtol=0.0, p=2):
    a = atol if rtol == 0 else max(atol, vnorm(values, p) * rtol)
    return {c: np.abs(v) > a for c, v in values.items()}


def truncerror(values, atol=0.0, rtol=0.0, p=2):
    emax = max(atol ** p, rtol ** p * vnorm(values, p))
    keys, flat, owner = _flat(values)
    err = np.abs(flat) ** p * np.array([O.qdim(keys[o]) for o in owner], float)
    keep = np.ones(flat.size, bool)
    total = 0.0
    for i in np.argsort(np.abs(flat), kind="stable"):
        total += err[i]
        if total > emax:
            break
        keep[i] = False
    return _split(keep, keys, values)


def truncation_error(values, kept, p=2):
    return vnorm({c: v[~kept[c]] for c, v in values.items()}, p)
