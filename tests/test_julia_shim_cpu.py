"""The Julia drop-in written out in INTEGRATION.md, ported line by line to Python.

There is no Julia here, so the Julia shim itself cannot run. Its two pieces of host logic are
ported statement for statement and checked against the arrays the package's own C-ABI callers
produce:
- `flatten` of an AbelianTreeTransformer / GenericTreeTransformer (the data layout of
  src/tensors/treetransformers.jl:10-120) must give exactly `FlatTable`'s arrays;
- `gemm_descriptors` (the sector merge of src/tensors/linalg.jl:341-366) must give exactly
  `block_gemm_descriptors`' blocks, for plain and lazy-adjoint operands.
Julia's 1-based ranges appear here as the package's 0-based (start, stop) pairs, so
`first(r) - 1` becomes `r[0]`.
"""
import itertools

import numpy as np
import pytest
import torch

from helpers import O, VSU2, VU1, VU1SU2, cfg1_spaces, cfg2_spaces, five_leg, to_hom
import tensorkit_b200 as tk
from tensorkit_b200 import _lib as L
from tensorkit_b200.linalg import block_gemm_descriptors
from tensorkit_b200.structure import blockstructure
from tensorkit_b200.treetransformers import (AbelianTreeTransformer, flatten_transformer,
                                             treebraider)


# ---- port of INTEGRATION.md's Julia -------------------------------------------------------
def jl_perm0(p):
    flat = tuple(p[0]) + tuple(p[1])
    return [flat[k - 1] - 1 if k <= len(flat) else 0 for k in range(1, 9)]


def jl_flatten_abelian(tr, p):
    N = len(p[0]) + len(p[1])
    Lg = len(tr.data)
    gsrc = list(range(0, Lg + 1)); gdst = list(range(0, Lg + 1)); cptr = list(range(0, Lg + 1))
    coeffs = [None] * Lg
    sizes = np.empty((Lg, N), dtype=np.int64)       # Julia N×L column-major = L×N row-major
    sstr = np.empty((Lg, N), dtype=np.int64); soff = [None] * Lg
    dstr = np.empty((Lg, N), dtype=np.int64); doff = [None] * Lg
    for g, (coeff, (_, str_dst, off_dst), (sz_src, str_src, off_src)) in enumerate(tr.data):
        coeffs[g] = coeff
        sizes[g, :] = sz_src
        sstr[g, :] = str_src; soff[g] = off_src
        dstr[g, :] = str_dst; doff[g] = off_dst
    return dict(N=N, perm=jl_perm0(p), gsrc=gsrc, gdst=gdst, cptr=cptr, coeffs=coeffs, sizes=sizes,
                sstr=sstr, soff=soff, dstr=dstr, doff=doff)


def jl_flatten_generic(tr, p):
    N = len(p[0]) + len(p[1])
    gsrc = [0]; gdst = [0]; cptr = [0]; coeffs = []
    sizes = []; sstr = []; soff = []; dstr = []; doff = []
    for (U, (_, structs_dst), (sz_src, structs_src)) in tr.data:
        rows, cols = U.shape
        gsrc.append(gsrc[-1] + cols); gdst.append(gdst[-1] + rows); cptr.append(cptr[-1] + rows * cols)
        for i in range(1, rows + 1):
            for j in range(1, cols + 1):
                coeffs.append(U[i - 1, j - 1])
        sizes.extend(sz_src)
        for (st, off) in structs_src:
            sstr.extend(st); soff.append(off)
        for (st, off) in structs_dst:
            dstr.extend(st); doff.append(off)
    return dict(N=N, perm=jl_perm0(p), gsrc=gsrc, gdst=gdst, cptr=cptr, coeffs=coeffs, sizes=sizes,
                sstr=sstr, soff=soff, dstr=dstr, doff=doff)


def jl_flatten(tr, p):
    return jl_flatten_abelian(tr, p) if isinstance(tr, AbelianTreeTransformer) else jl_flatten_generic(tr, p)


def jl_operand_blocks(t):
    if isinstance(t, tk.AdjointTensorMap):
        P = t.parent
        op = 2 if P.is_complex() else 1
        return {c: (r[0], d2, d1, d1, op) for c, ((d1, d2), r) in blockstructure(P.space).items()}
    return {c: (r[0], d1, d2, d1, 0) for c, ((d1, d2), r) in blockstructure(t.space).items()}


def jl_gemm_descriptors(tC, tA, tB):
    A = jl_operand_blocks(tA); B = jl_operand_blocks(tB)
    out = []
    for c, ((d1, d2), r) in blockstructure(tC.space).items():
        if c in A and c in B:
            oa, _, ka, lda, opa = A[c]; ob, _, _, ldb, opb = B[c]
            out.append((d1, d2, ka, oa, ob, r[0], lda, ldb, d1, opa, opb))
        else:
            out.append((d1, d2, 0, 0, 0, r[0], 1, 1, d1, 0, 0))
    return out


# ---- checks ----------------------------------------------------------------------------------
def _same_table(tr, p):
    ref = flatten_transformer(tr, p)
    jl = jl_flatten(tr, p)
    N = jl["N"]
    assert N == ref.nind
    assert jl["perm"][:N] == [int(x) for x in ref.perm] and all(x == 0 for x in jl["perm"][N:])
    for key, arr in (("gsrc", ref.group_src_ptr), ("gdst", ref.group_dst_ptr), ("cptr", ref.coeff_ptr),
                     ("soff", ref.src_offsets), ("doff", ref.dst_offsets)):
        assert np.array_equal(np.asarray(jl[key], dtype=np.int64), arr), key
    assert np.array_equal(np.asarray(jl["coeffs"], dtype=np.float64), ref.coeffs)  # bitwise: same values
    for key, arr in (("sizes", ref.sizes), ("sstr", ref.src_strides), ("dstr", ref.dst_strides)):
        assert np.array_equal(np.asarray(jl[key], dtype=np.int64).reshape(-1), arr.reshape(-1)), key


def _tables(W, perms):
    Wp = to_hom(W)
    n = 0
    for p in perms:
        Vdst = Wp.permute(p)
        levels = (tuple(range(1, len(p[0]) + 1)), tuple(range(len(p[0]) + 1, len(p[0]) + len(p[1]) + 1)))
        tr = treebraider(Vdst, Wp, p, levels)
        _same_table(tr, p)
        n += 1
    return n


def test_flatten_workload_transformers():
    V, Pp = cfg1_spaces()
    assert _tables(O.Hom([V, Pp], [V]), [((1, 3), (2,)), ((3,), (1, 2)), ((2, 1), (3,))]) == 3
    V2, P2 = cfg2_spaces()
    assert _tables(O.Hom([V2, P2], [V2]), [((2, 3), (1,)), ((3,), (1, 2)), ((1,), (3, 2))]) == 3


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_flatten_five_leg_transformers(spaces):
    """five-leg spaces: SU(2) and U(1)⊠SU(2) give multi-tree fusion blocks (U larger than 1×1)"""
    W = five_leg(spaces())
    perms = list(itertools.permutations(range(1, 6)))[::23]
    ps = [(tuple(p[:k]), tuple(p[k:])) for k in (1, 2, 3) for p in perms]
    assert _tables(W, ps) == len(ps)


def _cpu_tensor(W, dtype=torch.float64):
    Wp = to_hom(W)
    n = tk.degeneracystructure(Wp).totaldim
    return tk.TensorMap(torch.zeros(n, dtype=dtype), Wp)


@pytest.mark.parametrize("dtype", [torch.float64, torch.complex128], ids=["f64", "c128"])
def test_gemm_descriptors_match(dtype):
    V, Pp = cfg2_spaces()
    A = _cpu_tensor(O.Hom([V, Pp], [V]), dtype)   # V⊗P ← V
    E = _cpu_tensor(O.Hom([V], [V]), dtype)       # V ← V
    C = _cpu_tensor(O.Hom([V, Pp], [V]), dtype)
    assert jl_gemm_descriptors(C, A, E) == block_gemm_descriptors(C, A, E)
    # lazy adjoint operand: A' is V ← V⊗P; A'·A is V ← V
    Ad = A.adjoint()
    C2 = _cpu_tensor(O.Hom([V], [V]), dtype)
    got = jl_gemm_descriptors(C2, Ad, A)
    assert got == block_gemm_descriptors(C2, Ad, A)
    assert all(d[9] == (L.TKB_OP_C if dtype == torch.complex128 else L.TKB_OP_T) for d in got if d[2] > 0)


def test_gemm_descriptors_missing_sectors():
    """sectors of C absent from A or B get k = 0 (the reference's rmul!(C, β))"""
    V = O.Space({O.U1(q): 2 for q in range(-2, 3)})
    Vs = O.Space({O.U1(q): 2 for q in range(-1, 2)})
    A = _cpu_tensor(O.Hom([V], [Vs]))
    B = _cpu_tensor(O.Hom([Vs], [V]))
    C = _cpu_tensor(O.Hom([V], [V]))
    got = jl_gemm_descriptors(C, A, B)
    assert got == block_gemm_descriptors(C, A, B)
    assert any(d[2] == 0 for d in got) and any(d[2] > 0 for d in got)
