"""TensorOperations backend interface on device tensors, and the `@tensor` lowering.

Follows `src/tensors/tensoroperations.jl`:
- `tensoradd!` (`:44-62`): conj handled through the lazy adjoint and `adjointtensorindices`;
- `tensorcontract!` (`:130-161`) → `contract!` (`:318-357`), which evaluates the four index
  orders of `_contract_candidates` (`:360-376`) with `_contract_memcost` (`:378-383`) and
  calls `blas_contract!` (`:392-462`): permute A and B into (open; contracted) form unless
  they already are, blockwise `mul!`, permute C back unless it is a BLAS destination;
- `tensoradd_structure` / `tensorcontract_structure` (`:72-81`, `:174-182`).

Index tuples are 1-based (p = (p₁, p₂)), exactly as in TensorKit.

`tensor(expr, **tensors)` lowers an `@tensor` expression
(`"C[a,p,q;b] := A[a,p;c]*B[c,q;b]"`, factors optionally wrapped in `conj(...)`) into
pairwise `tensorcontract!` calls from left to right, as TensorOperations' `@tensor` does
without an explicit contraction order. Intermediates keep (open legs of the left operand ;
open legs of the right operand) as (codomain ; domain), which makes them BLAS
destinations of the blockwise `mul!`.
"""
from __future__ import annotations

import re

from .indexmanipulations import permute, permute_
from .linalg import mul_
from .spaces import HomSpace, SpaceMismatch
from .tensor import AdjointTensorMap, TensorMap, new_tensor

__all__ = ["tensoradd_", "tensorcontract_", "tensorcontract", "contract_", "blas_contract_",
           "tensortrace_", "tensortrace", "tensortrace_structure",
           "tensoradd_structure", "tensorcontract_structure", "tensor", "parse_tensor_expr",
           "adjointtensorindices"]


# ---- index helpers ------------------------------------------------------------------
def adjointtensorindex(t, i):
    return t.numin() + i if i <= t.numout() else i - t.numout()


def adjointtensorindices(t, p):
    if len(p) == 2 and isinstance(p[0], tuple):
        return (tuple(adjointtensorindex(t, i) for i in p[0]),
                tuple(adjointtensorindex(t, i) for i in p[1]))
    return tuple(adjointtensorindex(t, i) for i in p)


def _linearize(p):
    return tuple(p[0]) + tuple(p[1])


def _canonicalize(p, t):
    if len(p[0]) == t.numout() and len(p[1]) == t.numin():
        return (tuple(p[0]), tuple(p[1]))
    lin = _linearize(p)
    return (lin[:t.numout()], lin[t.numout():])


def _invperm(p):
    out = [0] * len(p)
    for i, x in enumerate(p):
        out[x - 1] = i + 1
    return tuple(out)


def _repartition(p, n1):
    return (tuple(p[:n1]), tuple(p[n1:]))


def _oindABinC(pAB, pA, pB):
    return _repartition(_invperm(_linearize(pAB)), len(pA[0]))


def _adjoint(t):
    return t.parent if isinstance(t, AdjointTensorMap) else AdjointTensorMap(t)


# ---- structures -----------------------------------------------------------------------
def tensoradd_structure(A, pA, conjA=False) -> HomSpace:
    if not conjA:
        return A.space.select(pA)
    return tensoradd_structure(_adjoint(A), adjointtensorindices(A, pA), False)


def tensorcontract_structure(A, pA, conjA, B, pB, conjB, pAB) -> HomSpace:
    sA = tensoradd_structure(A, pA, conjA)
    sB = tensoradd_structure(B, pB, conjB)
    return sA.compose(sB).permute(pAB)


# ---- tensoradd! -------------------------------------------------------------------------
def tensoradd_(C, A, pA, conjA, alpha=1.0, beta=0.0):
    if conjA:
        Ap = _adjoint(A)
        pAp = adjointtensorindices(A, _canonicalize(pA, C))
        return permute_(C, Ap, pAp, alpha, beta)
    return permute_(C, A, _canonicalize(pA, C), alpha, beta)


# ---- contraction --------------------------------------------------------------------------
def has_shared_permute(t, p):
    p = (tuple(p[0]), tuple(p[1]))
    if isinstance(t, AdjointTensorMap):
        q = (adjointtensorindices(t, p[1]), adjointtensorindices(t, p[0]))
        return has_shared_permute(t.parent, q)
    return p == (t.codomainind(), t.domainind())


def _isblas(t, p):
    return has_shared_permute(t, p)


def _contract_candidates(pA, pB, pAB):
    N1, N2 = len(pA[0]), len(pB[1])
    qA = sorted(range(len(pA[1])), key=lambda i: pA[1][i])
    pA1 = (pA[0], tuple(pA[1][i] for i in qA))
    pB1 = (tuple(pB[0][i] for i in qA), pB[1])
    qB = sorted(range(len(pB[0])), key=lambda i: pB[0][i])
    pA2 = (pA[0], tuple(pA[1][i] for i in qB))
    pB2 = (tuple(pB[0][i] for i in qB), pB[1])
    f = lambda n: n - N1 if n > N1 else n + N2
    pABp = (tuple(map(f, pAB[0])), tuple(map(f, pAB[1])))
    return pA1, pB1, pA2, pB2, pABp


def _memcost(dA, dB, dC, C, A, pA, B, pB, pAB):
    ipAB = _oindABinC(pAB, pA, pB)
    return (dA * (not _isblas(A, pA) or A.data.dtype != C.data.dtype)
            + dB * (not _isblas(B, pB) or B.data.dtype != C.data.dtype)
            + dC * (not _isblas(C, ipAB)))


def _dim(t):
    return t.space.dim() if not isinstance(t, AdjointTensorMap) else t.parent.space.dim()


def contract_(C, A, pA, B, pB, pAB, alpha=1.0, beta=0.0):
    if len(pA[1]) != len(pB[0]):
        raise IndexError("number of contracted indices does not match")
    pA1, pB1, pA2, pB2, pABp = _contract_candidates(pA, pB, pAB)
    dA, dB, dC = _dim(A), _dim(B), _dim(C)
    m1 = _memcost(dA, dB, dC, C, A, pA1, B, pB1, pAB)
    m2 = _memcost(dA, dB, dC, C, A, pA2, B, pB2, pAB)
    rv = lambda p: (p[1], p[0])
    m3 = _memcost(dB, dA, dC, C, B, rv(pB1), A, rv(pA1), pABp)
    m4 = _memcost(dB, dA, dC, C, B, rv(pB2), A, rv(pA2), pABp)
    if min(m1, m2) <= min(m3, m4):
        if m1 <= m2:
            return blas_contract_(C, A, pA1, B, pB1, pAB, alpha, beta)
        return blas_contract_(C, A, pA2, B, pB2, pAB, alpha, beta)
    if m3 <= m4:
        return blas_contract_(C, B, rv(pB1), A, rv(pA1), pABp, alpha, beta)
    return blas_contract_(C, B, rv(pB2), A, rv(pA2), pABp, alpha, beta)


def _alloc(W, like):
    return new_tensor(W, like.data.dtype, like.data.device)


def blas_contract_(C, A, pA, B, pB, pAB, alpha=1.0, beta=0.0, plan_hook=None):
    copyA = not (_isblas(A, pA) and A.data.dtype == C.data.dtype)
    if copyA:
        Anew = _alloc(tensoradd_structure(A, pA, False), C)
        tensoradd_(Anew, A, pA, False, 1.0, 0.0)
    else:
        Anew = permute(A, pA)
    copyB = not (_isblas(B, pB) and B.data.dtype == C.data.dtype)
    if copyB:
        Bnew = _alloc(tensoradd_structure(B, pB, False), C)
        tensoradd_(Bnew, B, pB, False, 1.0, 0.0)
    else:
        Bnew = permute(B, pB)
    pAnew = (Anew.codomainind(), Anew.domainind())
    pBnew = (Bnew.codomainind(), Bnew.domainind())
    ipAB = _oindABinC(pAB, pAnew, pBnew)
    if not _isblas(C, ipAB):
        Cnew = _alloc(tensoradd_structure(C, ipAB, False), C)
        mul_(Cnew, Anew, Bnew, 1.0, 0.0)
        tensoradd_(C, Cnew, pAB, False, alpha, beta)
    else:
        Cnew = permute(C, ipAB)
        mul_(Cnew, Anew, Bnew, alpha, beta)
    return C


def tensorcontract_(C, A, pA, conjA, B, pB, conjB, pAB, alpha=1.0, beta=0.0):
    pA = (tuple(pA[0]), tuple(pA[1]))
    pB = (tuple(pB[0]), tuple(pB[1]))
    pABc = _canonicalize(pAB, C)
    W = tensorcontract_structure(A, pA, conjA, B, pB, conjB, pABc)
    if W != C.space:
        raise SpaceMismatch(f"incompatible spaces for tensorcontract: {W} ≠ {C.space}")
    if conjA:
        A, pA = _adjoint(A), adjointtensorindices(A, pA)
    if conjB:
        B, pB = _adjoint(B), adjointtensorindices(B, pB)
    return contract_(C, A, pA, B, pB, pABc, alpha, beta)


def tensorcontract(A, pA, conjA, B, pB, conjB, pAB, alpha=1.0):
    W = tensorcontract_structure(A, pA, conjA, B, pB, conjB, pAB)
    C = _alloc(W, A)
    return tensorcontract_(C, A, pA, conjA, B, pB, conjB, pAB, alpha, 0.0)


# ---- @tensor -------------------------------------------------------------------------------
_TERM = re.compile(r"\s*(conj\()?\s*([A-Za-z_][A-Za-z_0-9′']*)\s*\[([^\]]*)\]\s*(\))?\s*")


def _labels(s):
    if ";" in s:
        a, b = s.split(";", 1)
    else:
        a, b = s, ""
    sp = lambda x: tuple(y.strip() for y in x.split(",") if y.strip())
    return sp(a), sp(b)


def parse_tensor_expr(expr):
    """Parse 'C[a;b] := A[a;c]*conj(B[c;b])' → (lhs_name, (cod, dom), op, [(name, labels, conj)])."""
    for op in (":=", "+=", "="):
        if op in expr:
            lhs, rhs = expr.split(op, 1)
            break
    else:
        raise ValueError("expression needs :=, = or +=")
    m = _TERM.fullmatch(lhs)
    if not m:
        raise ValueError(f"cannot parse left-hand side {lhs!r}")
    lhs_name = m.group(2)
    lcod, ldom = _labels(m.group(3))
    factors = []
    for part in rhs.split("*"):
        mm = _TERM.fullmatch(part)
        if not mm:
            raise ValueError(f"cannot parse factor {part!r}")
        conj = mm.group(1) is not None
        if conj != (mm.group(4) is not None):
            raise ValueError(f"unbalanced conj in {part!r}")
        c, d = _labels(mm.group(3))
        factors.append((mm.group(2), c + d, conj))
    return lhs_name, (lcod, ldom), op, factors


def tensortrace_structure(A, p, conjA=False) -> HomSpace:
    """Space of the traced result: select(space(op(A)), p), the structure of tensoradd!
    (`src/tensors/tensoroperations.jl:72-81`, also used when indices are traced)."""
    return tensoradd_structure(A, p, conjA)


def tensortrace_(C, A, p, q, conjA=False, alpha=1.0, beta=0.0):
    """TO.tensortrace!(C, A, p, q, conjA, α, β) (`src/tensors/tensoroperations.jl:83-98`):
    conj(A) through the lazy adjoint with `adjointtensorindices`, then `trace_permute!`."""
    from .trace import trace_permute_
    if conjA:
        Ap = _adjoint(A)
        p2 = adjointtensorindices(A, _canonicalize(p, C))
        q2 = adjointtensorindices(A, q)
        return trace_permute_(C, Ap, p2, q2, alpha, beta)
    return trace_permute_(C, A, _canonicalize(p, C), q, alpha, beta)


def tensortrace(A, p, q, conjA=False, alpha=1.0):
    """New tensor α·tensortrace(op(A), p, q)."""
    C = _alloc(tensortrace_structure(A, p, conjA), A)
    return tensortrace_(C, A, p, q, conjA, alpha, 0.0)


def _pairwise_steps(lhs, factors):
    """Plan of pairwise contractions: list of (labelsA, conjA, labelsB, conjB, pA, pB, pAB,
    out_labels, is_final)."""
    steps = []
    cur_labels, cur_conj = factors[0][1], factors[0][2]
    n = len(factors)
    for idx in range(1, n):
        lb, cb = factors[idx][1], factors[idx][2]
        for lab in set(cur_labels):
            if cur_labels.count(lab) > 1:
                raise NotImplementedError("traces inside @tensor are not supported")
        contracted = [l for l in cur_labels if l in lb]
        openA = [l for l in cur_labels if l not in lb]
        openB = [l for l in lb if l not in cur_labels]
        pA = (tuple(cur_labels.index(l) + 1 for l in openA), tuple(cur_labels.index(l) + 1 for l in contracted))
        pB = (tuple(lb.index(l) + 1 for l in contracted), tuple(lb.index(l) + 1 for l in openB))
        out = openA + openB
        final = idx == n - 1
        if final:
            lcod, ldom = lhs
            if sorted(lcod + ldom) != sorted(out):
                raise ValueError(f"left-hand side labels {lcod + ldom} ≠ open labels {out}")
            pAB = (tuple(out.index(l) + 1 for l in lcod), tuple(out.index(l) + 1 for l in ldom))
        else:
            pAB = (tuple(range(1, len(openA) + 1)), tuple(range(len(openA) + 1, len(out) + 1)))
        steps.append((cur_labels, cur_conj, lb, cb, pA, pB, pAB, tuple(out), final))
        cur_labels, cur_conj = tuple(out), False
    return steps


def _trace_labels(labels):
    """Leg pairs (q₁, q₂) of the labels repeated within one factor (1-based)."""
    reps = [l for l in dict.fromkeys(labels) if labels.count(l) > 1]
    for l in reps:
        if labels.count(l) > 2:
            raise ValueError(f"label {l!r} appears more than twice in one factor")
    q1 = tuple(labels.index(l) + 1 for l in reps)
    q2 = tuple(len(labels) - labels[::-1].index(l) for l in reps)
    return reps, (q1, q2)


def _pretrace(A, labels, conj):
    """Trace the labels a factor repeats (TensorOperations traces a factor before it enters
    a contraction); returns the traced tensor and its remaining labels."""
    reps, q = _trace_labels(labels)
    if not reps:
        return A, tuple(labels), conj
    nout = A.numout()
    keep = [i for i, l in enumerate(labels) if l not in reps]
    p = (tuple(i + 1 for i in keep if i < nout), tuple(i + 1 for i in keep if i >= nout))
    return tensortrace(A, p, q, conj), tuple(labels[i] for i in keep), False


def tensor(expr, out=None, alpha=1.0, **tensors):
    """Evaluate an @tensor expression on device TensorMaps.

    `:=` allocates the result; `=` writes into `out` (β = 0); `+=` accumulates (β = 1).
    Labels repeated within one factor are traced (`tensortrace!`)."""
    lhs_name, lhs, op, factors = parse_tensor_expr(expr)
    if len(factors) == 1:
        name, labels, conj = factors[0]
        A = tensors[name]
        lcod, ldom = lhs
        pA = (tuple(labels.index(l) + 1 for l in lcod), tuple(labels.index(l) + 1 for l in ldom))
        beta = 1.0 if op == "+=" else 0.0
        reps, q = _trace_labels(labels)
        if out is None:
            out = _alloc(tensoradd_structure(A, pA, conj), A)
        if reps:
            return tensortrace_(out, A, pA, q, conj, alpha, beta)
        return tensoradd_(out, A, pA, conj, alpha, beta)
    pre = [_pretrace(tensors[n], lab, cj) for n, lab, cj in factors]
    factors = [(n, lab, cj) for (n, _, _), (_, lab, cj) in zip(factors, pre)]
    steps = _pairwise_steps(lhs, factors)
    cur = pre[0][0]
    for i, (la, ca, lb, cb, pA, pB, pAB, outl, final) in enumerate(steps):
        B = pre[i + 1][0]
        if final:
            W = tensorcontract_structure(cur, pA, ca, B, pB, cb, pAB)
            if out is None:
                if op != ":=":
                    raise ValueError("'=' and '+=' need an existing output tensor")
                out = _alloc(W, cur)
                beta = 0.0
            else:
                beta = 1.0 if op == "+=" else 0.0
            tensorcontract_(out, cur, pA, ca, B, pB, cb, pAB, alpha, beta)
            return out
        cur = tensorcontract(cur, pA, ca, B, pB, cb, pAB, 1.0)
    raise AssertionError("unreachable")
