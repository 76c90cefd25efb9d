"""Reverse-mode rules (ChainRules `rrule`s) on device tensors.

Restates `ext/TensorKitChainRulesCoreExt/tensoroperations.jl` and `src/pullbacks/*.jl`:
- `rrule_tensorcontract` (`tensoroperations.jl:60-150`):
    dA = tensorcontract(ΔC, pΔC, conjA, B, reverse(pB), conjA ? conjB : !conjB, ipA, conjA ? α : conj(α))
    dB = tensorcontract(A, reverse(pA), conjB ? conjA : !conjA, ΔC, pΔC, conjB, ipB, conjB ? α : conj(α))
    dα = ⟨A·B, ΔC⟩,  dβ = ⟨C, ΔC⟩,  dC = conj(β)·ΔC
  with ipAB = invperm(linearize(pAB)), pΔC = repartition(ipAB, length(pA[1])),
  ipA = repartition(invperm(linearize(pA)), numout(A)) (and likewise ipB). Twists are
  trivial for bosonic sectors.
- `rrule_tensoradd` (`:8-58`): dA = tensoradd(ΔC, pdA, conjA, conjA ? α : conj(α)).
- `rrule_tensortrace` (`:152-199`): dA = ΔC ⊗ id(traced legs), permuted back, times
  conj(α) (α when conjA).
- `rrule_permute` (`src/pullbacks/indexmanipulations.jl:1-31`, `ext/.../linalg.jl:62-70`):
  the inverse permutation with conj(α); `rrule_transpose` (`ext/.../linalg.jl:72-81`): the
  inverse cyclic permutation, through transpose! again; `rrule_flip`: flip with `inv` toggled.
- `rrule_tr`: Δ ↦ conj(Δ)·id;  `rrule_norm`: Δ ↦ (Δ/‖t‖)·t.

All adjoints run on the forward kernels: the transpose transform reads its source with the
conj flag (lazy adjoint), the adjoint GEMMs use op C/T. Complex cotangents follow the
ChainRules convention: for a real loss L, dL = Re⟨Δx, dx⟩.

`network_with_pullback(expr, **tensors)` differentiates a whole `@tensor` expression through
its pairwise contractions; the pairwise intermediates are kept for the backward pass while
their total size stays under `memory_budget` bytes (default 8 GB) and recomputed from the
inputs otherwise.
"""
from __future__ import annotations

from .indexmanipulations import permute, permute_
from .linalg import add_, inner, norm
from .tensor import AdjointTensorMap, TensorMap, new_tensor
from .tensoroperations import (_alloc, _pairwise_steps, parse_tensor_expr, tensoradd_,
                               tensoradd_structure, tensorcontract, tensorcontract_,
                               tensorcontract_structure)

__all__ = ["rrule_tensorcontract", "rrule_tensoradd", "rrule_tensortrace", "rrule_permute", "rrule_transpose",
           "rrule_flip", "rrule_tr",
           "rrule_norm",
           "network_with_pullback", "TensorContract"]


def _invperm(p):
    out = [0] * len(p)
    for i, x in enumerate(p):
        out[x - 1] = i + 1
    return tuple(out)


def _lin(p):
    return tuple(p[0]) + tuple(p[1])


def _rep(p, n1):
    return (tuple(p[:n1]), tuple(p[n1:]))


def _rev(p):
    return (tuple(p[1]), tuple(p[0]))


def _conj(x):
    return complex(x).conjugate() if isinstance(x, complex) else x


def rrule_tensorcontract(C, A, pA, conjA, B, pB, conjB, pAB, alpha=1.0, beta=0.0):
    """Returns (C′, pullback) with C′ = β·C + α·contract(A, B); pullback(ΔC) →
    (dC, dA, dB, dα, dβ)."""
    Cp = TensorMap(C.data.clone(), C.space) if C is not None else None
    if Cp is None:
        Cp = tensorcontract(A, pA, conjA, B, pB, conjB, pAB, alpha)
    else:
        tensorcontract_(Cp, A, pA, conjA, B, pB, conjB, pAB, alpha, beta)

    def pullback(dC_):
        ipAB = _invperm(_lin(pAB))
        pdC = _rep(ipAB, len(pA[0]))
        dC = None
        if beta != 0 and C is not None:
            dC = TensorMap(dC_.data.clone(), dC_.space)
            from .linalg import scale_
            scale_(dC, _conj(beta))
        ipA = _rep(_invperm(_lin(pA)), A.numout())
        conjBp = conjB if conjA else (not conjB)
        dA = tensorcontract(dC_, pdC, conjA, B, _rev(pB), conjBp, ipA,
                            alpha if conjA else _conj(alpha))
        ipB = _rep(_invperm(_lin(pB)), B.numout())
        conjAp = conjA if conjB else (not conjA)
        dB = tensorcontract(A, _rev(pA), conjAp, dC_, pdC, conjB, ipB,
                            alpha if conjB else _conj(alpha))
        AB = tensorcontract(A, pA, conjA, B, pB, conjB, pAB, 1.0)
        dalpha = inner(AB, dC_)
        dbeta = inner(C, dC_) if C is not None else 0.0
        return dC, dA, dB, dalpha, dbeta

    return Cp, pullback


def rrule_tensoradd(C, A, pA, conjA, alpha=1.0, beta=0.0):
    Cp = TensorMap(C.data.clone(), C.space)
    tensoradd_(Cp, A, pA, conjA, alpha, beta)

    def pullback(dC_):
        ipA = _invperm(_lin(pA))
        pdA = _rep(ipA, A.numout())
        dA = _alloc(tensoradd_structure(dC_, pdA, conjA), dC_)
        tensoradd_(dA, dC_, pdA, conjA, alpha if conjA else _conj(alpha), 0.0)
        dC = None
        if beta != 0:
            dC = TensorMap(dC_.data.clone(), dC_.space)
            from .linalg import scale_
            scale_(dC, _conj(beta))
        return dC, dA

    return Cp, pullback


def _identity(W, like):
    """one!(TensorMap of space W): identity blocks (W must be square)."""
    import torch
    from .structure import blockstructure
    out = TensorMap(torch.zeros(W.dim(), dtype=like.data.dtype, device=like.data.device), W)
    for c, ((d1, d2), (a, _)) in blockstructure(W).items():
        out.data[a:a + d1 * d2].view(d2, d1).diagonal().fill_(1.0)
    return out


def rrule_tensortrace(C, A, p, q, conjA=False, alpha=1.0, beta=0.0):
    """Returns (C′, pullback) with C′ = β·C + α·tensortrace(op(A), p, q); pullback(ΔC) →
    (dC, dA, dα, dβ) following `ext/TensorKitChainRulesCoreExt/tensoroperations.jl:152-199`:
    dA = tensorproduct(ΔC, (trivial(p); ()), conjA, E, ((); trivial(q)), conjA, pdA,
    conjA ? α : conj(α)) with E = one!(space of the traced legs) and
    pdA = repartition(invperm((linearize(p)..., q₁..., q₂...)), numout(A)); twists are
    trivial for bosonic sectors."""
    from .tensoroperations import tensortrace, tensortrace_
    Cp = TensorMap(C.data.clone(), C.space)
    tensortrace_(Cp, A, p, q, conjA, alpha, beta)

    def pullback(dC_):
        dC = None
        if beta != 0:
            dC = TensorMap(dC_.data.clone(), dC_.space)
            from .linalg import scale_
            scale_(dC, _conj(beta))
        ip = _invperm(_lin(p) + tuple(q[0]) + tuple(q[1]))
        pdA = _rep(ip, A.numout())
        E = _identity(tensoradd_structure(A, q, conjA), A)
        nq = len(q[0]) + len(q[1])
        np_ = len(p[0]) + len(p[1])
        pE = ((), tuple(range(1, nq + 1)))
        pdC = (tuple(range(1, np_ + 1)), ())
        dA = tensorcontract(dC_, pdC, conjA, E, pE, conjA, pdA, alpha if conjA else _conj(alpha))
        dalpha = inner(tensortrace(A, p, q, conjA), dC_)
        dbeta = inner(C, dC_)
        return dC, dA, dalpha, dbeta

    return Cp, pullback


def rrule_permute(t, p, alpha=1.0):
    out = permute(t, p, copy=True)
    if alpha != 1.0:
        from .linalg import scale_
        scale_(out, alpha)

    def pullback(dC):
        ip = _invperm(_lin(p))
        pdA = _rep(ip, t.numout())
        dA = new_tensor(dC.space.permute(pdA), dC.data.dtype, dC.data.device)
        permute_(dA, dC, pdA, _conj(alpha), 0.0)
        return dA

    return out, pullback


def rrule_transpose(t, p=None):
    """transpose(t, p) (a cyclic permutation; default (reverse(domain), reverse(codomain)))
    and its pullback: transpose of the cotangent by the inverse permutation, split like t
    (`ext/TensorKitChainRulesCoreExt/linalg.jl:72-81`)."""
    from .indexmanipulations import transpose, transpose_
    if p is None:
        p = (tuple(reversed(t.domainind())), tuple(reversed(t.codomainind())))
    p = (tuple(p[0]), tuple(p[1]))
    out = transpose(t, p, copy=True)

    def pullback(dC):
        pdA = _rep(_invperm(_lin(p)), t.numout())
        dA = new_tensor(dC.space.permute(pdA), dC.data.dtype, dC.data.device)
        transpose_(dA, dC, pdA, 1.0, 0.0)
        return dA

    return out, pullback


def rrule_flip(t, I, inv=False):
    """flip(t, I) and its pullback flip(Δ, I, inv = not inv): the flip is a ±1-signed map of
    sub-blocks, whose adjoint is its inverse (`ext/TensorKitChainRulesCoreExt/linalg.jl`, flip rule)."""
    from .indexmanipulations import flip
    out = flip(t, I, inv)

    def pullback(dC):
        return flip(dC, I, not inv)

    return out, pullback


def rrule_tr(t):
    from .linalg import tr
    val = tr(t)

    def pullback(d):
        import torch
        from .structure import blockstructure
        out = TensorMap(torch.zeros_like(t.data), t.space)
        for c, ((d1, d2), (a, _)) in blockstructure(t.space).items():
            blk = out.data[a:a + d1 * d2].view(d2, d1)
            blk.diagonal().fill_(_conj(d) if out.is_complex() else float(complex(d).real))
        return out

    return val, pullback


def rrule_norm(t):
    n = norm(t)

    def pullback(d):
        out = TensorMap(t.data.clone(), t.space)
        from .linalg import scale_
        scale_(out, float(complex(d).real) / n if n != 0 else 0.0)
        return out

    return n, pullback


def _nbytes(t):
    return t.data.numel() * t.data.element_size()


def network_with_pullback(expr, memory_budget=8 << 30, **tensors):
    """Forward value of an @tensor expression and a pullback ΔOut ↦ {name: gradient}.

    Gradients of a name that occurs several times (e.g. A and conj(A)) are summed."""
    lhs_name, lhs, op, factors = parse_tensor_expr(expr)
    if op != ":=":
        raise ValueError("differentiable networks use ':='")
    steps = _pairwise_steps(lhs, factors)

    def forward(keep):
        cur = tensors[factors[0][0]]
        saved = [cur]
        for i, (la, ca, lb, cb, pA, pB, pAB, outl, final) in enumerate(steps):
            B = tensors[factors[i + 1][0]]
            cur = tensorcontract(cur, pA, ca, B, pB, cb, pAB, 1.0)
            if keep or final:
                saved.append(cur)
        return cur, saved

    out, saved = forward(True)
    inter = sum(_nbytes(t) for t in saved[1:-1])
    if inter > memory_budget:
        saved = None  # recompute in the backward pass

    def pullback(dOut):
        nonlocal saved
        inputs = saved if saved is not None else forward(True)[1]
        grads = {}

        def acc(name, g):
            if name in grads:
                add_(grads[name], g, 1.0, 1.0)
            else:
                grads[name] = g

        d = dOut
        for i in range(len(steps) - 1, -1, -1):
            la, ca, lb, cb, pA, pB, pAB, outl, final = steps[i]
            A = inputs[i]
            B = tensors[factors[i + 1][0]]
            _, pb = _pullback_only(A, pA, ca, B, pB, cb, pAB)
            _, dA, dB, _, _ = pb(d)
            acc(factors[i + 1][0], dB)
            if i == 0:
                acc(factors[0][0], dA)
            d = dA
        if saved is None:
            del inputs
        return grads

    return out, pullback


def _pullback_only(A, pA, conjA, B, pB, conjB, pAB):
    """The pullback of tensorcontract without re-evaluating the forward product."""
    def pullback(dC_):
        ipAB = _invperm(_lin(pAB))
        pdC = _rep(ipAB, len(pA[0]))
        ipA = _rep(_invperm(_lin(pA)), A.numout())
        conjBp = conjB if conjA else (not conjB)
        dA = tensorcontract(dC_, pdC, conjA, B, _rev(pB), conjBp, ipA, 1.0)
        ipB = _rep(_invperm(_lin(pB)), B.numout())
        conjAp = conjA if conjB else (not conjA)
        dB = tensorcontract(A, _rev(pA), conjAp, dC_, pdC, conjB, ipB, 1.0)
        return None, dA, dB, None, None
    return None, pullback


class TensorContract:
    """torch.autograd.Function bridge: differentiate a pairwise contraction of TensorMaps
    through torch's autograd on their data vectors."""

    @staticmethod
    def make():
        import torch

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, a_data, b_data, A, pA, conjA, B, pB, conjB, pAB):
                Am = TensorMap(a_data, A.space)
                Bm = TensorMap(b_data, B.space)
                C = tensorcontract(Am, pA, conjA, Bm, pB, conjB, pAB, 1.0)
                ctx.meta = (Am, pA, conjA, Bm, pB, conjB, pAB, C.space)
                return C.data

            @staticmethod
            def backward(ctx, g):
                Am, pA, conjA, Bm, pB, conjB, pAB, WC = ctx.meta
                # torch and ChainRules share the cotangent convention for complex data:
                # for a real loss L, the gradient of z is ∂L/∂Re z + i·∂L/∂Im z
                dC = TensorMap(g.contiguous(), WC)
                _, pb = _pullback_only(Am, pA, conjA, Bm, pB, conjB, pAB)
                _, dA, dB, _, _ = pb(dC)
                return dA.data, dB.data, None, None, None, None, None, None, None

        return _Fn
