"""Reverse-mode oracle — TEST INFRASTRUCTURE ONLY.

Restates, on the CPU block-sparse oracle (oracle/core.py), the ChainRules rule of
TO.tensorcontract! (ext/TensorKitChainRulesCoreExt/tensoroperations.jl:60-150) for α = 1,
β = 0 and bosonic sectors (trivial twists):
    dA = tensorcontract(ΔC, pΔC, conjA, B, reverse(pB), conjA ? conjB : !conjB, ipA)
    dB = tensorcontract(A, reverse(pA), conjB ? conjA : !conjA, ΔC, pΔC, conjB, ipB)
and applies it backwards through the pairwise contractions of an @tensor network. It is
checked itself against central finite differences in tests/test_gpu_ad.py.
"""
from __future__ import annotations

from . import core as O


def _adjidx(t: O.BT, i):
    n1, n2 = t.W.n1(), t.W.n2()
    return n2 + i if i <= n1 else i - n1


def tensorcontract(A, pA, conjA, B, pB, conjB, pAB):
    if conjA:
        pA = (tuple(_adjidx(A, i) for i in pA[0]), tuple(_adjidx(A, i) for i in pA[1]))
    if conjB:
        pB = (tuple(_adjidx(B, i) for i in pB[0]), tuple(_adjidx(B, i) for i in pB[1]))
    An = O.permute(A, pA, adjoint=conjA)
    Bn = O.permute(B, pB, adjoint=conjB)
    return O.permute(O.mul(An, Bn), pAB)


def _invperm(p):
    out = [0] * len(p)
    for i, x in enumerate(p):
        out[x - 1] = i + 1
    return tuple(out)


def _rep(p, n1):
    return (tuple(p[:n1]), tuple(p[n1:]))


def pullback(A, pA, conjA, B, pB, conjB, pAB, dC):
    ipAB = _invperm(tuple(pAB[0]) + tuple(pAB[1]))
    pdC = _rep(ipAB, len(pA[0]))
    ipA = _rep(_invperm(tuple(pA[0]) + tuple(pA[1])), A.W.n1())
    ipB = _rep(_invperm(tuple(pB[0]) + tuple(pB[1])), B.W.n1())
    rev = lambda p: (tuple(p[1]), tuple(p[0]))
    dA = tensorcontract(dC, pdC, conjA, B, rev(pB), conjB if conjA else (not conjB), ipA)
    dB = tensorcontract(A, rev(pA), conjA if conjB else (not conjA), dC, pdC, conjB, ipB)
    return dA, dB


def network_steps(factors, lhs):
    """Pairwise steps with the same index bookkeeping as the left-to-right @tensor lowering:
    intermediates are (open legs of the left operand ; open legs of the right operand)."""
    steps = []
    cur = list(factors[0][1])
    for k in range(1, len(factors)):
        lb = list(factors[k][1])
        con = [l for l in cur if l in lb]
        oa = [l for l in cur if l not in lb]
        ob = [l for l in lb if l not in cur]
        pA = (tuple(cur.index(l) + 1 for l in oa), tuple(cur.index(l) + 1 for l in con))
        pB = (tuple(lb.index(l) + 1 for l in con), tuple(lb.index(l) + 1 for l in ob))
        out = oa + ob
        if k == len(factors) - 1:
            pAB = (tuple(out.index(l) + 1 for l in lhs[0]), tuple(out.index(l) + 1 for l in lhs[1]))
            out = list(lhs[0]) + list(lhs[1])
        else:
            pAB = (tuple(range(1, len(oa) + 1)), tuple(range(len(oa) + 1, len(out) + 1)))
        steps.append((pA, pB, pAB))
        cur = out
    return steps


def network_grad(factors, lhs, tensors, dOut):
    steps = network_steps(factors, lhs)
    vals = [tensors[factors[0][0]]]
    for k, (pA, pB, pAB) in enumerate(steps):
        ca = factors[0][2] if k == 0 else False
        vals.append(tensorcontract(vals[-1], pA, ca, tensors[factors[k + 1][0]], pB, factors[k + 1][2], pAB))
    grads = {}

    def acc(name, g):
        grads[name] = g if name not in grads else O.BT(g.W, grads[name].data + g.data)

    d = dOut
    for k in range(len(steps) - 1, -1, -1):
        pA, pB, pAB = steps[k]
        ca = factors[0][2] if k == 0 else False
        dA, dB = pullback(vals[k], pA, ca, tensors[factors[k + 1][0]], pB, factors[k + 1][2], pAB, d)
        acc(factors[k + 1][0], dB)
        if k == 0:
            acc(factors[0][0], dA)
        d = dA
    return vals[-1], grads
