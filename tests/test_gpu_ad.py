"""Differentiation through the device kernels (U(1)⊠SU(2) workload).

Loss f = real(tr(E_L·A·E_R·A†)), written as the @tensor network
    f[] := EL[a;c]*A[c,p;d]*ER[d;b]*conj(A[a,p;b])
with A ∈ V⊗P←V, E_L, E_R ∈ V←V, ComplexF64, seed 4 (V = U(1)⊠SU(2), q = -2..2, j = 0..3/2).
Gradients come from the rrule restatement (ext/TensorKitChainRulesCoreExt/
tensoroperations.jl:60-150) running the adjoint transforms (conj-flag source) and adjoint
grouped GEMMs (op C). Checked against
 - the oracle's own restatement of the rule on the CPU (1e-12 relative), and
 - central finite differences with step 1e-6 along random directions (1e-7 relative),
as test/chainrules/tensoroperations.jl:32-112 checks the reference's rules with FD."""
import numpy as np
import pytest
import torch

from helpers import O, cfg5_spaces, from_hom, relerr, to_device, to_hom
from oracle import ad as OA
import tensorkit_b200 as tk
from tensorkit_b200 import chainrules as CR
from tensorkit_b200.tensoroperations import parse_tensor_expr

pytestmark = pytest.mark.gpu
EXPR = "f[] := EL[a;c]*A[c,p;d]*ER[d;b]*conj(A[a,p;b])"


def _inputs():
    V, Pp = cfg5_spaces()
    return {"A": O.randn(O.Hom([V, Pp], [V]), 4, True),
            "EL": O.randn(O.Hom([V], [V]), 41, True),
            "ER": O.randn(O.Hom([V], [V]), 42, True)}


def _loss(dev):
    out = tk.tensor(EXPR, **dev)
    return float(out.data[0].real.item())


def _unit_cotangent(out):
    return tk.TensorMap(torch.ones(1, dtype=out.data.dtype, device=out.data.device), out.space)


@pytest.mark.parametrize("budget", [8 << 30, 0])
def test_gradients_match_oracle_rule(budget):
    tens = _inputs()
    dev = {k: to_device(v) for k, v in tens.items()}
    out, pb = CR.network_with_pullback(EXPR, memory_budget=budget, **dev)
    grads = pb(_unit_cotangent(out))
    _, lhs, _, factors = parse_tensor_expr(EXPR)
    dO = O.BT(from_hom(out.space), np.ones(1, dtype=complex))
    val, ograds = OA.network_grad(factors, lhs, tens, dO)
    assert abs(out.data[0].item() - val.data[0]) <= 1e-12 * abs(val.data[0])
    for k in ("A", "EL", "ER"):
        assert grads[k].space == to_hom(ograds[k].W)
        assert relerr(grads[k].to_host(), ograds[k].data) <= 1e-12, k


@pytest.mark.parametrize("name", ["A", "EL", "ER"])
def test_gradients_central_differences(name):
    tens = _inputs()
    dev = {k: to_device(v) for k, v in tens.items()}
    out, pb = CR.network_with_pullback(EXPR, **dev)
    g = pb(_unit_cotangent(out))[name]
    rng = np.random.default_rng(99)
    X = dev[name]
    n = X.data.numel()
    delta = torch.from_numpy((rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2)).to(X.data.device)
    eps = 1e-6
    base = X.data.clone()
    X.data.copy_(base + eps * delta)
    fp = _loss(dev)
    X.data.copy_(base - eps * delta)
    fm = _loss(dev)
    X.data.copy_(base)
    fd = (fp - fm) / (2 * eps)
    D = tk.TensorMap(delta, X.space)
    an = tk.inner(g, D).real
    assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (fd, an)


def test_permute_pullback_is_inverse_permute():
    V, Pp = cfg5_spaces()
    t = to_device(O.randn(O.Hom([V, Pp], [V]), 7, True))
    p = ((3,), (1, 2))
    out, pb = CR.rrule_permute(t, p, 0.5 + 0.25j)
    dC = to_device(O.randn(from_hom(out.space), 8, True))
    dA = pb(dC)
    # <dC, permute(t)> = <pullback(dC), t> (adjointness, with conj(α))
    lhs = tk.inner(dC, out)
    rhs = tk.inner(dA, t)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("p", [None, ((2, 3), (1,)), ((3,), (2, 1)), ((1,), (3, 2)), ((), (2, 1, 3)), ((3, 1, 2), ())])
def test_transpose_pullback_is_adjoint(p):
    """<dC, transpose(t, p)> = <pullback(dC), t> for cyclic p (the pullback transposes back)."""
    V, Pp = cfg5_spaces()
    t = to_device(O.randn(O.Hom([V, Pp], [V]), 9, True))
    out, pb = CR.rrule_transpose(t, p)
    dC = to_device(O.randn(from_hom(out.space), 10, True))
    dA = pb(dC)
    assert dA.space == t.space
    lhs = tk.inner(dC, out)
    rhs = tk.inner(dA, t)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("I", [(1,), (3,), (2, 3)])
def test_flip_pullback_is_adjoint(I):
    """<dC, flip(t, I)> = <pullback(dC), t> (the pullback flips back with inv toggled)."""
    V, Pp = cfg5_spaces()
    t = to_device(O.randn(O.Hom([V, Pp], [V]), 11, True))
    out, pb = CR.rrule_flip(t, I)
    dC = to_device(O.randn(from_hom(out.space), 12, True))
    dA = pb(dC)
    assert dA.space == t.space
    lhs = tk.inner(dC, out)
    rhs = tk.inner(dA, t)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_torch_autograd_bridge():
    V, Pp = cfg5_spaces()
    A = to_device(O.randn(O.Hom([V, Pp], [V]), 1, True))
    E = to_device(O.randn(O.Hom([V], [V]), 2, True))
    Fn = CR.TensorContract.make()
    a = A.data.clone().requires_grad_(True)
    e = E.data.clone().requires_grad_(True)
    pA, pB, pAB = ((1, 2), (3,)), ((1,), (2,)), ((1, 2), (3,))
    c = Fn.apply(a, e, A, pA, False, E, pB, False, pAB)
    w = torch.randn_like(c)
    loss = (c * w.conj()).real.sum()
    ga, ge = torch.autograd.grad(loss, (a, e))
    # the same cotangents from the rule, with ΔC = w
    C = tk.tensorcontract(A, pA, False, E, pB, False, pAB)
    _, pb = CR.rrule_tensorcontract(None, A, pA, False, E, pB, False, pAB)
    _, dA, dE, _, _ = pb(tk.TensorMap(w, C.space))
    assert relerr(ga.detach().cpu().numpy(), dA.to_host()) <= 1e-12
    assert relerr(ge.detach().cpu().numpy(), dE.to_host()) <= 1e-12
