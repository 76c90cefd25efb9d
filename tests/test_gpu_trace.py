"""Partial traces on the device (tkb_tracetransform) vs the oracle, on the cases of the
reference's trace tests (test/tensors/contractions.jl:17-67): trace_permute! with α and β,
the conjA path of TO.tensortrace! (lazy adjoint source), traces inside @tensor, and the
tensortrace! rrule against central differences."""
import numpy as np
import pytest

from helpers import O, VSU2, VU1, VU1SU2, relerr, to_device, to_hom
from test_trace_cpu import cases
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu
TOL = 1e-12
SPACES = [VU1, VSU2, VU1SU2]
IDS = ["U1", "SU2", "U1xSU2"]


@pytest.mark.parametrize("spaces", SPACES, ids=IDS)
def test_trace_permute_alpha_beta(spaces):
    V1, V2, V3 = spaces()[:3]
    for k, (W, p, q) in enumerate(cases(V1, V2, V3)):
        t = O.randn(W, 60 + k, True)
        d0 = O.randn(W.select(p), 70 + k, True)
        alpha, beta = 0.7 - 0.2j, -1.3 + 0.5j
        ref = O.trace_permute(t, p, q, alpha, tdst=d0, beta=beta)
        tdst = to_device(d0)
        tk.trace_permute_(tdst, to_device(t), p, q, alpha, beta)
        assert tdst.space == to_hom(ref.W)
        assert relerr(tdst.to_host(), ref.data) <= TOL, (k, p, q)


@pytest.mark.parametrize("spaces", SPACES, ids=IDS)
def test_tensortrace_conj(spaces):
    """tensortrace!(C, A, p, q, conjA = true): p and q index A, the trace reads conj(A)."""
    V1, V2, V3 = spaces()[:3]
    W = O.Hom([V1, V2], [V1, V3])
    A = O.randn(W, 81, True)
    p, q = ((2,), (4,)), ((1,), (3,))
    n1, n2 = W.n1(), W.n2()
    adj = lambda i: n2 + i if i <= n1 else i - n1
    Aadj = O.permute(A, (tuple(range(1, n2 + 1)), tuple(range(n2 + 1, n1 + n2 + 1))), adjoint=True)
    pa = (tuple(adj(i) for i in p[0]), tuple(adj(i) for i in p[1]))
    qa = (tuple(adj(i) for i in q[0]), tuple(adj(i) for i in q[1]))
    ref = O.trace_permute(Aadj, pa, qa)
    C = tk.tensortrace(to_device(A), p, q, True)
    assert C.space == to_hom(ref.W)
    assert relerr(C.to_host(), ref.data) <= TOL


@pytest.mark.parametrize("spaces", [VU1, VSU2], ids=["U1", "SU2"])
def test_trace_in_tensor_expressions(spaces):
    """t2[a,b] := t[c,d,b,d,c,a] (contractions.jl:61-66), and a traced factor inside a
    contraction: y[a;b] := A[a,c;d,c]*E[d;b]."""
    V1, V2, V3 = spaces()[:3]
    d = lambda v: v.flipdual()
    W = O.Hom([V1, d(V2), V3, V2, d(V1), d(V3)], [])
    t = O.randn(W, 91, True)
    ref = O.trace_permute(t, ((6, 3), ()), ((1, 2), (5, 4)))
    t2 = tk.tensor("t2[a,b] := t[c,d,b,d,c,a]", t=to_device(t))
    assert relerr(t2.to_host(), ref.data) <= TOL
    A = O.randn(O.Hom([V1, V2], [V3, V2]), 92, True)
    E = O.randn(O.Hom([V3], [V1]), 93, True)
    At = O.trace_permute(A, ((1,), (3,)), ((2,), (4,)))
    ref2 = O.network([("At", ("a", "d"), False), ("E", ("d", "b"), False)], (("a",), ("b",)),
                     {"At": At, "E": E})
    y = tk.tensor("y[a;b] := A[a,c;d,c]*E[d;b]", A=to_device(A), E=to_device(E))
    assert y.space == to_hom(ref2.W)
    assert relerr(y.to_host(), ref2.data) <= TOL


@pytest.mark.parametrize("spaces", SPACES, ids=IDS)
@pytest.mark.parametrize("conjA", [False, True])
def test_tensortrace_rrule_central_differences(spaces, conjA):
    """The tensortrace! rrule (ext/TensorKitChainRulesCoreExt/tensoroperations.jl:152-199)
    against central differences of L(A) = Re⟨W, β·C + α·tensortrace(op(A), p, q)⟩ (step
    1e-6), as test/chainrules/tensoroperations.jl:32-49 checks the reference's rule."""
    import torch
    from helpers import from_hom
    from tensorkit_b200 import chainrules as CR
    V1, V2, V3 = spaces()[:3]
    W = O.Hom([V1, V2], [V1, V3])
    p, q = ((2,), (4,)), ((1,), (3,))
    A = to_device(O.randn(W, 101, True))
    C0 = tk.tensortrace(A, p, q, conjA)
    Wc = to_device(O.randn(from_hom(C0.space), 102, True))
    alpha, beta = 0.8 + 0.3j, 0.5 - 0.2j
    _, pb = CR.rrule_tensortrace(C0, A, p, q, conjA, alpha, beta)
    dC, dA, dalpha, dbeta = pb(Wc)
    rng = np.random.default_rng(7)
    n = A.data.numel()
    D = torch.from_numpy((rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2)).to(A.data.device)

    def L(x):
        X = tk.TensorMap(x, A.space)
        out = tk.TensorMap(C0.data.clone(), C0.space)
        tk.tensortrace_(out, X, p, q, conjA, alpha, beta)
        return tk.inner(Wc, out).real

    eps = 1e-6
    fd = (L(A.data + eps * D) - L(A.data - eps * D)) / (2 * eps)
    an = tk.inner(dA, tk.TensorMap(D, A.space)).real
    assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (fd, an)
    assert dC is not None and relerr(dC.to_host(), (np.conj(beta) * Wc.data).cpu().numpy()) <= TOL
