"""@tensor contractions of the workloads on the device vs the oracle.

Workloads (seeded synthetic tensors of the stated shapes):
 1. U(1) small:  C[a,p,q;b] := A[a,p;c]*B[c,q;b], then permute(C, (1,3), (2,4))
 2. SU(2) environment update: En[a;b] := conj(A[c,p;a])*E[c;d]*A[d,p;b]
 4. SU(2) large (degeneracies ×8), Float64 and ComplexF64, plain and split precision
Tolerance 1e-12 relative (max-norm), as the contraction test of the reference
(test/tensors/contractions.jl:78-92) compares against an independent evaluation."""
import numpy as np
import pytest

from helpers import O, cfg1_spaces, cfg2_spaces, relerr, to_device, to_hom
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_cfg1_u1_small():
    V, Pp = cfg1_spaces()
    W = O.Hom([V, Pp], [V])
    A, B = O.randn(W, 0), O.randn(W, 0)
    fac = [("A", ("a", "p", "c"), False), ("B", ("c", "q", "b"), False)]
    ref = O.network(fac, (("a", "p", "q"), ("b",)), {"A": A, "B": B})
    refp = O.permute(ref, ((1, 3), (2, 4)))
    Ad, Bd = to_device(A), to_device(B)
    C = tk.tensor("C[a,p,q;b] := A[a,p;c]*B[c,q;b]", A=Ad, B=Bd)
    assert C.space == to_hom(ref.W)
    assert relerr(C.to_host(), ref.data) <= TOL
    Cp = tk.permute(C, ((1, 3), (2, 4)))
    assert relerr(Cp.to_host(), refp.data) <= TOL


@pytest.mark.parametrize("prec", ["plain", "split"])
def test_u1_two_site_heff(prec):
    """y[a,p,q;b] := L[a,w;c]*x[c,r,s;d]*W1[w,p;r,v]*W2[v,q;s,u]*R[d,u;b] — many uneven
    blocks, tall-skinny GEMMs against the MPO bond, four pairwise steps; also replayed
    as a CUDA graph."""
    from helpers import cfg3_spaces
    V, Pp, Wm = cfg3_spaces()
    Wd = Wm.flipdual()
    tens = {"L": O.randn(O.Hom([V, Wd], [V]), 2), "x": O.randn(O.Hom([V, Pp, Pp], [V]), 2),
            "W1": O.randn(O.Hom([Wm, Pp], [Pp, Wm]), 2), "W2": O.randn(O.Hom([Wm, Pp], [Pp, Wm]), 2),
            "R": O.randn(O.Hom([V, Wm], [V]), 2)}
    expr = "y[a,p,q;b] := L[a,w;c]*x[c,r,s;d]*W1[w,p;r,v]*W2[v,q;s,u]*R[d,u;b]"
    from tensorkit_b200.tensoroperations import parse_tensor_expr
    _, lhs, _, factors = parse_tensor_expr(expr)
    ref = O.network(factors, lhs, tens)
    dev = {k: to_device(v) for k, v in tens.items()}
    plan = tk.NetworkPlan(expr, precision=prec, **dev).capture()
    y = plan.replay()
    plan.ctx.synchronize()
    assert y.space == to_hom(ref.W)
    assert relerr(y.to_host(), ref.data) <= TOL
    # a second replay after changing an input in place
    dev["x"].data.mul_(2.0)
    y = plan.replay()
    plan.ctx.synchronize()
    assert relerr(y.to_host(), 2.0 * ref.data) <= TOL
    plan.free()


@pytest.mark.parametrize("mult,prec,cplx", [(1, "plain", False), (1, "split", False),
                                            (8, "plain", False), (8, "split", False),
                                            (8, "plain", True), (8, "split", True)])
def test_env_update_su2(mult, prec, cplx):
    V, Pp = cfg2_spaces(mult)
    A = O.randn(O.Hom([V, Pp], [V]), 1 if mult == 1 else 3, cplx)
    E = O.randn(O.Hom([V], [V]), 1 if mult == 1 else 3, cplx)
    fac = [("A", ("c", "p", "a"), True), ("E", ("c", "d"), False), ("A", ("d", "p", "b"), False)]
    ref = O.network(fac, (("a",), ("b",)), {"A": A, "E": E})
    Ad, Ed = to_device(A), to_device(E)
    with tk.using_precision(prec):
        En = tk.tensor("En[a;b] := conj(A[c,p;a])*E[c;d]*A[d,p;b]", A=Ad, E=Ed)
    assert En.space == to_hom(ref.W)
    assert relerr(En.to_host(), ref.data) <= TOL


def test_auto_precision_su2_large(tmp_path, monkeypatch):
    """precision "auto" tunes each block structure once (precision × split-K decomposition,
    accuracy-checked against plain FP64) and keeps the fastest; the result meets the same bound and
    every GEMM plan records its choice."""
    V, Pp = cfg2_spaces(8)
    A = O.randn(O.Hom([V, Pp], [V]), 3)
    E = O.randn(O.Hom([V], [V]), 3)
    fac = [("A", ("c", "p", "a"), True), ("E", ("c", "d"), False), ("A", ("d", "p", "b"), False)]
    ref = O.network(fac, (("a",), ("b",)), {"A": A, "E": E})
    Ad, Ed = to_device(A), to_device(E)
    monkeypatch.setenv("TKB_TUNE_CACHE", str(tmp_path / "tune.json"))
    tk.get_context(0).empty_caches()
    with tk.using_precision("auto"):
        En = tk.tensor("En[a;b] := conj(A[c,p;a])*E[c;d]*A[d,p;b]", A=Ad, E=Ed)
    assert relerr(En.to_host(), ref.data) <= TOL
    ctx = tk.get_context(0)
    tuned = [p.tuned for k, p in ctx.plans.items() if k[0] == "gemm" and k[5] == "auto"]
    assert len(tuned) == 2 and all(t["choice"][0] in ("plain", "split") for t in tuned)
