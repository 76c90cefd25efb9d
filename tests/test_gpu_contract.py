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
