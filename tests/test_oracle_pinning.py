"""Pins the oracle (no GPU) with the reference's own test identities — there are no golden
vectors in the reference, and Julia is unavailable here:
- permute commutes with dense conversion through Clebsch–Gordan fusion tensors
  (test/tensors/indexmanipulations.jl:77-99), for every split k of a five-leg tensor;
- dense round trip convert/project (src/tensors/abstracttensor.jl:733-792);
- contraction equals the dense contraction (test/tensors/contractions.jl:78-92);
- norm and dot are invariant under permutations (indexmanipulations.jl:55-75)."""
import itertools

import numpy as np
import pytest

from helpers import O, VSU2, VU1, VU1SU2, cfg2_spaces, five_leg
from oracle import dense as D


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_permute_via_dense(spaces):
    W = five_leg(spaces())
    t = O.randn(W, 123456, True)
    a = D.to_dense(t)
    assert np.abs(D.from_dense(W, a).data - t.data).max() < 1e-13
    assert abs(np.linalg.norm(a) - O.norm(t)) < 1e-12 * O.norm(t)
    perms = list(itertools.permutations(range(1, 6)))[::5]
    for k in range(6):
        for p in perms:
            p1, p2 = tuple(p[:k]), tuple(p[k:])
            ap = D.to_dense(O.permute(t, (p1, p2)))
            assert np.abs(ap - np.transpose(a, [x - 1 for x in p1 + p2])).max() < 1e-13


@pytest.mark.parametrize("spaces", [VU1, VSU2], ids=["U1", "SU2"])
def test_norm_dot_invariance(spaces):
    W = five_leg(spaces())
    t, t2 = O.randn(W, 1, True), O.randn(W, 2, True)
    n0, d0 = O.norm(t), O.inner(t2, t)
    for p in list(itertools.permutations(range(1, 6)))[::13]:
        for k in (1, 3):
            q = (tuple(p[:k]), tuple(p[k:]))
            assert abs(O.norm(O.permute(t, q)) - n0) < 1e-12 * n0
            assert abs(O.inner(O.permute(t2, q), O.permute(t, q)) - d0) < 1e-12 * abs(d0)


def test_contraction_via_dense_su2():
    V = O.Space({O.SU2(0): 2, O.SU2(0.5): 2, O.SU2(1): 1})
    Pp = O.Space({O.SU2(0.5): 1})
    A = O.randn(O.Hom([V, Pp], [V]), 1, True)
    E = O.randn(O.Hom([V], [V]), 2, True)
    fac = [("A", ("c", "p", "a"), True), ("E", ("c", "d"), False), ("A", ("d", "p", "b"), False)]
    En = O.network(fac, (("a",), ("b",)), {"A": A, "E": E})
    a, e = D.to_dense(A), D.to_dense(E)
    ref = np.einsum("cpa,cd,dpb->ab", np.conj(a), e, a)
    assert np.abs(D.to_dense(En) - ref).max() < 1e-12 * np.abs(ref).max()


def test_contraction_via_dense_u1_five_leg():
    VS = VU1()
    A = O.randn(O.Hom(VS[:3], [VS[3].flipdual()]), 3, True)
    B = O.randn(O.Hom([VS[3].flipdual()], [VS[4].flipdual()]), 4, True)
    fac = [("A", ("a", "b", "c", "d"), False), ("B", ("d", "e"), False)]
    C = O.network(fac, (("a", "e"), ("c", "b")), {"A": A, "B": B})
    ref = np.einsum("abcd,de->aecb", D.to_dense(A), D.to_dense(B))
    assert np.abs(D.to_dense(C) - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("spaces", [VU1, VSU2], ids=["U1", "SU2"])
def test_trace_via_dense(spaces):
    """t ∈ V1⊗V2'⊗V3⊗V2⊗V1'⊗V3', t2[a,b] := t[c,d,b,d,c,a] equals the dense partial trace
    (test/tensors/contractions.jl:60-67)."""
    V1, V2, V3 = spaces()[:3]
    W = O.Hom([V1, V2.flipdual(), V3, V2, V1.flipdual(), V3.flipdual()], [])
    t = O.randn(W, 7, True)
    t2 = O.trace_permute(t, ((6, 3), ()), ((1, 2), (5, 4)))
    ref = np.einsum("cdbdca->ab", D.to_dense(t))
    assert np.abs(D.to_dense(t2) - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_partial_trace_self_consistency(spaces):
    """t ∈ V1⊗V2⊗V3 ← V1⊗V2⊗V3: t2[a;b] := t[c d b; c d a] equals tracing twice through
    t4[a b; c d] := t[e d c; e b a], t5[a; b] := t4[a c; b c] (contractions.jl:46-53)."""
    V1, V2, V3 = spaces()[:3]
    t = O.randn(O.Hom([V1, V2, V3], [V1, V2, V3]), 8, True)
    # labels of t: (c, d, b ; c, d, a): legs 1..6
    t2 = O.trace_permute(t, ((6,), (3,)), ((1, 2), (4, 5)))
    t4 = O.trace_permute(t, ((6, 5), (3, 2)), ((1,), (4,)))
    t5 = O.trace_permute(t4, ((1,), (3,)), ((2,), (4,)))
    assert np.abs(t2.data - t5.data).max() < 1e-12 * np.abs(t2.data).max()
