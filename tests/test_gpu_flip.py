"""flip on the device (`src/tensors/indexmanipulations.jl:21-29`): one transform launch with the identity
permutation and the tree pairs' flip factors. Checked the way the reference's tests use it:
flip(flip(t, I), I; inv=true) == t, and flipping two legs that are then contracted with each other leaves
the contraction unchanged (half-integer SU(2) legs, where the factor is -1 on dual legs, included).
Tolerance: exact for the round trip (factors ±1), 1e-12 relative for the contraction."""
import pytest

from helpers import O, VSU2, VU1, VU1SU2, five_leg, relerr, to_device
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
@pytest.mark.parametrize("cplx", [False, True])
def test_flip_inverse_round_trip(spaces, cplx):
    W = five_leg(spaces(), ndom=2)
    t = O.randn(W, 41, cplx)
    td = to_device(t)
    for I in [(1,), (4,), (2, 5), (1, 3, 4)]:
        f = tk.flip(td, I)
        assert f.space == td.space.flip(I)
        back = tk.flip(f, I, inv=True)
        assert back.space == td.space
        assert relerr(back.to_host(), t.data) == 0.0, I


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
@pytest.mark.parametrize("xleg", [4, 3], ids=["x_plain", "x_dual"])
def test_flip_contracted_pair_leaves_contraction_unchanged(spaces, xleg):
    VS = spaces()
    V1, V3, X = VS[0], VS[2], VS[xleg]  # VS[3] is a dual space (spin 1/2 in SU(2): χ = -1)
    A = to_device(O.randn(O.Hom([V1, V3], [X]), 42, True))
    B = to_device(O.randn(O.Hom([X], [V3]), 43, True))
    C = tk.tensor("C[a,b;c] := A[a,b;x]*B[x;c]", A=A, B=B)
    # flip the contracted leg x on both sides: leg 3 of A (domain), leg 1 of B (codomain)
    Af, Bf = tk.flip(A, 3), tk.flip(B, 1)
    Cf = tk.tensor("C[a,b;c] := A[a,b;x]*B[x;c]", A=Af, B=Bf)
    assert Cf.space == C.space
    assert relerr(Cf.to_host(), C.to_host()) <= 1e-12
