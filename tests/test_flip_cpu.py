"""Host-side (no GPU): flip of tree pairs and spaces (`src/fusiontrees/braiding_manipulations.jl:388-436`,
`src/tensors/indexmanipulations.jl:21-29`). flip followed by flip(inv=True) is the identity, four flips
are the identity (flip is not an involution: a dual half-integer leg picks up χ = -1), and the flip
transformer maps every sub-block of the source onto a sub-block of the flipped space with a ±1 factor."""
import numpy as np
import pytest

from helpers import VSU2, VU1, VU1SU2, five_leg, to_hom
from tensorkit_b200 import fusiontrees as F
from tensorkit_b200.structure import sectorstructure
from tensorkit_b200.treetransformers import flatten_transformer, treeflipper


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_tree_flip_inverse_and_period_four(spaces):
    W = to_hom(five_leg(spaces(), ndom=2))
    for I in [(1,), (4,), (2, 5), (1, 3, 4)]:
        for pair in sectorstructure(W).fusiontrees:
            q, c = F.flip(pair, I)
            back, cb = F.flip(q, I, inv=True)
            assert back == pair and c * cb == 1.0
            r, acc = pair, 1.0
            for _ in range(4):
                r, cc = F.flip(r, I)
                acc *= cc
            assert r == pair and acc == 1.0


def test_tree_flip_factor_is_frobenius_schur_on_dual_half_integer_legs():
    from tensorkit_b200.sectors import SU2Irrep
    half, one = SU2Irrep(0.5), SU2Irrep(1)
    f1 = F.FusionTree((half, half), one, (True, False), ())
    f2 = F.FusionTree((one,), one, (False,), ())
    (g1, g2), c = F.flip((f1, f2), (1,))
    assert g1.isdual == (False, False) and c == -1.0   # dual spin-1/2 leg: χ = -1
    (g1, g2), c = F.flip((f1, f2), (2,))
    assert g1.isdual == (True, True) and c == 1.0      # non-dual leg: factor 1
    (g1, g2), c = F.flip((f1, f2), (3,))
    assert g2.isdual == (True,) and c == 1.0           # integer spin: χ = 1


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_flip_space_and_table(spaces):
    W = to_hom(five_leg(spaces(), ndom=2))
    n1, n = W.numout(), W.numind()
    p = (tuple(range(1, n1 + 1)), tuple(range(n1 + 1, n + 1)))
    for I in [(1,), (5,), (2, 4)]:
        Wf = W.flip(I)
        assert Wf.dims() == W.dims() and Wf.dim() == W.dim()
        assert Wf != W and Wf.flip(I) == W  # on spaces flip is an involution
        ft = flatten_transformer(treeflipper(Wf, W, I), p)
        assert set(np.unique(np.abs(ft.coeffs))) <= {0.0, 1.0}
        # every source element goes to exactly one destination element
        assert int(ft.group_src_ptr[-1]) == int(ft.group_dst_ptr[-1]) == len(sectorstructure(W).fusiontrees)
