"""Parity of transpose! / repartition on the device with the oracle.

transpose!(tdst, tsrc, p) takes a cyclic (planar) permutation and moves the trees by folds, bends
and rotations only (`src/tensors/indexmanipulations.jl:378-391`, tables from
`treetransposer`); for these bosonic sectors the result equals permute!, which the oracle
computes. Five-leg tensors over the reference's U(1), SU(2) and U(1)⊠SU(2) test spaces, every
cyclic permutation for three splits, real and complex data, α/β accumulation and a lazy-adjoint
source. Tolerance: 1e-12 relative (FP64)."""
import pytest

from helpers import O, VSU2, VU1, VU1SU2, five_leg, relerr, to_device, to_hom
from test_fold_cpu import _cyclic_perms
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
@pytest.mark.parametrize("cplx", [False, True])
def test_transpose_five_leg(spaces, cplx):
    for nd in (1, 2, 3):
        W = five_leg(spaces(), ndom=nd)
        t = O.randn(W, 13 + nd, cplx)
        td = to_device(t)
        for p in _cyclic_perms(5 - nd, nd):
            ref = O.permute(t, p)
            got = tk.transpose(td, p)
            assert got.space == to_hom(ref.W)
            assert relerr(got.to_host(), ref.data) <= TOL, (nd, p)


@pytest.mark.parametrize("spaces", [VU1, VSU2], ids=["U1", "SU2"])
def test_transpose_default_and_repartition(spaces):
    W = five_leg(spaces(), ndom=2)
    t = O.randn(W, 21, False)
    td = to_device(t)
    # default: (reverse(domain), reverse(codomain))
    got = tk.transpose(td)
    ref = O.permute(t, ((5, 4), (3, 2, 1)))
    assert relerr(got.to_host(), ref.data) <= TOL
    # repartition keeps the cyclic order: codomain 1..N₁ of (1, 2, 3, 5, 4)
    for n1 in range(6):
        lin = [1, 2, 3, 5, 4]
        p = (tuple(lin[:n1]), tuple(reversed(lin[n1:])))
        got = tk.repartition(td, n1)
        ref = O.permute(t, p)
        assert got.space == to_hom(ref.W)
        assert relerr(got.to_host(), ref.data) <= TOL, n1


@pytest.mark.parametrize("spaces", [VU1, VSU2], ids=["U1", "SU2"])
def test_transpose_alpha_beta_and_adjoint_source(spaces):
    W = five_leg(spaces(), ndom=2)
    t = O.randn(W, 31, True)
    td = to_device(t)
    p = ((2, 3), (1, 4, 5))
    c = O.randn(W.select(p), 32, True)
    cd = to_device(c)
    alpha, beta = 0.75 + 0.5j, -1.5 + 0.25j
    tk.transpose_(cd, td, p, alpha, beta)
    ref = O.permute(t, p, alpha=alpha, tdst=c, beta=beta)
    assert relerr(cd.to_host(), ref.data) <= TOL
    adj = tk.AdjointTensorMap(td)
    for pa in _cyclic_perms(2, 3)[3::4]:
        got = tk.transpose(adj, pa)
        ref = O.permute(t, pa, adjoint=True)
        assert relerr(got.to_host(), ref.data) <= TOL, pa
