"""Parity of the device tree transform (permute!/braid!/add_transform!) with the oracle.

Mirrors the reference's permutation tests (test/tensors/indexmanipulations.jl:55-99 and
test/cuda/tensors.jl:292-306): five-leg tensors over the reference's own U(1) and SU(2)
test spaces, every split k and a spread of permutations; real and complex data, α/β
accumulation and lazy-adjoint sources. Tolerance: 1e-12 relative (FP64)."""
import itertools

import numpy as np
import pytest

from helpers import O, VSU2, VU1, VU1SU2, five_leg, relerr, to_device, to_hom
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _perms(n, step):
    allp = list(itertools.permutations(range(1, n + 1)))
    return allp[::step]


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
@pytest.mark.parametrize("cplx", [False, True])
def test_permute_five_leg(spaces, cplx):
    W = five_leg(spaces())
    t = O.randn(W, 11, cplx)
    td = to_device(t)
    for k in range(6):
        for p in _perms(5, 7):
            p1, p2 = tuple(p[:k]), tuple(p[k:])
            ref = O.permute(t, (p1, p2))
            got = tk.permute(td, (p1, p2), copy=True)
            assert got.space == to_hom(ref.W)
            assert relerr(got.to_host(), ref.data) <= TOL, (k, p)


@pytest.mark.parametrize("spaces", [VU1, VSU2], ids=["U1", "SU2"])
def test_permute_alpha_beta(spaces):
    W = five_leg(spaces(), ndom=3)
    t = O.randn(W, 5, True)
    td = to_device(t)
    p = ((3, 1), (5, 2, 4))
    W2 = W.select(p)
    c = O.randn(W2, 6, True)
    cd = to_device(c)
    alpha, beta = 0.5 - 1.25j, 2.0 + 0.5j
    tk.permute_(cd, td, p, alpha, beta)
    ref = O.permute(t, p, alpha=alpha, tdst=c, beta=beta)
    assert relerr(cd.to_host(), ref.data) <= TOL


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_permute_adjoint_source(spaces):
    W = five_leg(spaces())
    t = O.randn(W, 7, True)
    td = to_device(t)
    adj = tk.AdjointTensorMap(td)
    for p in [((1, 2), (3, 4, 5)), ((5, 1), (2, 3, 4)), ((2, 4, 1, 3), (5,)), ((), (3, 1, 2, 5, 4))]:
        ref = O.permute(t, p, adjoint=True)
        got = tk.permute(adj, p, copy=True)
        assert got.space == to_hom(ref.W)
        assert relerr(got.to_host(), ref.data) <= TOL, p


def test_norm_dot_invariance():
    """norm and dot are invariant under every permutation (indexmanipulations.jl:55-75)."""
    W = five_leg(VSU2())
    t = to_device(O.randn(W, 1, True))
    t2 = to_device(O.randn(W, 2, True))
    n0 = tk.norm(t)
    d0 = tk.inner(t2, t)
    for k in (0, 2, 5):
        for p in _perms(5, 31):
            p1, p2 = tuple(p[:k]), tuple(p[k:])
            a = tk.permute(t, (p1, p2), copy=True)
            b = tk.permute(t2, (p1, p2), copy=True)
            assert abs(tk.norm(a) - n0) <= 1e-12 * n0
            assert abs(tk.inner(b, a) - d0) <= 1e-12 * abs(d0)


def test_permute_deterministic():
    W = five_leg(VSU2())
    td = to_device(O.randn(W, 3, False))
    p = ((4, 1), (2, 5, 3))
    a = tk.permute(td, p, copy=True).to_host()
    b = tk.permute(td, p, copy=True).to_host()
    assert np.array_equal(a, b)
