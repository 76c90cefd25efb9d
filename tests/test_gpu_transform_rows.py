"""The row-copy transform kernel against the staged kernels and the oracle.

Tables whose groups all keep their fastest leg in place (every abelian permute that leaves
the leading leg first, test/tensors/indexmanipulations.jl:55-99 in the reference) run as exact
row tiles. The same call through the staged ring (TKB_TRANSFORM_KERNEL=pipe) and the plain
kernel (=plain) does the same arithmetic per element, α·(u·v) + β·d, so the results must agree
bit for bit; the oracle checks them to 1e-12 (FP64). Cases: rows longer than one tile (split
into chunks), sub-blocks of one element (scalar rows), α/β accumulation, complex data and a
lazy-adjoint source (conjugating loads), a few small transpose groups among the row groups, and
a permute that moves the leading leg (transpose groups throughout, which keep the staged kernel)."""
import numpy as np
import pytest
import torch

from helpers import O, U1, relerr, to_device, to_hom
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu
TOL = 1e-12
KERNELS = ("", "pipe", "plain")


def _long_rows():
    V = O.Space({U1(0): 2600, U1(1): 37, U1(-1): 300, U1(2): 1})
    Pp = O.Space({U1(0): 1, U1(1): 1})
    return O.Hom([V, Pp, Pp], [V])


def _mixed_transpose():
    # sub-blocks whose leading sector has dimension 1 lose that leg, and a permute that keeps leg
    # 1 first but swaps legs 2 and 3 turns them into transpose groups: 30 of 76 030 elements, so
    # the table still runs as row tiles with those few groups read uncoalesced
    V = O.Space({U1(0): 2000, U1(1): 1})
    V2 = O.Space({U1(0): 4, U1(1): 3})
    V3 = O.Space({U1(0): 5, U1(1): 6, U1(2): 2})
    return O.Hom([V, V2], [V3])


def _scalar_blocks():
    Pp = O.Space({U1(0): 1, U1(1): 1, U1(-1): 1})
    return O.Hom([Pp, Pp, Pp], [Pp, Pp])


def _run(monkeypatch, kernel, fn):
    if kernel:
        monkeypatch.setenv("TKB_TRANSFORM_KERNEL", kernel)
    else:
        monkeypatch.delenv("TKB_TRANSFORM_KERNEL", raising=False)
    out = fn()
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("make,perms", [
    (_long_rows, [((1, 3), (2, 4)), ((1,), (4, 2, 3)), ((1, 4, 2), (3,)), ((4, 1), (2, 3))]),
    (_scalar_blocks, [((1, 3, 2), (5, 4)), ((1,), (2, 3, 4, 5)), ((3, 1, 2, 5), (4,))]),
    (_mixed_transpose, [((1, 3), (2,)), ((1,), (3, 2)), ((3, 1), (2,))]),
], ids=["long_rows", "scalar_blocks", "mixed_transpose"])
@pytest.mark.parametrize("cplx", [False, True])
def test_rows_kernel_bitwise_and_oracle(monkeypatch, make, perms, cplx):
    W = make()
    t = O.randn(W, 21, cplx)
    td = to_device(t)
    for p in perms:
        ref = O.permute(t, p)
        outs = [_run(monkeypatch, k, lambda: tk.permute(td, p, copy=True)) for k in KERNELS]
        assert outs[0].space == to_hom(ref.W)
        for o in outs[1:]:
            assert torch.equal(outs[0].data, o.data), p
        assert relerr(outs[0].to_host(), ref.data) <= TOL, p


def test_rows_kernel_alpha_beta_adjoint(monkeypatch):
    W = _long_rows()
    t = O.randn(W, 22, True)
    td = to_device(t)
    p = ((1, 3), (2, 4))
    c = O.randn(W.select(p), 23, True)
    alpha, beta = 0.75 - 0.5j, -1.5 + 0.25j
    results = []
    for k in KERNELS:
        cd = to_device(c)
        _run(monkeypatch, k, lambda: tk.permute_(cd, td, p, alpha, beta))
        results.append(cd)
    for o in results[1:]:
        assert torch.equal(results[0].data, o.data)
    ref = O.permute(t, p, alpha=alpha, tdst=c, beta=beta)
    assert relerr(results[0].to_host(), ref.data) <= TOL

    adj = tk.AdjointTensorMap(td)
    for q in [((4, 1), (2, 3)), ((4,), (3, 2, 1))]:
        ref = O.permute(t, q, adjoint=True)
        outs = [_run(monkeypatch, k, lambda: tk.permute(adj, q, copy=True)) for k in KERNELS]
        for o in outs[1:]:
            assert torch.equal(outs[0].data, o.data), q
        assert relerr(outs[0].to_host(), ref.data) <= TOL, q
