"""Split precision where the slices alone would miss 1e-12: the per-block slice count and the
per-tile FP64 check, against the FP64 oracle.

- Random blocks (the workloads' inputs) keep 7 slices and no tile is sent to FP64.
- Cancellation: C = A·B with the columns of B close to the null space of A's rows, so |C| is
  about 1e-7 of |A|·|B|. The slicing statistics cannot see this; the tile check after the
  products must send the tiles to FP64, and the result meets 1e-12 of the (small) exact C.
- A wide exponent range inside rows and columns: every row of op(A) and column of op(B) has
  one entry 1e6 times the rest, at K positions that never coincide, so the small entries (which
  keep only a few significant bits next to the large one) decide most of C. The block
  statistics pick FP64 for such a block before any product runs, while an ordinary block of
  the same contraction keeps its slices.
"""
import numpy as np
import pytest

from helpers import O, cfg2_spaces, relerr, to_device, to_hom
import tensorkit_b200 as tk
from tensorkit_b200.linalg import gemm_plan

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _one_sector(d):
    return O.Space({O.U1(0): d})


def _bt(W, mat):
    return O.BT(W, np.asfortranarray(mat).reshape(-1, order="F").copy())


def _run(A, B, prec="split"):
    ref = O.mul(A, B)
    Ad, Bd = to_device(A), to_device(B)
    C = tk.TensorMap.zeros(to_hom(ref.W), dtype=Ad.dtype, device=Ad.device)
    tk.mul_(C, Ad, Bd, 1.0, 0.0, prec=prec)
    plan = gemm_plan(tk.get_context(Ad.device.index), C, Ad, Bd, prec)
    return C.to_host(), ref.data, plan


@pytest.mark.parametrize("cplx", [False, True])
def test_random_blocks_keep_seven_slices(cplx):
    V, Pp = cfg2_spaces(8)
    A = O.randn(O.Hom([V, Pp], [V]), 1, cplx)
    B = O.randn(O.Hom([V], [V]), 2, cplx)
    got, ref, plan = _run(A, B)
    assert relerr(got, ref) <= TOL
    slices, fp64_tiles = plan.last_slices()
    assert all(s == 7 for s in slices if s >= 0) and fp64_tiles == 0, (slices, fp64_tiles)


@pytest.mark.parametrize("beta_zero", [True, False])
def test_cancellation_goes_to_fp64(beta_zero):
    rng = np.random.default_rng(5)
    m, k, n = 192, 320, 96
    a = rng.standard_normal((m, k))
    # columns of b: null-space vectors of a's rows plus a 1e-6 perturbation
    _, _, vt = np.linalg.svd(a)
    null = vt[m:].T                                   # k × (k − m)
    b = null[:, :n] * 10.0 + 1e-6 * rng.standard_normal((k, n))
    A = _bt(O.Hom([_one_sector(m)], [_one_sector(k)]), a)
    B = _bt(O.Hom([_one_sector(k)], [_one_sector(n)]), b)
    ref = O.mul(A, B)
    assert np.abs(ref.data).max() < 1e-4 * np.abs(a).max() * np.abs(b).max() * np.sqrt(k)
    Ad, Bd = to_device(A), to_device(B)
    C0 = O.randn(ref.W, 6)
    Cd = to_device(C0)
    beta = 0.0 if beta_zero else 0.5
    tk.mul_(Cd, Ad, Bd, 1.0, beta, prec="split")
    want = ref.data + beta * C0.data
    assert relerr(Cd.to_host(), want) <= TOL
    plan = gemm_plan(tk.get_context(Ad.device.index), Cd, Ad, Bd, "split")
    slices, fp64_tiles = plan.last_slices()
    assert fp64_tiles > 0, (slices, fp64_tiles)


def test_wide_exponent_range_block_runs_fp64():
    rng = np.random.default_rng(7)
    # sector 0: an ordinary random block; sector 1: rows of op(A) and columns of op(B) that each
    # have one entry 1e6 times the rest, at K positions that never coincide
    m, k, n = 160, 256, 128
    Vm = O.Space({O.U1(0): m, O.U1(1): m})
    Vk = O.Space({O.U1(0): k, O.U1(1): k})
    Vn = O.Space({O.U1(0): n, O.U1(1): n})
    A = O.randn(O.Hom([Vm], [Vk]), 8)
    B = O.randn(O.Hom([Vk], [Vn]), 9)
    a1 = rng.standard_normal((m, k))
    b1 = rng.standard_normal((k, n))
    for i in range(m):
        a1[i, i % (k // 2)] *= 1e6                 # large entries of A in the first half of K
    for j in range(n):
        b1[k // 2 + j % (k // 2), j] *= 1e6        # large entries of B in the second half
    A.block(O.U1(1))[...] = a1
    B.block(O.U1(1))[...] = b1
    got, ref, plan = _run(A, B)
    assert relerr(got, ref) <= TOL
    slices, _ = plan.last_slices()
    assert sorted(s for s in slices if s >= 0) == [0, 7], slices
