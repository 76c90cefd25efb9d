"""Parity of the grouped block GEMM (mul!) with the oracle, plain FP64 and split precision.

Mirrors mul! semantics (src/tensors/linalg.jl:330-370): matching coupled sectors multiply,
sectors of C missing from A or B are scaled by β. Tolerances: plain FP64 1e-12 relative
(max-norm over the result); split precision (int8 slices) 1e-12 relative at the default
7 slices."""
import numpy as np
import pytest

from helpers import O, VSU2, cfg1_spaces, cfg2_spaces, relerr, to_device, to_hom
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu
TOL_PLAIN = 1e-12
TOL_SPLIT = 1e-12


def _mats(cplx, mult=1):
    V, Pp = cfg2_spaces(mult)
    WA = O.Hom([V, Pp], [V])
    WB = O.Hom([V], [V])
    A = O.randn(WA, 1, cplx)
    B = O.randn(WB, 2, cplx)
    return A, B


@pytest.mark.parametrize("prec", ["plain", "split"])
@pytest.mark.parametrize("cplx", [False, True])
def test_mul_su2(prec, cplx):
    A, B = _mats(cplx)
    ref = O.mul(A, B)
    Ad, Bd = to_device(A), to_device(B)
    C = tk.TensorMap.zeros(to_hom(ref.W), dtype=Ad.dtype, device=Ad.device)
    tk.mul_(C, Ad, Bd, 1.0, 0.0, prec=prec)
    assert relerr(C.to_host(), ref.data) <= (TOL_PLAIN if prec == "plain" else TOL_SPLIT)


@pytest.mark.parametrize("prec", ["plain", "split"])
def test_mul_alpha_beta_adjoint(prec):
    A, B = _mats(True)
    # C = α·A'·A + β·C with a lazy adjoint left operand
    ref0 = O.mul(A, A, adjA=True)
    C0 = O.randn(ref0.W, 9, True)
    Ad = to_device(A)
    Cd = to_device(C0)
    alpha, beta = 0.75 + 0.5j, -1.5 + 0.25j
    tk.mul_(Cd, tk.AdjointTensorMap(Ad), Ad, alpha, beta, prec=prec)
    ref = alpha * ref0.data + beta * C0.data
    assert relerr(Cd.to_host(), ref) <= (TOL_PLAIN if prec == "plain" else TOL_SPLIT)


@pytest.mark.parametrize("prec", ["plain", "split"])
def test_mul_missing_sectors_scale_by_beta(prec):
    """Sectors of C absent from A·B get C_c = β·C_c."""
    V = O.Space({O.U1(q): 3 for q in range(-2, 3)})
    V2 = O.Space({O.U1(q): 2 for q in range(0, 2)})
    WA = O.Hom([V], [V2])
    WB = O.Hom([V2], [V])
    A, B = O.randn(WA, 1), O.randn(WB, 2)
    ref = O.mul(A, B)
    C0 = O.randn(ref.W, 3)
    Cd = to_device(C0)
    tk.mul_(Cd, to_device(A), to_device(B), 2.0, 0.5, prec=prec)
    want = 2.0 * ref.data + 0.5 * C0.data
    assert relerr(Cd.to_host(), want) <= 1e-12


@pytest.mark.parametrize("slices", [4, 5, 6, 7])
def test_split_error_decreases_with_slices(slices):
    """A fixed slice count (3..7) is used for every block, with no FP64 check."""
    A, B = _mats(False)
    ref = O.mul(A, B)
    Ad, Bd = to_device(A), to_device(B)
    C = tk.TensorMap.zeros(to_hom(ref.W), device=Ad.device)
    tk.mul_(C, Ad, Bd, prec="split", slices=slices)
    err = relerr(C.to_host(), ref.data)
    # truncation bound of the slicing: ~2^-7S per operand, times a modest k-dependent factor
    assert err <= 2.0 ** (-7 * slices) * 64


@pytest.mark.parametrize("cplx", [False, True])
def test_split_k_reductions(cplx):
    """Few output tiles with long K: a tile's K loop is split into two halves that run on the two
    CTAs of a cluster; each CTA adds the peer's half of the columns it keeps (through the peer's
    shared memory) and applies α and β to that half. Run twice through the cached plan (the
    exchange barriers and counters are fresh or cleared between launches)."""
    A, B = _mats(cplx, mult=8)
    ref = O.mul(A, B)
    C0 = O.randn(ref.W, 4, cplx)
    Ad, Bd = to_device(A), to_device(B)
    want = 0.5 * ref.data - 2.0 * C0.data
    for _ in range(2):
        Cd = to_device(C0)
        tk.mul_(Cd, Ad, Bd, 0.5, -2.0, prec="split")
        assert relerr(Cd.to_host(), want) <= TOL_SPLIT


def test_split_long_k_multiwave():
    """K beyond the exact int32 range of one products item (≈ 19K positions at 7 slices) forces
    two pieces per tile (the two CTAs of a cluster), and more tile pairs than clusters: the
    persistent clusters take several pairs in turn."""
    Vm = O.Space({O.U1(0): 1024})
    Vk = O.Space({O.U1(0): 20000})
    Vn = O.Space({O.U1(0): 640})
    A = O.randn(O.Hom([Vm], [Vk]), 11)
    B = O.randn(O.Hom([Vk], [Vn]), 12)
    ref = O.mul(A, B)
    Ad, Bd = to_device(A), to_device(B)
    C = tk.TensorMap.zeros(to_hom(ref.W), dtype=Ad.dtype, device=Ad.device)
    tk.mul_(C, Ad, Bd, 1.0, 0.0, prec="split")
    assert relerr(C.to_host(), ref.data) <= TOL_SPLIT


@pytest.mark.parametrize("cplx", [False, True])
def test_split_many_short_k_tasks(cplx):
    """Hundreds of slicing tasks with short K (more than one per CTA) and more output tiles than
    CTAs (several items per CTA: the accumulators pass back and forth between the MMA warp and
    the epilogue); op(A) rows and op(B) columns through both load layouts (B given as Bᴴ)."""
    Vm = O.Space({O.U1(0): 24000, O.U1(1): 300})
    Vk = O.Space({O.U1(0): 128, O.U1(1): 40})
    Vn = O.Space({O.U1(0): 96, O.U1(1): 20})
    A = O.randn(O.Hom([Vm], [Vk]), 21, cplx)
    Bt = O.randn(O.Hom([Vn], [Vk]), 22, cplx)
    ref = O.mul(A, Bt, adjB=True)
    Ad, Btd = to_device(A), to_device(Bt)
    C = tk.TensorMap.zeros(to_hom(ref.W), dtype=Ad.dtype, device=Ad.device)
    tk.mul_(C, Ad, tk.AdjointTensorMap(Btd), 1.0, 0.0, prec="split")
    assert relerr(C.to_host(), ref.data) <= TOL_SPLIT


def _skinny(kmax, nmax, cplx, adjA):
    """Tall blocks (≥ 2048 rows) against narrow bonds: every block has n, k ≤ 16, so the
    plan runs the skinny row kernel; kmax/nmax pick its width class (2, 4, 6, 8, 16)."""
    V = O.Space({O.U1(0): 3000, O.U1(1): 2500, O.U1(-1): 2100})
    Wk = O.Space({O.U1(0): kmax, O.U1(1): max(1, kmax - 1), O.U1(-1): 1})
    Wn = O.Space({O.U1(0): max(1, nmax - 1), O.U1(1): nmax, O.U1(-1): 2 if nmax > 1 else 1})
    A = O.randn(O.Hom([Wk], [V]) if adjA else O.Hom([V], [Wk]), 31, cplx)
    B = O.randn(O.Hom([Wk], [Wn]), 32, cplx)
    return A, B


@pytest.mark.parametrize("prec", ["plain", "split"])
@pytest.mark.parametrize("kn", [(2, 2), (3, 4), (5, 5), (7, 6), (13, 16)], ids=lambda x: f"k{x[0]}n{x[1]}")
@pytest.mark.parametrize("cplx", [False, True])
def test_mul_skinny_blocks(prec, kn, cplx):
    kmax, nmax = kn
    for adjA in (False, True):
        A, B = _skinny(kmax, nmax, cplx, adjA)
        ref0 = O.mul(A, B, adjA=adjA)
        Ad, Bd = to_device(A), to_device(B)
        opA = tk.AdjointTensorMap(Ad) if adjA else Ad
        C = tk.TensorMap.zeros(to_hom(ref0.W), dtype=Ad.dtype, device=Ad.device)
        tk.mul_(C, opA, Bd, 1.0, 0.0, prec=prec)
        assert relerr(C.to_host(), ref0.data) <= TOL_PLAIN, adjA
        C0 = O.randn(ref0.W, 33, cplx)
        Cd = to_device(C0)
        alpha, beta = (0.75 + 0.5j, -1.5 + 0.25j) if cplx else (0.75, -1.5)
        tk.mul_(Cd, opA, Bd, alpha, beta, prec=prec)
        assert relerr(Cd.to_host(), alpha * ref0.data + beta * C0.data) <= TOL_PLAIN, adjA


@pytest.mark.parametrize("prec", ["plain", "split"])
@pytest.mark.parametrize("cplx", [False, True])
def test_mul_skinny_missing_sector_scales_by_beta(prec, cplx):
    """A tall narrow sector of C that A·B does not reach (k = 0 on the skinny path) gets β·C_c;
    the other sectors get α·A_c·B_c + β·C_c (src/tensors/linalg.jl:341-366)."""
    V = O.Space({O.U1(0): 3000, O.U1(1): 2500, O.U1(2): 2200})
    Wk = O.Space({O.U1(0): 3, O.U1(1): 2})
    Wn = O.Space({O.U1(0): 2, O.U1(1): 3, O.U1(2): 4})
    A = O.randn(O.Hom([V], [Wk]), 41, cplx)
    B = O.randn(O.Hom([Wk], [Wn]), 42, cplx)
    C0 = O.randn(O.Hom([V], [Wn]), 43, cplx)
    ref = O.mul(A, B)
    assert ref.W == C0.W
    alpha, beta = (1.25 - 0.5j, 0.5 + 0.75j) if cplx else (1.25, 0.5)
    Cd = to_device(C0)
    tk.mul_(Cd, to_device(A), to_device(B), alpha, beta, prec=prec)
    assert relerr(Cd.to_host(), alpha * ref.data + beta * C0.data) <= TOL_PLAIN
