"""Edge cases of the device path: a full contraction to a scalar, split-precision rows whose
maxima sit at the ends of the FP64 exponent range (including zero rows and subnormal maxima),
and an exact-zero operand. Tolerances as in the other GEMM tests: 1e-12 relative."""
import numpy as np
import pytest

from helpers import O, cfg2_spaces, relerr, to_device, to_hom
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["plain", "split"])
def test_full_contraction_to_scalar(prec):
    V, Pp = cfg2_spaces()
    A = O.randn(O.Hom([V, Pp], [V]), 3, True)
    Ad = to_device(A)
    with tk.using_precision(prec):
        s = tk.tensor("s[] := A[a,p;b]*conj(A[a,p;b])", A=Ad)
    got = complex(s.to_host().sum())
    want = tk.norm(Ad) ** 2
    assert abs(got - want) <= 1e-12 * want


def test_split_extreme_row_scales():
    """Rows of op(A) scaled by 1e-150 … 1e150, a zero row, a row of subnormal values, and
    columns of op(B) scaled by 1e-100 … 1e100: each output entry keeps its accuracy relative to
    its row and column scales, because every row and column is sliced with its own exponent
    (including the two-factor scaling of subnormal rows and the ldexp path of the epilogue)."""
    Vm = O.Space({O.U1(0): 70})
    Vk = O.Space({O.U1(0): 96})
    Vn = O.Space({O.U1(0): 50})
    A = O.randn(O.Hom([Vm], [Vk]), 31)
    B = O.randn(O.Hom([Vk], [Vn]), 32)
    a = A.block(O.U1(0))   # views into the flat data (column-major blocks)
    b = B.block(O.U1(0))
    rs = np.logspace(-150, 150, a.shape[0])
    a *= rs[:, None]
    a[5, :] = 0.0
    a[6, :] = np.random.default_rng(7).standard_normal(a.shape[1]) * 1e-310  # subnormal row
    cs = np.logspace(-100, 100, b.shape[1])
    b *= cs[None, :]
    ref = O.mul(A, B)
    Ad, Bd = to_device(A), to_device(B)
    C = tk.TensorMap.zeros(to_hom(ref.W), dtype=Ad.dtype, device=Ad.device)
    tk.mul_(C, Ad, Bd, 1.0, 0.0, prec="split")
    got = C.to_host()
    r = ref.block(O.U1(0))
    g = got.reshape(r.shape[1], r.shape[0]).T
    # error per entry against the scale |row max|·|col max|·k of its row and column; entries
    # whose scale falls below the normal range (the subnormal row times the smallest columns)
    # carry only absolute precision, in the oracle's FP64 product as well
    scale = np.abs(a).max(1)[:, None] * np.abs(b).max(0)[None, :] * a.shape[1]
    normal = scale > 1e-290
    assert np.all(np.abs(g - r)[normal] <= 1e-12 * scale[normal])
    assert np.all(np.abs(g - r)[~normal] <= 1e-300)
    assert np.all(g[5, :] == 0.0)
    assert np.count_nonzero(normal[6]) > 10  # the subnormal row is checked relative to its scale


def test_split_zero_operand():
    V, Pp = cfg2_spaces()
    A = O.randn(O.Hom([V, Pp], [V]), 4)
    A.data[:] = 0.0
    B = O.randn(O.Hom([V], [V]), 5)
    C0 = O.randn(O.mul(A, B).W, 6)
    Ad, Bd, Cd = to_device(A), to_device(B), to_device(C0)
    tk.mul_(Cd, Ad, Bd, 1.0, 0.5, prec="split")
    assert relerr(Cd.to_host(), 0.5 * C0.data) <= 1e-15
