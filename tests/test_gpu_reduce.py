"""norm / inner / tr on the device vs the oracle (src/tensors/linalg.jl:257-282, 319-327;
src/tensors/vectorinterface.jl:114-130): dim(c)-weighted FP64 reductions, 1e-13 relative."""
import numpy as np
import pytest

from helpers import O, VSU2, cfg2_spaces, cfg5_spaces, five_leg, to_device
import tensorkit_b200 as tk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cplx", [False, True])
def test_norm_inner(cplx):
    W = five_leg(VSU2())
    x, y = O.randn(W, 1, cplx), O.randn(W, 2, cplx)
    xd, yd = to_device(x), to_device(y)
    assert abs(tk.norm(xd) - O.norm(x)) <= 1e-13 * O.norm(x)
    ref = O.inner(x, y)
    assert abs(tk.inner(xd, yd) - ref) <= 1e-13 * abs(ref)


@pytest.mark.parametrize("spaces", [cfg2_spaces, cfg5_spaces])
@pytest.mark.parametrize("cplx", [False, True])
def test_trace(spaces, cplx):
    V, _ = spaces()
    E = O.randn(O.Hom([V], [V]), 4, cplx)
    Ed = to_device(E)
    ref = O.tr(E)
    assert abs(tk.tr(Ed) - ref) <= 1e-13 * max(1.0, abs(ref))


def test_reduce_deterministic():
    V, _ = cfg2_spaces(8)
    x = to_device(O.randn(O.Hom([V], [V]), 5))
    vals = {tk.norm(x) for _ in range(5)}
    assert len(vals) == 1
