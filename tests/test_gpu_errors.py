"""Failure detection without a GPU fault: a bounded device wait that runs out (a flag that
nothing sets) is reported by the next synchronisation as TKB_ERR_TIMEOUT with a message, the
record is cleared, and the context keeps working."""

import pytest

from helpers import O, cfg2_spaces, relerr, to_device, to_hom
import tensorkit_b200 as tk
from tensorkit_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_bounded_wait_timeout_is_reported_and_cleared():
    ctx = tk.get_context(0)
    lib = ctx.lib
    assert lib.tkb_ctx_synchronize(ctx.handle) == L.TKB_OK
    assert lib.tkb_selftest_bounded_wait(ctx.handle, 2000) == L.TKB_OK
    assert lib.tkb_ctx_synchronize(ctx.handle) == L.TKB_ERR_TIMEOUT
    assert b"never set" in lib.tkb_last_error(ctx.handle)
    assert lib.tkb_ctx_synchronize(ctx.handle) == L.TKB_OK  # the record was cleared
    # out-of-range limits are argument errors, nothing is launched
    assert lib.tkb_selftest_bounded_wait(ctx.handle, 0) == L.TKB_ERR_ARG
    assert lib.tkb_selftest_bounded_wait(ctx.handle, 2_000_000) == L.TKB_ERR_ARG
    # the context still computes
    V, Pp = cfg2_spaces()
    A, B = O.randn(O.Hom([V, Pp], [V]), 1), O.randn(O.Hom([V], [V]), 2)
    ref = O.mul(A, B)
    Cd = tk.TensorMap.zeros(to_hom(ref.W), device="cuda")
    tk.mul_(Cd, to_device(A), to_device(B), prec="split")
    assert relerr(Cd.to_host(), ref.data) <= 1e-12
