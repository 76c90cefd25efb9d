"""The GEMM autotuner on the GPU: precision "auto" times every candidate (precision × split-K
decomposition) on the operands, keeps the fastest one within 1e-12 of plain FP64, records it in
the on-disk cache, and a fresh plan cache finds the record without timing."""
import pytest

from helpers import O, cfg2_spaces, relerr, to_device, to_hom
import tensorkit_b200 as tk
from tensorkit_b200 import tuning as T
from tensorkit_b200.linalg import gemm_plan

pytestmark = pytest.mark.gpu


def test_autotune_choice_cached_and_accurate(tmp_path, monkeypatch):
    monkeypatch.setenv("TKB_TUNE_CACHE", str(tmp_path / "tune.json"))
    V, Pp = cfg2_spaces(8)
    A = O.randn(O.Hom([V, Pp], [V]), 1)
    B = O.randn(O.Hom([V], [V]), 2)
    ref = O.mul(A, B)
    Ad, Bd = to_device(A), to_device(B)
    ctx = tk.get_context(Ad.device.index)
    ctx.empty_caches()
    C = tk.TensorMap.zeros(to_hom(ref.W), dtype=Ad.dtype, device=Ad.device)
    tk.mul_(C, Ad, Bd, 1.0, 0.0, prec="auto")
    assert relerr(C.to_host(), ref.data) <= 1e-12
    plan = gemm_plan(ctx, C, Ad, Bd, "auto")
    rec = plan.tuned
    assert rec["cached"] is False
    t = rec["timings"]
    chosen = t["/".join(map(str, rec["choice"]))]["us"]
    # the defaults of both precisions were candidates: the choice is not slower than either
    assert chosen <= min(t["plain/8/4"]["us"], t["split/8/4"]["us"])
    # a fresh plan cache (a new process would look the same) reuses the record without timing
    ctx.empty_caches()
    C2 = tk.TensorMap.zeros(to_hom(ref.W), dtype=Ad.dtype, device=Ad.device)
    tk.mul_(C2, Ad, Bd, 1.0, 0.0, prec="auto")
    plan2 = gemm_plan(ctx, C2, Ad, Bd, "auto")
    assert plan2.tuned["cached"] is True and plan2.tuned["choice"] == rec["choice"]
    assert relerr(C2.to_host(), ref.data) <= 1e-12
    ctx.empty_caches()
