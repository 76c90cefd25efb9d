"""tkb_reduce_noalloc — the allocation-free reduction — against tkb_reduce.

Callers whose device memory belongs entirely to another allocator (a Julia CUDA.jl pool, a
framework that has reserved the whole device), or that run where a device allocation may
block or fail, cannot call cudaMalloc; this entry point serves them from a static device
scratch array. The test calls it through the C ABI twice in a row (norm², then an inner
product that reuses the same scratch) and compares with the allocating entry point,
to 1e-13 relative. This file is collected last so that a run stopping at the first failure
has already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from helpers import O, cfg2_spaces, to_device

pytestmark = pytest.mark.gpu


def _segments(t):
    from tensorkit_b200.structure import blockstructure
    segs = [(a, d1 * d2, 1, float(c.dim())) for c, ((d1, d2), (a, _)) in blockstructure(t.space).items()]
    off = np.array([s[0] for s in segs], np.int64)
    cnt = np.array([s[1] for s in segs], np.int64)
    st = np.array([s[2] for s in segs], np.int64)
    w = np.array([s[3] for s in segs], np.float64)
    return off, cnt, st, w


def _noalloc(lib, dev, stream, kind, dtype, x, y, segs):
    from tensorkit_b200 import _lib as L
    off, cnt, st, w = segs
    out = np.zeros(2)
    rc = lib.tkb_reduce_noalloc(dev, C.c_void_p(stream), kind, dtype, C.c_void_p(x.data_ptr()),
                                C.c_void_p(y.data_ptr() if y is not None else 0), x.numel(), len(off),
                                L.ptr(off), L.ptr(cnt), L.ptr(st), L.ptr(w),
                                out.ctypes.data_as(C.POINTER(C.c_double)))
    L.check(rc)
    return out


def test_noalloc_matches_reduce_twice():
    import torch
    import tensorkit_b200 as tk
    from tensorkit_b200 import _lib as L
    lib = L.load()
    V, _ = cfg2_spaces(8)
    W = O.Hom([V], [V])
    xo, yo = O.randn(W, 21, True), O.randn(W, 22, True)
    x = to_device(xo)
    y = to_device(yo)
    segs = _segments(x)
    stream = torch.cuda.current_stream().cuda_stream
    dev = x.data.device.index

    # call 1: weighted squared norm, against the allocating entry point and the CPU oracle
    got = _noalloc(lib, dev, stream, L.TKB_NORM2, L.TKB_C128, x.data, None, segs)
    want = tk.norm(x) ** 2
    assert abs(got[0] - want) <= 1e-13 * want
    assert abs(got[0] - O.norm(xo) ** 2) <= 1e-13 * want
    # call 2: inner product, same scratch
    got = _noalloc(lib, dev, stream, L.TKB_INNER, L.TKB_C128, x.data, y.data, segs)
    want = tk.inner(x, y)
    assert abs(complex(got[0], got[1]) - want) <= 1e-13 * abs(want)
    assert abs(complex(got[0], got[1]) - O.inner(xo, yo)) <= 1e-13 * abs(want)
    # a real vector through the same scratch
    xro = O.randn(W, 23, False)
    xr = to_device(xro)
    got = _noalloc(lib, dev, stream, L.TKB_NORM2, L.TKB_F64, xr.data, None, _segments(xr))
    want = tk.norm(xr) ** 2
    assert abs(got[0] - want) <= 1e-13 * want
    assert abs(got[0] - O.norm(xro) ** 2) <= 1e-13 * want


def test_noalloc_trace_strided_and_empty():
    """trace: strided diagonal segments (stride d1 + 1) with an empty segment in between, which
    exercises the partial kernel's search over equal prefix sums; then calls that reduce
    nothing. Compared with tkb_reduce on the same segments and with the CPU oracle."""
    import torch
    import tensorkit_b200 as tk
    from tensorkit_b200 import _lib as L
    from tensorkit_b200.structure import blockstructure
    lib = L.load()
    V, _ = cfg2_spaces(8)
    W = O.Hom([V], [V])
    xo = O.randn(W, 24, False)
    x = to_device(xo)
    stream = torch.cuda.current_stream().cuda_stream
    dev = x.data.device.index
    diag = [(a, d1, d1 + 1, float(c.dim())) for c, ((d1, d2), (a, _)) in blockstructure(x.space).items()]
    diag.insert(3, (0, 0, 1, 5.0))  # empty segment
    segs = tuple(np.array([d[i] for d in diag], np.int64 if i < 3 else np.float64) for i in range(4))
    got = _noalloc(lib, dev, stream, L.TKB_TRACE, L.TKB_F64, x.data, None, segs)
    want = tk.tr(x)
    assert abs(got[0] - want) <= 1e-12 * max(1.0, abs(want))
    assert abs(got[0] - O.tr(xo)) <= 1e-12 * max(1.0, abs(want))
    # the allocating entry point on the identical segment list
    ctx = tk.get_context(dev)
    plan = tk.backend.ReducePlan(ctx, list(diag), x.data.numel())
    ref = np.zeros(2)
    L.check(lib.tkb_reduce(ctx.handle, plan.handle, L.TKB_TRACE, L.TKB_F64, C.c_void_p(x.data.data_ptr()),
                           None, ref.ctypes.data_as(C.POINTER(C.c_double))), ctx.handle)
    assert abs(got[0] - ref[0]) <= 1e-13 * max(1.0, abs(ref[0]))
    # nothing to reduce: no segments, then only empty segments
    for n in (0, 2):
        off = np.zeros(n, np.int64)
        cnt = np.zeros(n, np.int64)
        one = np.ones(n, np.int64)
        w = np.ones(n)
        got = _noalloc(lib, dev, stream, L.TKB_NORM2, L.TKB_F64, x.data, None, (off, cnt, one, w))
        assert got[0] == 0.0 and got[1] == 0.0


def test_noalloc_rejects_too_many_segments():
    import torch
    from tensorkit_b200 import _lib as L
    lib = L.load()
    x = torch.zeros(4096, dtype=torch.float64, device="cuda")
    n = 1025
    off = np.arange(n, dtype=np.int64)
    one = np.ones(n, np.int64)
    w = np.ones(n)
    out = np.zeros(2)
    rc = lib.tkb_reduce_noalloc(0, None, L.TKB_NORM2, L.TKB_F64, C.c_void_p(x.data_ptr()), None,
                                x.numel(), n, L.ptr(off), L.ptr(one), L.ptr(one), L.ptr(w),
                                out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == L.TKB_ERR_SIZE
    assert b"1024" in lib.tkb_last_error(None)
