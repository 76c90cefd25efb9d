"""Partial-trace tables (no GPU): the flattened trace_permute! of the package, executed by a
numpy stand-in of the device kernel, equals the oracle's trace on the cases of the
reference's own tests (test/tensors/contractions.jl:17-67): full trace, partial trace of a
six-leg tensor, the two-step partial trace, and a tensor with domain legs."""
import numpy as np
import pytest

from helpers import O, VSU2, VU1, VU1SU2, to_hom
from tensorkit_b200.trace import build_trace_table


def run_table(flat, src, dst_len):
    """Executes a trace table the way tkb_tracetransform does (α = 1, β = 0)."""
    dst = np.zeros(dst_len, dtype=src.dtype)
    it = src.itemsize
    nf, nt = flat.nfree, flat.ntrace
    for g in range(flat.ngroups):
        sz = tuple(flat.sizes[g * nf:(g + 1) * nf])
        dv = np.lib.stride_tricks.as_strided(dst[flat.dst_offsets[g]:], sz,
                                             tuple(int(s) * it for s in flat.dst_strides[g * nf:(g + 1) * nf]))
        for e in range(flat.group_entry_ptr[g], flat.group_entry_ptr[g + 1]):
            shape = sz + tuple(flat.trace_sizes[e * nt:(e + 1) * nt])
            strides = tuple(flat.src_strides[e * nf:(e + 1) * nf]) + tuple(flat.trace_strides[e * nt:(e + 1) * nt])
            sv = np.lib.stride_tricks.as_strided(src[flat.src_offsets[e]:], shape, tuple(int(s) * it for s in strides))
            dv += flat.coeffs[e] * sv.sum(axis=tuple(range(nf, nf + nt)))
    return dst


def cases(V1, V2, V3):
    d = lambda v: v.flipdual()
    return [
        # t2[a, b] := t[c, d, b, d, c, a] on V1⊗V2'⊗V3⊗V2⊗V1'⊗V3'
        (O.Hom([V1, d(V2), V3, V2, d(V1), d(V3)], []), ((6, 3), ()), ((1, 2), (5, 4))),
        # t2[a; b] := t[c d b; c d a] and the two-step version on V1⊗V2⊗V3 ← V1⊗V2⊗V3
        (O.Hom([V1, V2, V3], [V1, V2, V3]), ((6,), (3,)), ((1, 2), (4, 5))),
        (O.Hom([V1, V2, V3], [V1, V2, V3]), ((6, 5), (3, 2)), ((1,), (4,))),
        # full trace of V1⊗V2'⊗V2⊗V1' permuted to ((1, 2), (4, 3))
        (O.Hom([V1, d(V2), V2, d(V1)], []), ((), ()), ((1, 2), (4, 3))),
        # trace over a codomain/domain pair, output keeps one leg on each side
        (O.Hom([V1, V2], [V1, V3]), ((2,), (4,)), ((1,), (3,))),
    ]


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_trace_table_vs_oracle(spaces):
    V1, V2, V3 = spaces()[:3]
    for k, (W, p, q) in enumerate(cases(V1, V2, V3)):
        t = O.randn(W, 40 + k, True)
        ref = O.trace_permute(t, p, q)
        flat = build_trace_table(to_hom(W), p, q)
        got = run_table(flat, t.data, ref.data.size)
        scale = max(np.abs(ref.data).max(), 1e-300)
        assert np.abs(got - ref.data).max() <= 1e-13 * scale, (k, p, q)
