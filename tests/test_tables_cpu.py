"""Host-side parity (no GPU): block structure, fusion-tree tables and symbols of the product
against the oracle — bit-exact for integers (sizes, strides, offsets) and for the
recoupling coefficient of every single-tree fusion block; multi-tree blocks accumulate U
through matrix products, so they agree to 1e-14 (summation order)."""
import itertools

import numpy as np
import pytest

from helpers import (O, VSU2, VU1, VU1SU2, cfg1_spaces, cfg2_spaces, cfg3_spaces, cfg5_spaces,
                     five_leg, to_hom, to_sector)
import tensorkit_b200 as tk
from tensorkit_b200 import sectors as S
from tensorkit_b200.treetransformers import flatten_transformer, treebraider


def _check_layout(W):
    Wp = to_hom(W)
    total, blocks, subs, pairs = O.layout(W)
    ds = tk.degeneracystructure(Wp)
    ss = tk.sectorstructure(Wp)
    assert ds.totaldim == total
    assert len(ss.fusiontrees) == len(pairs)
    for (f1, f2), (sz, st, off) in zip(ss.fusiontrees, ds.subblockstructure):
        key = ((tuple(map(_osec, f1.uncoupled)), _osec(f1.coupled), f1.isdual, tuple(map(_osec, f1.innerlines))),
               (tuple(map(_osec, f2.uncoupled)), _osec(f2.coupled), f2.isdual, tuple(map(_osec, f2.innerlines))))
        assert subs[key] == (sz, st, off)
    assert [(_osec(c)) for c in ss.blocksectors] == list(blocks.keys())


def _osec(s):
    if isinstance(s, S.U1Irrep):
        return ("U1", s.q2)
    if isinstance(s, S.SU2Irrep):
        return ("SU2", s.j2)
    return ("P", tuple(_osec(x) for x in s.sectors))


def test_workload_layouts_and_sizes():
    V, Pp = cfg1_spaces()
    W1 = O.Hom([V, Pp], [V])
    assert O.layout(W1)[0] == 1216
    _check_layout(W1)
    V2, P2 = cfg2_spaces()
    W2 = O.Hom([V2, P2], [V2])
    assert O.layout(W2)[0] == 9576 and V2.dim() == 454
    _check_layout(W2)
    _check_layout(O.Hom([V2], [V2]))
    V4, P4 = cfg2_spaces(8)
    assert O.layout(O.Hom([V4, P4], [V4]))[0] == 612864 and V4.dim() == 3632
    V3, P3, Wm = cfg3_spaces()
    assert V3.dim() == 1924
    W3 = O.Hom([V3, Wm.flipdual()], [V3])
    assert O.layout(W3)[0] == 2398936
    _check_layout(W3)
    _check_layout(O.Hom([V3, P3, P3], [V3]))
    V5, P5 = cfg5_spaces()
    assert V5.dim() == 1321
    _check_layout(O.Hom([V5, P5], [V5]))


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_reference_test_space_layouts(spaces):
    for nd in range(0, 6):
        _check_layout(five_leg(spaces(), ndom=nd))


def _compare_tables(W, p, adjoint=False):
    Wp = to_hom(W)
    if adjoint:
        Ws, parent = Wp.adjoint(), Wp
        Wso = W.adjoint()
    else:
        Ws, parent = Wp, None
        Wso = W
    Wd = Ws.permute(p)
    n1, n2 = Ws.numout(), Ws.numin()
    tr = treebraider(Wd, Ws, p, (tuple(range(1, n1 + 1)), tuple(range(n1 + 1, n1 + n2 + 1))), parent)
    ft = flatten_transformer(tr, p)
    otab = O.transformer_table(Wso, p, W if adjoint else None)
    om = {src[2]: {(d[2], d[0], d[1]): c for d, c in lst} for src, lst in otab}
    exact = close = 0
    for g in range(ft.ngroups):
        s0, s1 = ft.group_src_ptr[g], ft.group_src_ptr[g + 1]
        t0, t1 = ft.group_dst_ptr[g], ft.group_dst_ptr[g + 1]
        U = ft.coeffs[ft.coeff_ptr[g]:ft.coeff_ptr[g + 1]].reshape(t1 - t0, s1 - s0)
        dsz = tuple(int(x) for x in ft.sizes[g][list(ft.perm)])
        for j in range(s1 - s0):
            ref = om[int(ft.src_offsets[s0 + j])]
            got = {}
            for i in range(t1 - t0):
                if U[i, j] != 0.0:
                    got[(int(ft.dst_offsets[t0 + i]), dsz, tuple(int(x) for x in ft.dst_strides[t0 + i]))] = U[i, j]
            single = (s1 - s0) == 1 and (t1 - t0) == 1
            for key in set(got) | set(ref):
                a, b = got.get(key, 0.0), ref.get(key, 0.0)
                if single:
                    assert a == b  # bit-exact
                    exact += 1
                else:
                    # multi-tree blocks: U accumulated by matrix products (summation order)
                    assert abs(a - b) <= 1e-14
                    close += 1
    return exact, close


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_transformer_tables_five_leg(spaces):
    W = five_leg(spaces())
    perms = list(itertools.permutations(range(1, 6)))[::11]
    for k in range(6):
        for p in perms:
            _compare_tables(W, (tuple(p[:k]), tuple(p[k:])))


def test_transformer_tables_workloads_bit_exact():
    V, Pp = cfg2_spaces()
    W = O.Hom([V, Pp], [V])
    for p in [((2, 3), (1,)), ((3,), (1, 2)), ((1,), (3, 2)), ((2, 1), (3,))]:
        ex, cl = _compare_tables(W, p)
        assert cl == 0 and ex > 0
    for p in [((1, 2), (3,)), ((3,), (1, 2))]:
        ex, cl = _compare_tables(W, p, adjoint=True)
        assert cl == 0 and ex > 0


def test_su2_fsymbols_bit_exact():
    n = 0
    for s in itertools.product(range(0, 6), repeat=6):
        a, b, c, d, e, f = [S.SU2Irrep(twice=x) for x in s]
        if not (S.Nsymbol(a, b, e) and S.Nsymbol(e, c, d) and S.Nsymbol(b, c, f) and S.Nsymbol(a, f, d)):
            continue
        assert S.Fsymbol(a, b, c, d, e, f) == O.Fsym(*[("SU2", x) for x in s])
        n += 1
    assert n > 1000


def test_sector_order_and_fusion():
    qs = [S.U1Irrep(q) for q in (-2, -1, 0, 1, 2)]
    assert [s.charge for s in sorted(qs)] == [0, 1, -1, 2, -2]
    assert [x.j2 for x in S.SU2Irrep(1).otimes(S.SU2Irrep(1.5))] == [1, 3, 5]
    assert S.Fsymbol(*[S.SU2Irrep(0.5)] * 4, S.SU2Irrep(0), S.SU2Irrep(0)) == -0.5
