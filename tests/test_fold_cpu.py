"""Host-side (no GPU): the planar moves of the transpose path — multi_Fmove / multi_Fmove_inv,
foldright / foldleft, cycleclockwise / cycleanticlockwise and fstranspose
(`src/fusiontrees/basic_manipulations.jl:191-440`, `src/fusiontrees/duality_manipulations.jl:220-442`,
`:534-562`), and the transpose transformer built from them (`src/tensors/treetransformers.jl:175-180`).

Every sector here is bosonic, so a planar permutation equals the braided one: fstranspose must
reproduce the braid route (whose tables are pinned to the oracle in test_tables_cpu.py) on every
cyclic permutation, dual legs and half-integer spins included. Folding forth and back, and
rotating forth and back, must give the identity."""
import numpy as np
import pytest

from helpers import VSU2, VU1, VU1SU2, five_leg, to_hom
from tensorkit_b200 import fusiontrees as F
from tensorkit_b200.sectors import ProductSector, SU2Irrep, U1Irrep
from tensorkit_b200.treetransformers import flatten_transformer, treebraider, treetransposer


def _cyclic_perms(n1, n2):
    """Every (p₁, p₂) whose linearisation is a cyclic shift of the legs."""
    N = n1 + n2
    ring = list(range(1, n1 + 1)) + list(reversed(range(n1 + 1, N + 1)))
    out = []
    for r in range(N):
        rot = ring[r:] + ring[:r]
        for N1 in range(N + 1):
            p1, p2 = tuple(rot[:N1]), tuple(reversed(rot[N1:]))
            lin = F.linearizepermutation(p1, p2, n1, n2)
            if all(lin[(i + 1) % N] == (lin[i] % N) + 1 for i in range(N)) and (p1, p2) not in out:
                out.append((p1, p2))
    return out


def _su2(*js):
    return tuple(SU2Irrep(j) for j in js)


def _p(*qj):
    return tuple(ProductSector(U1Irrep(q), SU2Irrep(j)) for q, j in qj)


BLOCKS = {
    "su2_int": (_su2(1, 2, 1), _su2(2), (False, True, False), (True,)),
    "su2_int_5leg": (_su2(1, 1, 1), _su2(1, 2), (False, False, True), (False, True)),
    "su2_half": (_su2(0.5, 1, 0.5), _su2(1), (True, False, True), (False,)),
    "su2_half_5leg": (_su2(0.5, 0.5, 0.5), _su2(0.5, 1), (False, True, False), (True, False)),
    "su2_half_split_1_4": (_su2(1.5), _su2(0.5, 1, 0.5, 0.5), (True,), (False, True, True, False)),
    "u1xsu2": (_p((1, 0.5), (-1, 1), (0, 0.5)), _p((0, 1), (0, 0)), (False, True, False), (True, False)),
}


@pytest.mark.parametrize("name", list(BLOCKS))
def test_fstranspose_equals_braid_route_on_blocks(name):
    u1, u2, d1, d2 = BLOCKS[name]
    src = F.FusionTreeBlock((u1, u2), (d1, d2), u1[0].unit())
    assert len(src) > 0
    perms = _cyclic_perms(len(u1), len(u2))
    assert len(perms) >= (len(u1) + len(u2)) * 2
    for p1, p2 in perms:
        dst_t, U_t = F.fstranspose(src, p1, p2)
        dst_b, U_b = F.permute(src, (p1, p2))
        assert dst_t.trees == dst_b.trees
        assert np.abs(U_t - U_b).max() <= 1e-13, (p1, p2)


def test_fstranspose_equals_braid_route_on_u1_pairs():
    u = tuple(U1Irrep(q) for q in (1, -1, 2))
    blk = F.FusionTreeBlock((u, (U1Irrep(2),)), ((False, True, False), (False,)), u[0].unit())
    assert len(blk) > 0
    for pair in blk.trees:
        for p1, p2 in _cyclic_perms(3, 1):
            pt, ct = F.fstranspose(pair, p1, p2)
            pb, cb = F.permute(pair, (p1, p2))
            assert pt == pb and abs(ct - cb) <= 1e-15


def test_fold_and_rotation_round_trips():
    src = F.FusionTreeBlock((_su2(0.5, 1, 1.5), _su2(1, 1)), ((True, False, True), (False, True)),
                            SU2Irrep(0).unit())
    assert len(src) > 0
    I = np.eye(len(src))
    d1, U1 = F.foldright(src)
    d2, U2 = F.foldleft(d1)
    assert d2.trees == src.trees and np.abs(U2 @ U1 - I).max() <= 1e-13
    d1, U1 = F.cycleclockwise(src)
    d2, U2 = F.cycleanticlockwise(d1)
    assert d2.trees == src.trees and np.abs(U2 @ U1 - I).max() <= 1e-13
    # a full turn of N clockwise rotations is the identity too
    dst, U = src, I
    for _ in range(5):
        dst, Ut = F.cycleclockwise(dst)
        U = Ut @ U
    assert dst.trees == src.trees and np.abs(U - I).max() <= 1e-12


def test_multi_fmove_inverse_pair():
    """multi_Fmove_inv(a, b, ·) undoes multi_Fmove: recoupling the first leg off and back on
    gives the original tree with coefficient 1 (summed over the intermediate trees)."""
    for f in F.fusiontrees(tuple((s,) for s in _su2(0.5, 1, 0.5, 1.5)), SU2Irrep(1.5), (False, True, False, True)):
        back = {}
        for fp, c1 in F.multi_Fmove(f):
            for g, c2 in F.multi_Fmove_inv(f.uncoupled[0], f.coupled, fp, f.isdual[0]):
                back[g] = back.get(g, 0.0) + c1 * c2
        for g, c in back.items():
            assert abs(c - (1.0 if g == f else 0.0)) <= 1e-13


@pytest.mark.parametrize("spaces", [VU1, VSU2, VU1SU2], ids=["U1", "SU2", "U1xSU2"])
def test_transpose_tables_match_braid_tables(spaces):
    for nd in range(0, 6):
        W = to_hom(five_leg(spaces(), ndom=nd))
        n1, n2 = W.numout(), W.numin()
        levels = (tuple(range(1, n1 + 1)), tuple(range(n1 + 1, n1 + n2 + 1)))
        for p in _cyclic_perms(n1, n2):
            Wd = W.permute(p)
            ft = flatten_transformer(treetransposer(Wd, W, p), p)
            fb = flatten_transformer(treebraider(Wd, W, p, levels), p)
            for name in ("perm", "group_src_ptr", "group_dst_ptr", "coeff_ptr", "sizes", "src_strides",
                         "src_offsets", "dst_strides", "dst_offsets"):
                assert np.array_equal(getattr(ft, name), getattr(fb, name)), (nd, p, name)
            assert np.abs(ft.coeffs - fb.coeffs).max(initial=0.0) <= 1e-13, (nd, p)
