"""Checks shared by the host and device factorization tests (tests/test_factor_cpu.py,
tests/test_gpu_factor.py): blockwise SVD/QR/LQ/eigh against numpy per block, and the
sector-aware truncation strategies against the oracle's restatement of
src/factorizations/truncation.jl. Tolerance 1e-12 relative (max-norm)."""
import numpy as np

from helpers import O, cfg1_spaces, cfg2_spaces, from_sector, to_hom
import tensorkit_b200 as tk
from oracle import factor as F

TOL = 1e-12


def _tm(ot, device):
    import torch
    return tk.TensorMap(torch.from_numpy(np.ascontiguousarray(ot.data)).to(device), to_hom(ot.W))


def cases(cplx=False):
    V1, P1 = cfg1_spaces()
    V2, P2 = cfg2_spaces()
    return [(O.randn(O.Hom([V1, P1], [V1]), 0, cplx), True), (O.randn(O.Hom([V2, P2], [V2]), 1, cplx), False)]


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _np(x):
    return x.detach().cpu().numpy()


def check_svd(device, cplx):
    for ot, _ in cases(cplx):
        t = _tm(ot, device)
        U, S, Vh = tk.svd_compact(t)
        ov = F.svd_vals(ot)
        sv = tk.svd_vals(t)
        for c in t.blocksectors():
            oc = from_sector(c)
            b = ot.block(oc)
            u, s, vh = _np(U.block(c)), _np(S.block(c)), _np(Vh.block(c))
            assert _rel(u @ s @ vh, b) <= TOL
            assert _rel(u.conj().T @ u, np.eye(u.shape[1])) <= TOL
            assert _rel(np.diag(s), ov[oc]) <= TOL and _rel(_np(sv[c]), ov[oc]) <= TOL
        assert U.space.codomain == t.space.codomain and Vh.space.domain == t.space.domain


def check_truncation(device):
    for ot, unique in cases():
        t = _tm(ot, device)
        ov = F.svd_vals(ot)
        norm = F.vnorm(ov)
        smin = min(v.min() for v in ov.values())
        strategies = [
            (tk.truncrank(37), F.truncrank(ov, 37, unique)),
            (tk.trunctol(atol=0.5 * (smin + norm / 40)), F.trunctol(ov, atol=0.5 * (smin + norm / 40))),
            (tk.trunctol(rtol=0.05), F.trunctol(ov, rtol=0.05)),
            (tk.truncerror(rtol=0.3), F.truncerror(ov, rtol=0.3)),
            (tk.truncerror(atol=0.2 * norm), F.truncerror(ov, atol=0.2 * norm)),
        ]
        for strat, okept in strategies:
            U, S, Vh, err = tk.svd_trunc(t, strat)
            want = {c: int(m.sum()) for c, m in okept.items()}
            got = {from_sector(c): S.space.domain[0].dim(c) for c in t.blocksectors()}
            assert got == want, (type(strat).__name__, got, want)
            oerr = F.truncation_error(ov, okept)
            assert abs(err - oerr) <= TOL * max(norm, 1.0)
            # the kept part is the best rank-k approximation block by block
            for c in S.blocksectors():
                oc = from_sector(c)
                k = want[oc]
                assert _rel(np.diag(_np(S.block(c))), ov[oc][:k]) <= TOL
        # intersection and union of two strategies
        a, b = tk.truncrank(50), tk.trunctol(rtol=0.08)
        ka, kb = F.truncrank(ov, 50, unique), F.trunctol(ov, rtol=0.08)
        for strat, op in ((a & b, np.logical_and), (a | b, np.logical_or)):
            _, S, _, _ = tk.svd_trunc(t, strat)
            want = {c: int(op(ka[c], kb[c]).sum()) for c in ov}
            got = {from_sector(c): S.space.domain[0].dim(c) for c in t.blocksectors()}
            assert got == want
        # truncspace: at most dim(V, c) per sector
        Vt = tk.Vect({c: 3 for c in t.blocksectors()})
        _, S, _, _ = tk.svd_trunc(t, tk.truncspace(Vt))
        assert all(S.space.domain[0].dim(c) == min(3, len(ov[from_sector(c)])) for c in t.blocksectors())


def check_qr_lq(device, cplx):
    for ot, _ in cases(cplx):
        t = _tm(ot, device)
        Q, R = tk.qr_compact(t)
        L, Q2 = tk.lq_compact(t)
        for c in t.blocksectors():
            b = ot.block(from_sector(c))
            q, r = _np(Q.block(c)), _np(R.block(c))
            assert _rel(q @ r, b) <= TOL and np.allclose(np.tril(r, -1), 0)
            assert _rel(q.conj().T @ q, np.eye(q.shape[1])) <= TOL
            l, q2 = _np(L.block(c)), _np(Q2.block(c))
            assert _rel(l @ q2, b) <= TOL and np.allclose(np.triu(l, 1), 0)
            assert _rel(q2 @ q2.conj().T, np.eye(q2.shape[0])) <= TOL


def check_eigh(device, cplx):
    V2, _ = cfg2_spaces()
    oa = O.randn(O.Hom([V2], [V2]), 7, cplx)
    h = {c: b + b.conj().T for c, b in oa.blocks().items()}
    data = oa.data.copy()
    ot = O.BT(oa.W, data)
    for c, b in h.items():
        ot.block(c)[...] = b
    t = _tm(ot, device)
    D, V = tk.eigh_full(t)
    ow = F.eigh_vals(ot)
    for c in t.blocksectors():
        oc = from_sector(c)
        d, v = _np(D.block(c)), _np(V.block(c))
        assert _rel(v @ d @ v.conj().T, ot.block(oc)) <= TOL
        assert _rel(np.diag(d), ow[oc]) <= TOL
    # truncation keeps the largest |eigenvalue| first
    D, V, err = tk.eigh_trunc(t, tk.truncrank(40))
    okept = F.truncrank(ow, 40, False)
    got = {from_sector(c): D.space.domain[0].dim(c) for c in t.blocksectors()}
    assert got == {c: int(m.sum()) for c, m in okept.items()}
    assert abs(err - F.truncation_error(ow, okept)) <= TOL * F.vnorm(ow)
