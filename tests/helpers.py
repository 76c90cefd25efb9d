"""Shared fixtures: the spaces of the five contraction workloads, the reference's own test
space lists (test/setup.jl:225-231 for U(1), :268-274 for SU(2)), and converters between
the oracle's representation and the product's."""
from __future__ import annotations

import math

import numpy as np

from oracle import core as O
import tensorkit_b200 as tk

U1, SU2, P = O.U1, O.SU2, O.P


# ---- converters ------------------------------------------------------------------------
def to_sector(s):
    if s[0] == "U1":
        return tk.U1Irrep(twice=s[1])
    if s[0] == "SU2":
        return tk.SU2Irrep(twice=s[1])
    return tk.ProductSector(*[to_sector(x) for x in s[1]])


def to_space(sp: O.Space):
    return tk.Vect({to_sector(s): d for s, d in sp.degs.items()}, sp.dual)


def to_hom(W: O.Hom):
    u = to_sector(W.unit())
    return tk.HomSpace(tk.ProductSpace([to_space(s) for s in W.cod], u),
                       tk.ProductSpace([to_space(s) for s in W.dom], u), u)


def from_sector(s):
    from tensorkit_b200 import sectors as S
    if isinstance(s, S.U1Irrep):
        return ("U1", s.q2)
    if isinstance(s, S.SU2Irrep):
        return ("SU2", s.j2)
    return ("P", tuple(from_sector(x) for x in s.sectors))


def from_space(sp):
    degs = {from_sector(c.dual() if sp.isdual() else c): sp.dim(c) for c in sp.sectors()}
    return O.Space(degs, sp.isdual())


def from_hom(W):
    return O.Hom([from_space(v) for v in W.codomain], [from_space(v) for v in W.domain],
                 from_sector(W.unit()))


def to_device(t: O.BT, device="cuda"):
    import torch
    return tk.TensorMap(torch.from_numpy(np.ascontiguousarray(t.data)).to(device), to_hom(t.W))


def to_oracle(t: "tk.TensorMap", W: O.Hom):
    return O.BT(W, t.data.detach().cpu().numpy())


def relerr(x, y):
    x = np.asarray(x)
    y = np.asarray(y)
    den = max(np.abs(y).max(), 1e-300) if y.size else 1.0
    return float(np.abs(x - y).max() / den) if y.size else 0.0


# ---- reference test spaces -------------------------------------------------------------
def VU1():
    return [O.Space({U1(0): 2, U1(1): 2, U1(-1): 2}), O.Space({U1(0): 1, U1(1): 1, U1(-1): 1}, True),
            O.Space({U1(0): 3, U1(1): 1, U1(-1): 1}), O.Space({U1(0): 1, U1(1): 2, U1(-1): 1}, True),
            O.Space({U1(0): 1, U1(1): 1, U1(-1): 2})]


def VSU2():
    return [O.Space({SU2(0): 3, SU2(.5): 1}), O.Space({SU2(0): 2, SU2(1): 1}, True),
            O.Space({SU2(.5): 1, SU2(1): 1}), O.Space({SU2(0): 2, SU2(.5): 2}, True),
            O.Space({SU2(0): 1, SU2(.5): 1, SU2(1.5): 1})]


def VU1SU2():
    a = lambda q, j: P(U1(q), SU2(j))
    return [O.Space({a(0, 0): 2, a(1, .5): 1, a(-1, .5): 1}), O.Space({a(0, 0): 1, a(0, 1): 1}, True),
            O.Space({a(1, .5): 1, a(-1, .5): 1, a(0, 0): 1}), O.Space({a(0, 0): 2, a(1, .5): 1}, True),
            O.Space({a(0, 0): 1, a(-1, .5): 1, a(0, 1): 1})]


def five_leg(VS, ndom=2):
    """V1⊗V2⊗V3 ← (V4⊗V5)' style HomSpace with `ndom` domain legs."""
    cod = VS[:5 - ndom]
    dom = [v.flipdual() for v in reversed(VS[5 - ndom:])]
    return O.Hom(cod, dom)


# ---- workload spaces -------------------------------------------------------------------
def cfg1_spaces():
    V = O.Space({U1(q): 8 for q in range(-3, 4)})
    Pp = O.Space({U1(q): 1 for q in (-1, 0, 1)})
    return V, Pp


def cfg2_spaces(mult=1):
    degs = [32, 48, 40, 24, 12, 6, 2]
    V = O.Space({SU2(j / 2): d * mult for j, d in enumerate(degs)})
    Pp = O.Space({SU2(0.5): 1})
    return V, Pp


def cfg3_spaces():
    V = O.Space({U1(q): max(1, int(round(256 * math.exp(-q * q / 18)))) for q in range(-10, 11)})
    Pp = O.Space({U1(0): 1, U1(1): 1})
    Wm = O.Space({U1(-1): 2, U1(0): 3, U1(1): 2})
    return V, Pp, Wm


def cfg5_spaces():
    degs = {}
    for q in range(-2, 3):
        for j2 in range(0, 4):
            degs[P(U1(q), SU2(j2 / 2))] = max(1, int(round(64 * math.exp(-(q * q + j2) / 4))))
    V = O.Space(degs)
    Pp = O.Space({P(U1(1), SU2(.5)): 1, P(U1(-1), SU2(.5)): 1})
    return V, Pp


def julia_round(x):
    """Julia's round: half to even (matches Python's round)."""
    return int(round(x))
