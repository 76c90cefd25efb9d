"""Sector types for the symmetric-contraction path: U(1) irreps, SU(2) irreps and their
Deligne product (U1Irrep ⊠ SU2Irrep).

Each sector exposes the interface TensorKit's fusion-tree code reads
(TensorKitSectors, the external package named at `src/TensorKit.jl:127-130`):
`unit`, `dual`, `dim`, ordering (`isless`), `otimes` (the fusion product ⊗ in the
reference's iteration order), `Nsymbol`, `Fsymbol`, `Rsymbol`, `Bsymbol`,
`frobenius_schur_phase` and `twist`.

Conventions restated from the reference documentation:
- U1Irrep ordering `isless(|q1|,|q2|) || 0 < q1 == -q2`  (`docs/src/man/sectors.md:262-264`),
  i.e. 0, 1, -1, 2, -2, ...; all F, R, A, B symbols are 1 (`sectors.md:243-245`).
- SU2Irrep ordering by spin, ⊗ iterates j = |ja-jb| .. ja+jb (`sectors.md:367-376`);
  F = sqrtdim(s5)*sqrtdim(s6)*racahW(s1,s2,s4,s3,s5,s6) (`sectors.md:382-395`);
  R = (-1)^(ja+jb-jc) (`sectors.md:396-400`); scalar type Float64 (`sectors.md:379`).
- Bsymbol(a,b,c) = sqrt(da*db/dc) * F^{a b b̄}_a[c, 1] (`docs/src/appendix/categories.md:590-593`).

SU(2) Racah coefficients are evaluated exactly with rational arithmetic (the Racah
single-sum formula) and rounded once to float64, so every F-symbol is the correctly
rounded value of the exact coefficient times the two square roots, multiplied in the
order the reference writes it.
"""
from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

__all__ = [
    "Sector", "U1Irrep", "SU2Irrep", "ProductSector", "Nsymbol", "Fsymbol", "Rsymbol",
    "Bsymbol", "frobenius_schur_phase", "twist", "sqrtdim", "invsqrtdim",
]


class Sector:
    """Base class: hashable, totally ordered sector label."""
    __slots__ = ()
    fusionstyle = "unique"      # "unique" | "simple" (multiplicity-free)

    def __lt__(self, other):
        return self.sortkey() < other.sortkey()

    def __le__(self, other):
        return self.sortkey() <= other.sortkey()

    def __gt__(self, other):
        return self.sortkey() > other.sortkey()

    def __ge__(self, other):
        return self.sortkey() >= other.sortkey()

    def isunit(self) -> bool:
        return self == self.unit()


# ----------------------------------------------------------------------------------------
# U(1)
# ----------------------------------------------------------------------------------------
class U1Irrep(Sector):
    """U(1) irrep; `charge` may be half-integer, stored as twice its value."""
    __slots__ = ("q2", "_h")
    fusionstyle = "unique"

    def __init__(self, charge=0, *, twice=None):
        q2 = int(twice) if twice is not None else int(round(2 * Fraction(charge)))
        object.__setattr__(self, "q2", q2)
        object.__setattr__(self, "_h", hash(("U1", q2)))

    @property
    def charge(self):
        return self.q2 // 2 if self.q2 % 2 == 0 else Fraction(self.q2, 2)

    def __eq__(self, o):
        return type(o) is U1Irrep and o.q2 == self.q2

    def __hash__(self):
        return self._h

    def __repr__(self):
        return f"U1Irrep({self.charge})"

    def sortkey(self):
        # isless(abs(q1), abs(q2)) || 0 < q1 == -q2 : positive charge before negative
        return (abs(self.q2), self.q2 < 0)

    @staticmethod
    def unit():
        return _U1_ZERO

    def dual(self):
        return U1Irrep(twice=-self.q2)

    def dim(self):
        return 1

    def otimes(self, other):
        return (U1Irrep(twice=self.q2 + other.q2),)


_U1_ZERO = U1Irrep(0)


# ----------------------------------------------------------------------------------------
# SU(2)
# ----------------------------------------------------------------------------------------
class SU2Irrep(Sector):
    """SU(2) irrep of spin j (integer or half-integer), stored as twice its value."""
    __slots__ = ("j2", "_h")
    fusionstyle = "simple"

    def __init__(self, j=0, *, twice=None):
        j2 = int(twice) if twice is not None else int(round(2 * Fraction(j)))
        if j2 < 0:
            raise ValueError("Not a valid SU₂ irrep")
        object.__setattr__(self, "j2", j2)
        object.__setattr__(self, "_h", hash(("SU2", j2)))

    @property
    def j(self):
        return self.j2 // 2 if self.j2 % 2 == 0 else Fraction(self.j2, 2)

    def __eq__(self, o):
        return type(o) is SU2Irrep and o.j2 == self.j2

    def __hash__(self):
        return self._h

    def __repr__(self):
        return f"SU2Irrep({self.j})"

    def sortkey(self):
        return (self.j2,)

    @staticmethod
    def unit():
        return _SU2_ZERO

    def dual(self):
        return self

    def dim(self):
        return self.j2 + 1

    def otimes(self, other):
        lo = abs(self.j2 - other.j2)
        hi = self.j2 + other.j2
        return tuple(SU2Irrep(twice=t) for t in range(lo, hi + 1, 2))


_SU2_ZERO = SU2Irrep(0)


# ----------------------------------------------------------------------------------------
# Deligne product
# ----------------------------------------------------------------------------------------
class ProductSector(Sector):
    """Deligne product `a ⊠ b ⊠ ...` of sectors; symbols are componentwise products."""
    __slots__ = ("sectors", "_h")

    def __init__(self, *sectors):
        object.__setattr__(self, "sectors", tuple(sectors))
        object.__setattr__(self, "_h", hash(("P",) + self.sectors))

    @property
    def fusionstyle(self):
        return "unique" if all(s.fusionstyle == "unique" for s in self.sectors) else "simple"

    def __eq__(self, o):
        return type(o) is ProductSector and o.sectors == self.sectors

    def __hash__(self):
        return self._h

    def __repr__(self):
        return " ⊠ ".join(repr(s) for s in self.sectors)

    def sortkey(self):
        # lexicographic on the first differing component
        return tuple(s.sortkey() for s in self.sectors)

    def unit(self):
        return ProductSector(*(s.unit() for s in self.sectors))

    def dual(self):
        return ProductSector(*(s.dual() for s in self.sectors))

    def dim(self):
        d = 1
        for s in self.sectors:
            d *= s.dim()
        return d

    def otimes(self, other):
        # Iterators.product semantics: first component varies fastest
        outs = [a.otimes(b) for a, b in zip(self.sectors, other.sectors)]
        res = _product_first_fastest(outs)
        return tuple(ProductSector(*r) for r in res)


def _product_first_fastest(lists):
    out = []
    n = len(lists)
    idx = [0] * n
    if any(len(l) == 0 for l in lists):
        return out
    while True:
        out.append(tuple(lists[k][idx[k]] for k in range(n)))
        k = 0
        while k < n:
            idx[k] += 1
            if idx[k] < len(lists[k]):
                break
            idx[k] = 0
            k += 1
        if k == n:
            return out


def fusionstyle(s: Sector) -> str:
    return s.fusionstyle


# ----------------------------------------------------------------------------------------
# Symbols
# ----------------------------------------------------------------------------------------
def Nsymbol(a, b, c) -> int:
    if isinstance(a, U1Irrep):
        return int(a.q2 + b.q2 == c.q2)
    if isinstance(a, SU2Irrep):
        return int(_su2_delta(a.j2, b.j2, c.j2))
    if isinstance(a, ProductSector):
        n = 1
        for x, y, z in zip(a.sectors, b.sectors, c.sectors):
            n *= Nsymbol(x, y, z)
        return n
    raise TypeError(type(a))


def _su2_delta(a2, b2, c2) -> bool:
    return (c2 <= a2 + b2) and (c2 >= abs(a2 - b2)) and ((a2 + b2 + c2) % 2 == 0)


def sqrtdim(a) -> float:
    return 1.0 if a.fusionstyle == "unique" else math.sqrt(a.dim())


def invsqrtdim(a) -> float:
    return 1.0 if a.fusionstyle == "unique" else 1.0 / math.sqrt(a.dim())


def _fact(n: int) -> int:
    return math.factorial(n)


@lru_cache(maxsize=None)
def _racah_w_exact(a2, b2, c2, d2, e2, f2):
    """Exact Racah W(a b c d; e f) as (sign, Fraction squared magnitude).

    W(a b c d; e f) = (-1)^(a+b+c+d) {a b e; d c f}; the 6j symbol is evaluated with the
    Racah single-sum formula (all arguments are given as twice their value)."""
    # 6j {j1 j2 j3; j4 j5 j6} with j1=a, j2=b, j3=e, j4=d, j5=c, j6=f
    j1, j2, j3, j4, j5, j6 = a2, b2, e2, d2, c2, f2
    triads = ((j1, j2, j3), (j1, j5, j6), (j4, j2, j6), (j4, j5, j3))
    for x, y, z in triads:
        if not _su2_delta(x, y, z):
            return 0, Fraction(0)

    def delta2(x, y, z):  # Δ(xyz)^2 with twice-values
        return Fraction(_fact((x + y - z) // 2) * _fact((x - y + z) // 2) * _fact((-x + y + z) // 2),
                        _fact((x + y + z) // 2 + 1))

    pref = Fraction(1)
    for t in triads:
        pref *= delta2(*t)
    alphas = [(x + y + z) // 2 for (x, y, z) in triads]
    betas = [(j1 + j2 + j4 + j5) // 2, (j2 + j3 + j5 + j6) // 2, (j3 + j1 + j6 + j4) // 2]
    tmin = max(alphas)
    tmax = min(betas)
    s = 0
    for t in range(tmin, tmax + 1):
        num = _fact(t + 1)
        den = 1
        for al in alphas:
            den *= _fact(t - al)
        for be in betas:
            den *= _fact(be - t)
        term = Fraction(num, den)
        s += -term if (t % 2) else term
    s = Fraction(s)
    if s == 0:
        return 0, Fraction(0)
    sign6j = 1 if s > 0 else -1
    # phase (-1)^(a+b+c+d)
    ph = (a2 + b2 + c2 + d2) // 2
    sign = sign6j * (-1 if ph % 2 else 1)
    return sign, pref * s * s


def _sqrt_fraction_rounded(x: Fraction) -> float:
    """Correctly rounded float64 of sqrt(x) for a non-negative rational x."""
    if x == 0:
        return 0.0
    p, q = x.numerator, x.denominator
    # sqrt(p/q) = sqrt(p*q)/q ; compute with 2*K extra bits
    K = 140
    r = math.isqrt(p * q << (2 * K))
    exact = (r * r == (p * q << (2 * K)))
    val = Fraction(r, q << K)
    if not exact:
        # r is the floor; nudge by half a unit of the extended precision so that float()
        # rounds the interval midpoint (the true value lies in [r, r+1))
        val += Fraction(1, (q << K) * 2)
    return float(val)


@lru_cache(maxsize=None)
def racahW(a2, b2, c2, d2, e2, f2) -> float:
    """float64 Racah W coefficient (arguments twice the spins), correctly rounded."""
    sign, mag2 = _racah_w_exact(a2, b2, c2, d2, e2, f2)
    if sign == 0:
        return 0.0
    return sign * _sqrt_fraction_rounded(mag2)


@lru_cache(maxsize=None)
def _su2_F(s1, s2, s3, s4, s5, s6) -> float:
    if s1 == s2 == s3 == s4 == s5 == s6 == 0:
        return 1.0
    for (x, y, z) in ((s1, s2, s5), (s5, s3, s4), (s2, s3, s6), (s1, s6, s4)):
        if not _su2_delta(x, y, z):
            return 0.0
    return (math.sqrt(s5 + 1) * math.sqrt(s6 + 1)) * racahW(s1, s2, s4, s3, s5, s6)


def Fsymbol(a, b, c, d, e, f):
    """[F^{abc}_d]^e_f : recoupling (a⊗b→e)⊗c→d  into  a⊗(b⊗c→f)→d."""
    if isinstance(a, U1Irrep):
        return 1.0 if (Nsymbol(a, b, e) and Nsymbol(e, c, d) and Nsymbol(b, c, f)
                       and Nsymbol(a, f, d)) else 0.0
    if isinstance(a, SU2Irrep):
        return _su2_F(a.j2, b.j2, c.j2, d.j2, e.j2, f.j2)
    if isinstance(a, ProductSector):
        r = 1.0
        for comp in zip(a.sectors, b.sectors, c.sectors, d.sectors, e.sectors, f.sectors):
            r = r * Fsymbol(*comp)
        return r
    raise TypeError(type(a))


def Rsymbol(a, b, c):
    if isinstance(a, U1Irrep):
        return 1.0 if Nsymbol(a, b, c) else 0.0
    if isinstance(a, SU2Irrep):
        if not Nsymbol(a, b, c):
            return 0.0
        return 1.0 if ((a.j2 + b.j2 - c.j2) // 2) % 2 == 0 else -1.0
    if isinstance(a, ProductSector):
        r = 1.0
        for comp in zip(a.sectors, b.sectors, c.sectors):
            r = r * Rsymbol(*comp)
        return r
    raise TypeError(type(a))


def frobenius_schur_phase(a):
    if isinstance(a, U1Irrep):
        return 1.0
    if isinstance(a, SU2Irrep):
        return 1.0 if a.j2 % 2 == 0 else -1.0
    if isinstance(a, ProductSector):
        r = 1.0
        for s in a.sectors:
            r = r * frobenius_schur_phase(s)
        return r
    raise TypeError(type(a))


def twist(a):
    """Bosonic sectors: every twist is 1."""
    return 1.0


def Bsymbol(a, b, c):
    """B^{ab}_c = sqrtdim(a)*sqrtdim(b)*invsqrtdim(c) * F^{a b b̄}_a[c, 1]."""
    if a.fusionstyle == "unique":
        return 1.0 if Nsymbol(a, b, c) else 0.0
    return (sqrtdim(a) * sqrtdim(b) * invsqrtdim(c)) * Fsymbol(a, b, b.dual(), a, c, a.unit())


def Asymbol(a, b, c):
    """A^{ab}_c = sqrtdim(a)*sqrtdim(b)*invsqrtdim(c) * χ_ā * F^{ā a b}_b[1, c] (the folding
    coefficient; `docs/src/appendix/categories.md:590-593`, real for these sectors)."""
    if a.fusionstyle == "unique":
        return 1.0 if Nsymbol(a, b, c) else 0.0
    ad = a.dual()
    return ((sqrtdim(a) * sqrtdim(b) * invsqrtdim(c)) * frobenius_schur_phase(ad)
            * Fsymbol(ad, a, b, b, a.unit(), c))


def otimes_many(sectors, unit):
    """All coupled sectors of a tuple of sectors, as a list of unique values."""
    if len(sectors) == 0:
        return [unit]
    acc = [sectors[0]]
    for s in sectors[1:]:
        nxt = []
        seen = set()
        for a in acc:
            for c in a.otimes(s):
                if c not in seen:
                    seen.add(c)
                    nxt.append(c)
        acc = nxt
    return acc
