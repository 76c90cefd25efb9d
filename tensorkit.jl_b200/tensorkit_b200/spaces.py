"""Graded vector spaces, tensor-product spaces and HomSpaces.

Mirrors the parts of TensorKit's space layer that the contraction path reads:
- `GradedSpace` (`src/spaces/gradedspace.jl`): sector => degeneracy, stored sorted by the
  sector order; `sectors(V)` maps every stored key through `dual` when `V` is dual
  (`gradedspace.jl:180-187`), `dim(V, c)` reads the key `dual(c)` for a dual space
  (`gradedspace.jl:96-101`), `axes(V, c)` is the dense index range (`gradedspace.jl:103-110`).
- `ProductSpace` (`src/spaces/productspace.jl`): `blocksectors` (`:147-170`), `fusiontrees`
  (`:178-183`), `hasblock`, `blockdim` (`:193-213`).
- `HomSpace` (`src/spaces/homspace.jl`): indexing `W[i]` (`:76-79`), `permute`/`select`
  (`:212-243`), `compose` (`:262-265`), `adjoint`/`dual` (`:22-27`), `_blocksectors`
  (`:104-126`).

Leg indices in the public API are 1-based, exactly as in TensorKit.
"""
from __future__ import annotations

from itertools import product as _iproduct

from .sectors import Sector, otimes_many

__all__ = ["GradedSpace", "Vect", "ProductSpace", "HomSpace", "SpaceMismatch", "otimes",
           "product_sectors"]


class SpaceMismatch(ValueError):
    """Raised when spaces of tensors do not match (TensorKit's `SpaceMismatch`)."""


class GradedSpace:
    """⨁_c ℂ^{n_c} ⊗ R_c for sectors c of one sector type."""
    __slots__ = ("_keys", "_degs", "dual_flag", "_unit", "_h", "_sectors", "_dimmap")

    def __init__(self, dims, dual: bool = False, unit: Sector | None = None):
        items = list(dims.items()) if isinstance(dims, dict) else list(dims)
        items = [(c, int(d)) for (c, d) in items if int(d) > 0]
        items.sort(key=lambda cd: cd[0].sortkey())
        for i in range(1, len(items)):
            if items[i][0] == items[i - 1][0]:
                raise ValueError("duplicate sector in GradedSpace")
        self._keys = tuple(c for c, _ in items)
        self._degs = tuple(d for _, d in items)
        self.dual_flag = bool(dual)
        if unit is None:
            if not items:
                raise ValueError("empty GradedSpace needs an explicit unit sector")
            unit = items[0][0].unit()
        self._unit = unit
        self._h = hash((self._keys, self._degs, self.dual_flag))
        self._sectors = tuple(c.dual() for c in self._keys) if self.dual_flag else self._keys
        self._dimmap = dict(zip(self._keys, self._degs))

    # -- basic queries ----------------------------------------------------------------
    def sectors(self):
        return self._sectors

    def unit(self):
        return self._unit

    def isdual(self) -> bool:
        return self.dual_flag

    def dim(self, c: Sector | None = None) -> int:
        if c is None:
            return sum(s.dim() * self.dim(s) for s in self._sectors)
        key = c.dual() if self.dual_flag else c
        return self._dimmap.get(key, 0)

    def axes(self, c: Sector) -> range:
        off = 0
        for s in self._sectors:
            if s == c:
                break
            off += s.dim() * self.dim(s)
        return range(off, off + c.dim() * self.dim(c))

    def dual(self) -> "GradedSpace":
        return GradedSpace(list(zip(self._keys, self._degs)), not self.dual_flag, self._unit)

    conj = dual

    @property
    def T(self):  # convenience: V.T == V'
        return self.dual()

    def flip(self) -> "GradedSpace":
        if self.dual_flag:
            return GradedSpace({c: self.dim(c) for c in self._sectors}, False, self._unit)
        return GradedSpace({c.dual(): self.dim(c) for c in self._sectors}, False,
                           self._unit).dual()

    def __eq__(self, o):
        return (isinstance(o, GradedSpace) and o._keys == self._keys and o._degs == self._degs
                and o.dual_flag == self.dual_flag)

    def __hash__(self):
        return self._h

    def __repr__(self):
        body = ", ".join(f"{c!r}=>{d}" for c, d in zip(self._keys, self._degs))
        return f"Vect[{body}]" + ("'" if self.dual_flag else "")

    def __mul__(self, other):
        return otimes(self, other)

    def sectorhash_key(self):
        return (self._keys, self.dual_flag)


def Vect(dims, dual: bool = False, unit: Sector | None = None) -> GradedSpace:
    """`Vect[I](c => n, ...)` equivalent: Vect({c: n, ...})."""
    return GradedSpace(dims, dual, unit)


class ProductSpace:
    """Tensor product V₁ ⊗ ... ⊗ V_N of graded spaces (N may be 0)."""
    __slots__ = ("spaces", "_unit", "_h")

    def __init__(self, spaces, unit: Sector | None = None):
        self.spaces = tuple(spaces)
        if unit is None:
            if not self.spaces:
                raise ValueError("empty ProductSpace needs an explicit unit sector")
            unit = self.spaces[0].unit()
        self._unit = unit
        # the unit sector is part of the identity: spaces without legs of different sector
        # types (one(Vect[U1Irrep]) vs one(Vect[SU2Irrep])) must not compare equal
        self._h = hash(("PS", unit) + self.spaces)

    def __len__(self):
        return len(self.spaces)

    def __getitem__(self, i):
        return self.spaces[i]

    def __iter__(self):
        return iter(self.spaces)

    def __eq__(self, o):
        return isinstance(o, ProductSpace) and o.spaces == self.spaces and o._unit == self._unit

    def __hash__(self):
        return self._h

    def __repr__(self):
        if not self.spaces:
            return "one(S)"
        return " ⊗ ".join(repr(v) for v in self.spaces)

    def __mul__(self, other):
        return otimes(self, other)

    def unit(self):
        return self._unit

    def dims(self, uncoupled=None):
        if uncoupled is None:
            return tuple(v.dim() for v in self.spaces)
        return tuple(v.dim(s) for v, s in zip(self.spaces, uncoupled))

    def dim(self, uncoupled=None) -> int:
        r = 1
        for d in self.dims(uncoupled):
            r *= d
        return r

    def dual(self) -> "ProductSpace":
        return ProductSpace(tuple(v.dual() for v in reversed(self.spaces)), self._unit)

    def sectors(self):
        """Iterate over tuples of sectors, first space fastest (Iterators.product)."""
        return product_sectors([v.sectors() for v in self.spaces])

    def blocksectors(self):
        N = len(self.spaces)
        u = self._unit
        bs = []
        if N == 0:
            bs = [u]
        elif N == 1:
            bs = list(self.spaces[0].sectors())
        else:
            seen = set()
            for s in self.sectors():
                for c in otimes_many(s, u):
                    if c not in seen:
                        seen.add(c)
                        bs.append(c)
        bs.sort(key=lambda c: c.sortkey())
        return bs

    def fusiontrees(self, c):
        from .fusiontrees import fusiontrees
        return fusiontrees(tuple(v.sectors() for v in self.spaces), c,
                           tuple(v.isdual() for v in self.spaces))

    def hasblock(self, c) -> bool:
        for _ in self.fusiontrees(c):
            return True
        return False

    def blockdim(self, c) -> int:
        return sum(self.dim(f.uncoupled) for f in self.fusiontrees(c))

    def axes(self, uncoupled):
        return tuple(v.axes(s) for v, s in zip(self.spaces, uncoupled))


def product_sectors(lists):
    lists = [tuple(l) for l in lists]
    if not lists:
        yield ()
        return
    # Iterators.product: first factor varies fastest
    for combo in _iproduct(*reversed(lists)):
        yield tuple(reversed(combo))


def otimes(*args) -> ProductSpace:
    spaces = []
    unit = None
    for a in args:
        if isinstance(a, ProductSpace):
            spaces.extend(a.spaces)
            unit = unit or a.unit()
        else:
            spaces.append(a)
            unit = unit or a.unit()
    return ProductSpace(spaces, unit)


def _as_product(x, unit=None) -> ProductSpace:
    if isinstance(x, ProductSpace):
        return x
    if isinstance(x, GradedSpace):
        return ProductSpace((x,))
    if isinstance(x, (tuple, list)):
        return ProductSpace(tuple(x), unit)
    raise TypeError(type(x))


class HomSpace:
    """Space of morphisms codomain ← domain."""
    __slots__ = ("codomain", "domain", "_h")

    def __init__(self, codomain, domain, unit: Sector | None = None):
        cod = _as_product(codomain, unit)
        dom = _as_product(domain, unit if unit is not None else cod.unit())
        if unit is None and not cod.spaces and dom.spaces:
            cod = ProductSpace((), dom.unit())
        self.codomain = cod
        self.domain = dom
        self._h = hash((cod, dom))

    # -- structure ------------------------------------------------------------------
    def numout(self):
        return len(self.codomain)

    def numin(self):
        return len(self.domain)

    def numind(self):
        return len(self.codomain) + len(self.domain)

    def unit(self):
        return self.codomain.unit()

    def __getitem__(self, i):
        """1-based: W[i] is codomain[i] for i ≤ N₁, else dual(domain[i-N₁])."""
        n1 = len(self.codomain)
        if not 1 <= i <= self.numind():
            raise IndexError(i)
        return self.codomain[i - 1] if i <= n1 else self.domain[i - n1 - 1].dual()

    def __eq__(self, o):
        return isinstance(o, HomSpace) and o.codomain == self.codomain and o.domain == self.domain

    def __hash__(self):
        return self._h

    def __repr__(self):
        return f"{self.codomain!r} ← {self.domain!r}"

    def dims(self):
        return self.codomain.dims() + self.domain.dims()

    def adjoint(self) -> "HomSpace":
        return HomSpace(self.domain, self.codomain, self.unit())

    def dual(self) -> "HomSpace":
        return HomSpace(self.domain.dual(), self.codomain.dual(), self.unit())

    def select(self, p) -> "HomSpace":
        p1, p2 = p
        cod = ProductSpace(tuple(self[n] for n in p1), self.unit())
        dom = ProductSpace(tuple(self[n].dual() for n in p2), self.unit())
        return HomSpace(cod, dom, self.unit())

    def permute(self, p) -> "HomSpace":
        p1, p2 = p
        flat = tuple(p1) + tuple(p2)
        if sorted(flat) != list(range(1, self.numind() + 1)):
            raise ValueError(f"{p} is not a valid permutation for {self}")
        return self.select(p)

    def flip(self, I) -> "HomSpace":
        """The legs i ∈ I (1-based, codomain first) flipped: W′[i] = flip(W[i])."""
        I = {int(i) for i in I}
        n1 = len(self.codomain)
        if not all(1 <= i <= self.numind() for i in I):
            raise IndexError(f"flip: indices {sorted(I)} out of range for {self}")
        cod = ProductSpace(tuple(V.flip() if k + 1 in I else V for k, V in enumerate(self.codomain)), self.unit())
        dom = ProductSpace(tuple(V.flip() if n1 + k + 1 in I else V for k, V in enumerate(self.domain)),
                           self.unit())
        return HomSpace(cod, dom, self.unit())

    def compose(self, other: "HomSpace") -> "HomSpace":
        if self.domain != other.codomain:
            raise SpaceMismatch(f"{self.domain} ≠ {other.codomain}")
        return HomSpace(self.codomain, other.domain, self.unit())

    def blocksectors(self):
        from .structure import sectorstructure
        return sectorstructure(self).blocksectors

    def _blocksectors(self):
        cod, dom = self.codomain, self.domain
        n1, n2 = len(cod), len(dom)
        u = self.unit()
        if n1 == 0 and n2 == 0:
            return [u]
        if n1 == 0:
            return [c for c in dom.blocksectors() if c.isunit()]
        if n2 == 0:
            return [c for c in cod.blocksectors() if c.isunit()]
        if n2 <= n1:
            return [c for c in dom.blocksectors() if cod.hasblock(c)]
        return [c for c in cod.blocksectors() if dom.hasblock(c)]

    def dim(self) -> int:
        from .structure import degeneracystructure
        return degeneracystructure(self).totaldim

    def sectorkey(self):
        return (tuple(v.sectorhash_key() for v in self.codomain),
                tuple(v.sectorhash_key() for v in self.domain))
