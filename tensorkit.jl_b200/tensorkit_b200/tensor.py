"""TensorMap with device storage and its lazy adjoint.

Mirrors `src/tensors/tensor.jl` (`TensorMap{T,S,N₁,N₂,A}`: one flat data vector + a
HomSpace, `:10-20`; `block(t, c)` = column-major reshape of a contiguous range, `:466-495`;
`subblock(t, (f₁, f₂))` = strided view, `:499-509`) and `src/tensors/adjoint.jl`
(`AdjointTensorMap`: `block` is the conjugate transpose of the parent's block, `subblock`
a conjugated permutedims view, `:28`, `:47-51`). Storage is a 1-D torch tensor on a CUDA
device (float64 or complex128) — the CuVector of `CuTensorMap`
(`ext/TensorKitCUDAExt/cutensormap.jl:1-8`).

Seeded random data: numpy `PCG64(seed)` standard normals drawn for the whole data vector
in block order (which is the reference's block-by-block fill order, `tensor.jl:420-425`);
complex entries are (x + i·y)/√2 from consecutive pairs.
"""
from __future__ import annotations

import numpy as np

from .spaces import HomSpace, SpaceMismatch
from .structure import blockstructure, degeneracystructure, sectorstructure, subblockstructure

__all__ = ["TensorMap", "AdjointTensorMap", "randn_tensor", "zeros_tensor", "space_randn_data",
           "new_tensor"]


def _torch():
    import torch
    return torch


# While a CUDA graph is being captured every buffer allocated for the network must outlive
# the capture (the graph replays into those addresses); allocations are logged here.
_ALLOC_LOG: list | None = None


def new_tensor(W: HomSpace, dtype, device) -> "TensorMap":
    torch = _torch()
    t = TensorMap(torch.empty(W.dim(), dtype=dtype, device=device), W)
    if _ALLOC_LOG is not None:
        _ALLOC_LOG.append(t.data)
    return t


def space_randn_data(W: HomSpace, seed: int, dtype="float64") -> np.ndarray:
    n = degeneracystructure(W).totaldim
    rng = np.random.Generator(np.random.PCG64(seed))
    if dtype in ("float64", np.float64):
        return rng.standard_normal(n)
    x = rng.standard_normal(2 * n).reshape(n, 2)
    return (x[:, 0] + 1j * x[:, 1]) / np.sqrt(2.0)


class AbstractTensorMap:
    def numout(self):
        return self.space.numout()

    def numin(self):
        return self.space.numin()

    def numind(self):
        return self.space.numind()

    def codomainind(self):
        return tuple(range(1, self.numout() + 1))

    def domainind(self):
        return tuple(range(self.numout() + 1, self.numind() + 1))

    def allind(self):
        return tuple(range(1, self.numind() + 1))

    @property
    def codomain(self):
        return self.space.codomain

    @property
    def domain(self):
        return self.space.domain

    def unit(self):
        return self.space.unit()


class TensorMap(AbstractTensorMap):
    __slots__ = ("data", "space")

    def __init__(self, data, space: HomSpace):
        if data.dim() != 1:
            raise ValueError("TensorMap data must be a flat vector")
        if data.numel() != space.dim():
            raise SpaceMismatch(f"data length {data.numel()} ≠ dim(space) {space.dim()}")
        self.data = data
        self.space = space

    # -- construction ----------------------------------------------------------------
    @staticmethod
    def zeros(space: HomSpace, dtype=None, device=None):
        torch = _torch()
        dtype = dtype or torch.float64
        return TensorMap(torch.zeros(space.dim(), dtype=dtype, device=device), space)

    @staticmethod
    def empty(space: HomSpace, dtype=None, device=None):
        torch = _torch()
        dtype = dtype or torch.float64
        return TensorMap(torch.empty(space.dim(), dtype=dtype, device=device), space)

    @staticmethod
    def from_numpy(arr: np.ndarray, space: HomSpace, device=None):
        torch = _torch()
        return TensorMap(torch.from_numpy(np.ascontiguousarray(arr)).to(device), space)

    @staticmethod
    def randn(space: HomSpace, seed: int = 0, dtype=None, device=None):
        torch = _torch()
        dtype = dtype or torch.float64
        npd = "float64" if dtype == torch.float64 else "complex128"
        return TensorMap.from_numpy(space_randn_data(space, seed, npd), space, device)

    def similar(self, dtype=None, space=None):
        torch = _torch()
        return TensorMap(torch.empty((space or self.space).dim(), dtype=dtype or self.data.dtype,
                                     device=self.data.device), space or self.space)

    def copy(self):
        return TensorMap(self.data.clone(), self.space)

    # -- properties --------------------------------------------------------------------
    @property
    def dtype(self):
        return self.data.dtype

    @property
    def device(self):
        return self.data.device

    def is_complex(self):
        return self.data.is_complex()

    def sectortype_unique(self):
        return self.unit().fusionstyle == "unique"

    def blocksectors(self):
        return sectorstructure(self.space).blocksectors

    def fusiontrees(self):
        return sectorstructure(self.space).fusiontrees

    def block(self, c):
        (d1, d2), (a, b) = blockstructure(self.space)[c]
        return self.data[a:b].view(d2, d1).transpose(0, 1)

    def blocks(self):
        bs = blockstructure(self.space)
        return {c: self.data[a:b].view(d2, d1).transpose(0, 1) for c, ((d1, d2), (a, b)) in bs.items()}

    def subblock(self, f1, f2=None):
        if f2 is None:
            f1, f2 = f1
        sz, st, off = subblockstructure(self.space)[(f1, f2)]
        return self.data.as_strided(sz, st, off)

    def to_host(self) -> np.ndarray:
        return self.data.detach().cpu().numpy()

    def adjoint(self):
        return AdjointTensorMap(self)

    @property
    def H(self):
        return AdjointTensorMap(self)

    def __repr__(self):
        return f"TensorMap({self.space!r}, dtype={self.data.dtype}, device={self.data.device})"

    # -- arithmetic conveniences (device kernels) ---------------------------------------
    def __matmul__(self, other):
        from .linalg import compose
        return compose(self, other)

    def norm(self):
        from .linalg import norm
        return norm(self)


class AdjointTensorMap(AbstractTensorMap):
    """Lazy adjoint: space(t') = adjoint(space(t)); no data is moved."""
    __slots__ = ("parent", "space")

    def __init__(self, parent: TensorMap):
        self.parent = parent
        self.space = parent.space.adjoint()

    @property
    def data(self):
        return self.parent.data

    @property
    def dtype(self):
        return self.parent.data.dtype

    @property
    def device(self):
        return self.parent.data.device

    def is_complex(self):
        return self.parent.data.is_complex()

    def adjoint(self):
        return self.parent

    def block(self, c):
        b = self.parent.block(c)
        return b.conj().transpose(0, 1) if b.is_complex() else b.transpose(0, 1)

    def __repr__(self):
        return f"adjoint({self.parent!r})"


def randn_tensor(space, seed=0, dtype=None, device=None):
    return TensorMap.randn(space, seed, dtype, device)


def zeros_tensor(space, dtype=None, device=None):
    return TensorMap.zeros(space, dtype, device)
