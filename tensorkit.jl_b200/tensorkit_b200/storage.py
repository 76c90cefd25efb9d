"""Conversion between device tensors and plain host dictionaries, for writing to and reading
from disk (checkpoints of environments and the like).

Follows `Base.convert(::Type{Dict}, t)` / `Base.convert(::Type{TensorMap}, d)` in
`src/tensors/tensor.jl:433-462`: the dictionary holds the codomain and domain as strings and
the data as one dense host array per coupled sector, keyed by the sector's string form
(`repr(c)`), so the stored arrays are plain column-major matrices and do not depend on the
device layout. Where the reference re-parses its strings with `eval`, this module adds a
structured form of the spaces (`:structure`: sector type, sectors, degeneracies, duality) and
rebuilds the spaces from it; the string forms are kept for readers of the file.

`save` / `load` write such a dictionary to a NumPy `.npz` archive (blocks as arrays, the rest
as a JSON header).
"""
from __future__ import annotations

import json

import numpy as np

from .sectors import ProductSector, SU2Irrep, U1Irrep
from .spaces import GradedSpace, HomSpace, ProductSpace
from .tensor import AdjointTensorMap, TensorMap

__all__ = ["to_dict", "from_dict", "save", "load"]


def _sector_desc(c):
    if isinstance(c, U1Irrep):
        return ["U1", int(c.q2)]
    if isinstance(c, SU2Irrep):
        return ["SU2", int(c.j2)]
    if isinstance(c, ProductSector):
        return ["Prod", [_sector_desc(s) for s in c.sectors]]
    raise TypeError(f"sector type {type(c).__name__} has no stored form")


def _sector_from(d):
    kind = d[0]
    if kind == "U1":
        return U1Irrep(twice=int(d[1]))
    if kind == "SU2":
        return SU2Irrep(twice=int(d[1]))
    if kind == "Prod":
        return ProductSector(*(_sector_from(x) for x in d[1]))
    raise ValueError(f"unknown stored sector kind {kind!r}")


def _space_desc(V: GradedSpace):
    return {"dual": bool(V.isdual()),
            "dims": [[_sector_desc(c), int(d)] for c, d in zip(V._keys, V._degs)]}


def _space_from(d, unit):
    return GradedSpace({_sector_from(c): n for c, n in d["dims"]}, dual=bool(d["dual"]), unit=unit)


def _structure(W: HomSpace):
    return {"unit": _sector_desc(W.unit()),
            "codomain": [_space_desc(V) for V in W.codomain],
            "domain": [_space_desc(V) for V in W.domain]}


def _homspace_from(s):
    unit = _sector_from(s["unit"])
    cod = ProductSpace(tuple(_space_from(d, unit) for d in s["codomain"]), unit)
    dom = ProductSpace(tuple(_space_from(d, unit) for d in s["domain"]), unit)
    return HomSpace(cod, dom, unit)


def to_dict(t) -> dict:
    """`convert(Dict, t)`: codomain, domain (strings), the structured spaces, and one dense host
    array per coupled sector (every block is copied to the host)."""
    if isinstance(t, AdjointTensorMap):
        raise TypeError("store the parent tensor (a lazy adjoint has no data of its own)")
    W = t.space
    data = {repr(c): np.array(b.detach().cpu().numpy(), order="F") for c, b in t.blocks().items()}
    return {"codomain": repr(W.codomain), "domain": repr(W.domain), "structure": _structure(W),
            "data": data}


def from_dict(d: dict, device=None, dtype=None) -> TensorMap:
    """`convert(TensorMap, d)`: rebuild the spaces and copy every block to `device`. A coupled
    sector missing from `d["data"]` is zero; a block whose shape differs from the space's is an
    error."""
    import torch
    W = _homspace_from(d["structure"])
    blocks = d["data"]
    if dtype is None:
        cplx = any(np.iscomplexobj(b) for b in blocks.values())
        dtype = torch.complex128 if cplx else torch.float64
    t = TensorMap.zeros(W, dtype=dtype, device=device)
    known = {repr(c): c for c in t.blocksectors()}
    for key, b in blocks.items():
        if key not in known:
            raise ValueError(f"stored block {key} is not a coupled sector of {W}")
        dst = t.block(known[key])
        arr = np.asarray(b)
        if tuple(arr.shape) != tuple(dst.shape):
            raise ValueError(f"stored block {key} has shape {arr.shape}, the space needs {tuple(dst.shape)}")
        dst.copy_(torch.from_numpy(np.ascontiguousarray(arr)).to(device=dst.device, dtype=dtype))
    return t


def save(path, t) -> None:
    """Write `to_dict(t)` to a NumPy `.npz` archive."""
    d = to_dict(t)
    keys = list(d["data"].keys())
    header = {"codomain": d["codomain"], "domain": d["domain"], "structure": d["structure"],
              "blocks": keys}
    arrays = {f"block{i}": d["data"][k] for i, k in enumerate(keys)}
    np.savez(path, header=np.frombuffer(json.dumps(header).encode(), dtype=np.uint8), **arrays)


def load(path, device=None, dtype=None) -> TensorMap:
    """Read an archive written by `save` back into a tensor on `device`."""
    with np.load(path, allow_pickle=False) as z:
        header = json.loads(bytes(z["header"]).decode())
        data = {k: z[f"block{i}"] for i, k in enumerate(header["blocks"])}
    d = {"codomain": header["codomain"], "domain": header["domain"],
         "structure": header["structure"], "data": data}
    return from_dict(d, device=device, dtype=dtype)
