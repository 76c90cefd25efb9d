"""Autotuner of the grouped block GEMM, with an on-disk cache per (block structure, dtype, device).

The reference runs every block of a `mul!` through BLAS (src/tensors/linalg.jl:330-370) and caches
only its tree transformers per structure (src/tensors/treetransformers.jl:156-205,
src/auxiliary/caches.jl). Here a grouped GEMM has a few decisions that depend on the block
structure: the precision (plain FP64 DMMA, or int8 slices with the per-block slice count and the
FP64 check) and the work decomposition (how far the K loops are cut into pieces when the output
tiles alone would leave SMs idle: at most `max_pieces` pieces of at least `min_piece_steps` K
steps). The tuner times each candidate on the operands at hand, rejects candidates whose result
differs from the plain FP64 result by more than the tolerance, keeps the fastest, and records the
choice in a JSON cache keyed by a hash of the block shapes and ops, the dtype, the device name and
the library version. Another process with the same key reuses the choice without timing.

The cache file is `$TKB_TUNE_CACHE`, else `~/.cache/tensorkit_b200/gemm_tuning.json`.
"""
from __future__ import annotations

import hashlib
import json
import os
import tempfile

__all__ = ["CANDIDATES", "structure_key", "TuneCache", "select", "default_cache"]

# (precision, max_pieces, min_piece_steps); the first is the library's default decomposition
CANDIDATES = [
    ("plain", 8, 4), ("plain", 1, 4), ("plain", 4, 8), ("plain", 16, 2),
    ("split", 8, 4), ("split", 1, 4), ("split", 4, 8), ("split", 16, 2),
]
TOLERANCE = 1e-12


def structure_key(blocks, dtype_code, device_name, version) -> str:
    """Hash of what the choice depends on: per block (m, n, k, opA, opB), the dtype, the device
    name and the library version."""
    rows = [[int(b[0]), int(b[1]), int(b[2]), int(b[9]), int(b[10])] for b in blocks]
    payload = json.dumps({"blocks": rows, "dtype": int(dtype_code), "device": str(device_name),
                          "version": int(version)}, sort_keys=True)
    return hashlib.sha256(payload.encode()).hexdigest()


def default_cache():
    path = os.environ.get("TKB_TUNE_CACHE")
    if not path:
        path = os.path.join(os.path.expanduser("~"), ".cache", "tensorkit_b200", "gemm_tuning.json")
    return TuneCache(path)


class TuneCache:
    """A JSON file {key: record}; records are written atomically (temporary file + rename) and
    the file is re-read before every write, so concurrent processes lose no entries of each other
    except on an exact race."""

    def __init__(self, path):
        self.path = path
        self._mem = None

    def _load(self):
        try:
            with open(self.path) as f:
                data = json.load(f)
            return data if isinstance(data, dict) else {}
        except (OSError, ValueError):
            return {}

    def get(self, key):
        if self._mem is None:
            self._mem = self._load()
        return self._mem.get(key)

    def put(self, key, record):
        data = self._load()
        data[key] = record
        d = os.path.dirname(self.path) or "."
        os.makedirs(d, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=d, prefix=".gemm_tuning.")
        try:
            with os.fdopen(fd, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except Exception:
            try:
                os.unlink(tmp)
            except OSError:
                pass
            raise
        self._mem = data


def select(candidates, measure, tolerance=TOLERANCE):
    """measure(candidate) -> (microseconds, relative error against plain FP64 or None when it is
    the reference itself). Returns (best candidate, record with every timing)."""
    timings = {}
    best, best_us = None, float("inf")
    for c in candidates:
        us, err = measure(c)
        ok = err is None or err <= tolerance
        timings["/".join(map(str, c))] = {"us": us, "rel_err": err, "accepted": ok}
        if ok and us < best_us:
            best, best_us = c, us
    if best is None:
        raise RuntimeError("no GEMM candidate met the tolerance")
    return best, {"choice": list(best), "timings": timings}
