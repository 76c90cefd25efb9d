"""Build libtkb200.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
from __future__ import annotations

import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "csrc")
LIBDIR = os.path.join(ROOT, "lib")
SOURCES = ["capi.cu", "transform.cu", "trace.cu", "gemm_f64.cu", "gemm_split.cu", "reduce.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES] + [
        os.path.join(CSRC, "tkb_internal.h"),
        os.path.join(os.path.dirname(ROOT), "include", "tkb200.h")]


def build(force: bool = False, verbose: bool = False, timeline: bool = False) -> str:
    """Compile every translation unit in parallel (one nvcc per file), then link the .so.

    timeline: build libtkb200_timeline.so instead, with the fused split kernel's global-timer
    stamps compiled in (read back with tkb_timeline_read); the default library has none."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libtkb200_timeline.so" if timeline else "libtkb200.so")
    if not force and os.path.exists(out):
        newest = max(os.path.getmtime(s) for s in sources())
        if os.path.getmtime(out) >= newest:
            return out
    objdir = os.path.join(LIBDIR, "obj_timeline" if timeline else "obj")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"] + (["-DTKB_TIMELINE"] if timeline else [])

    def compile_one(src):
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc()] + compile_flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", out] + objs
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, timeline="--timeline" in sys.argv))
