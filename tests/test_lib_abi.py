"""The C-ABI library loads and exports every symbol declared in include/tkb200.h (no GPU
compute is called here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "tkb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tkb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("tkb_ctx_create", "tkb_table_create", "tkb_treetransform", "tkb_gemm_plan_create",
              "tkb_grouped_gemm", "tkb_reduce", "tkb_graph_begin"):
        assert s in syms


def test_library_exports_all_declared_symbols():
    from tensorkit_b200 import _build, _lib
    path = _build.build()
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(declared_symbols())


def test_version_and_error_without_device():
    from tensorkit_b200 import _build, _lib
    _build.build()
    lib = _lib.load()
    assert lib.tkb_version() >= 100
    # a null handle is rejected on the host, before any device call
    assert lib.tkb_treetransform(None, None, 0, None, None, _lib.tkb_scalar(1, 0),
                                 _lib.tkb_scalar(0, 0), 0) == _lib.TKB_ERR_ARG
    assert b"null" in lib.tkb_last_error(None)
