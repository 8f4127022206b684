"""The C-ABI library loads without a GPU and exports every entry point that
include/gsplat_b200.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

from conftest import PKG, ROOT

HEADER = os.path.join(ROOT, "include", "gsplat_b200.h")
LIB = os.path.join(PKG, "gsplatcu", "libgsplat_b200.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gsb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "gsb_splat_draw" in names and "gsb_project" in names
    assert len(names) >= 18


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.fail(f"{LIB} missing: run reparamgs-palette_b200/build.py")
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from gsplatcu import _lib
    assert set(declared()) <= set(_lib.exported_symbols())


def test_version_and_error_string_without_gpu():
    from gsplatcu import _lib
    L = _lib.lib()
    assert L.gsb_version() >= 100
    assert isinstance(L.gsb_last_error(), bytes)


def test_argument_errors_need_no_gpu():
    """Invalid sizes are rejected on the host before any CUDA call."""
    from gsplatcu import _lib
    L = _lib.lib()
    rc = L.gsb_sh2weight(10, None, 0, 5, 5, None, None, None, None, None, None)
    assert rc == _lib.GSB_ERR_INVALID_ARGUMENT
    assert b"1, 4, 9 or 16" in L.gsb_last_error()
    rc = L.gsb_sh2weight_fast(10, None, None, None, 0, 5, 4, 15, 1, None, None, None, None, None, None)
    assert rc == _lib.GSB_ERR_INVALID_ARGUMENT
    assert L.gsb_splat_state_bytes(-1, 5, 64, 64) == 0
    assert L.gsb_splat_state_bytes(1000, 9, 64, 64) == 0


def test_workspace_sizes_grow_with_problem():
    from gsplatcu import _lib
    L = _lib.lib()
    import ctypes
    a = L.gsb_splat_state_bytes(1000, 5, 1080, 1920)
    b = L.gsb_splat_state_bytes(100000, 5, 1080, 1920)
    assert 0 < a < b
    assert b >= 100000 * (8 + 4 + 4 + 64)
    plan = _lib.SplatPlan(50000, 20000, 0)
    s1 = L.gsb_splat_sort_bytes(1000, 1080, 1920, ctypes.byref(plan))
    plan = _lib.SplatPlan(50000, 1 << 25, 0)  # > 32 key bits -> 64-bit radix keys
    s2 = L.gsb_splat_sort_bytes(1000, 1080, 1920, ctypes.byref(plan))
    assert s2 > s1 > 50000 * 16
