"""The C-ABI library loads and exports every entry point include/fullermd.h
declares; the Python binding declares a signature for each.  No compute
calls: these run on CPU-only machines."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def header_functions() -> list[str]:
    text = (ROOT / "include" / "fullermd.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmd_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = header_functions()
    for must in ("fmd_nlist_rigid", "fmd_nlist_lj_half", "fmd_nlist_rebo", "fmd_lj_rigid_forces",
                 "fmd_airebo_forces", "fmd_mm_forces", "fmd_rigid_step", "fmd_airebo_step", "fmd_mm_step",
                 "fmd_system_run"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from fuller_md_en_b200 import _lib
    if not _lib.LIB_PATH.exists():
        from fuller_md_en_b200 import build
        build.build_cuda()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_covers_header():
    from fuller_md_en_b200 import _lib
    assert set(header_functions()) <= set(_lib.exported_symbols())
    lib = _lib.load()   # declares argtypes for every symbol; raises if one is absent
    assert lib.fmd_version() >= 100
    assert lib.fmd_status_string(3) == b"capacity exceeded"


def test_no_device_is_an_error_not_a_crash():
    from fuller_md_en_b200 import _lib
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.fmd_ctx_create(ctypes.byref(h), 0)
    assert rc == _lib.FMD_ERR_CUDA and not h.value
