"""The C-ABI library: exports every entry point include/blgpu.h declares,
and the Python binding declares the same set (no GPU needed to load)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "blgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(blgpu_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("blgpu_create", "blgpu_advance", "blgpu_projection", "blgpu_compute_rhs", "blgpu_apply_bc"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from blgpu import _build
    if not os.path.exists(_build.LIB_PATH):
        pytest.skip("libblgpu.so not built")
    lib = ctypes.CDLL(_build.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from blgpu import _lib
    assert set(declared()) == set(_lib.exported_symbols())


def test_create_without_device_fails_cleanly():
    """No CUDA device here: create returns an error code and a message."""
    from blgpu import _build, _lib
    if not os.path.exists(_build.LIB_PATH):
        pytest.skip("libblgpu.so not built")
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    lib = _lib.load()
    cfg = _lib.Config(32, 16, 16, 1e-3, -1e-3, 0.0, 0.0, 3, 0, 0, 0, 0)
    h = ctypes.c_void_p()
    rc = lib.blgpu_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc != 0 and not h.value
    assert lib.blgpu_last_error(None)


def test_bad_config_rejected():
    from blgpu import _build, _lib
    if not os.path.exists(_build.LIB_PATH):
        pytest.skip("libblgpu.so not built")
    lib = _lib.load()
    h = ctypes.c_void_p()
    cfg = _lib.Config(3, 16, 16, 1e-3, -1e-3, 0.0, 0.0, 3, 0, 0, 0, 0)
    assert lib.blgpu_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    assert b"too small" in lib.blgpu_last_error(None)
    cfg = _lib.Config(32, 16, 16, 1e-3, -1e-3, 0.0, 0.0, 4, 0, 0, 0, 0)
    assert lib.blgpu_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
