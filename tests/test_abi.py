"""The C-ABI library loads (no GPU needed) and exports every entry point that
include/banshee_gpu.h declares; host-side error behaviour without a device."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = []
    for name in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            syms += re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(bg_\w+)\s*\(", text, re.M)
    return sorted(set(syms))


@pytest.fixture(scope="module")
def libso():
    from banshee_b200 import build
    path = build.build()
    return C.CDLL(path)


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ["bg_intersect_closest", "bg_intersect_any", "bg_scene_commit", "bg_render", "bg_last_error"]:
        assert s in syms


def test_library_exports_every_declared_symbol(libso):
    missing = [s for s in declared_symbols() if not hasattr(libso, s)]
    assert not missing, missing


def test_errors_without_device_or_arguments(libso):
    libso.bg_last_error.restype = C.c_char_p
    h = C.c_void_p()
    assert libso.bg_ctx_create(0, None) == -1                     # BG_ERR_INVALID_ARG
    rc = libso.bg_ctx_create(0, C.byref(h))
    import torch
    if not torch.cuda.is_available():
        assert rc == -8                                           # BG_ERR_NO_DEVICE
        assert b"device" in libso.bg_last_error()
    assert libso.bg_scene_create(None, None) == -1
    assert libso.bg_intersect_closest(None, None, None, 0, None) == -1


def test_allocation_cap_bookkeeping_without_device():
    """bg_alloc_limit / bg_alloc_stats_get are plain host bookkeeping."""
    from banshee_b200 import capi
    capi.alloc_limit(12345)
    try:
        assert capi.alloc_stats()["budget"] == 12345
    finally:
        capi.alloc_limit(None)
    st = capi.alloc_stats()
    assert st["budget"] == -1 and st["calls"] >= 0 and st["refused"] >= 0
