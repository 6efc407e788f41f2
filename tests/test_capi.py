"""C-ABI library checks that need no GPU: the in-tree library loads and
exports every entry point include/mkfit_b200.h declares, and calls fail
cleanly (status code, message) instead of aborting."""
import ctypes

import pytest

from mkfit_b200 import capi


def test_library_exports_all_header_symbols():
    lib = capi.load()
    syms = capi.header_symbols()
    assert len(syms) >= 8
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in capi.load().mkfg_version()


def test_context_create_without_device_reports_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    lib = capi.load()
    h = ctypes.c_void_p()
    rc = lib.mkfg_context_create(0, ctypes.byref(h))
    assert rc == 5  # MKFG_ERR_NO_DEVICE
    assert "device" in capi.last_error().lower()


def test_null_context_is_bad_input():
    lib = capi.load()
    a = capi.MkfgFitArgs()
    assert lib.mkfg_fit(None, ctypes.byref(a)) == 1
    assert "context" in capi.last_error()
