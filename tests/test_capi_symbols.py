"""The C ABI library loads without a GPU and exports every declared symbol."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fhb200.h")


def declared_symbols() -> set[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(fhb_[a-z0-9_]+)\s*\(", text))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for required in ("fhb_context_create", "fhb_forward_ntt", "fhb_inverse_ntt", "fhb_ckks_keyswitch_core",
                     "fhb_ckks_moddown", "fhb_ckks_relinearize", "fhb_ckks_rotate"):
        assert required in syms


def test_library_exports_every_declared_symbol():
    from fhelium_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("libfhb200.so not built")
    lib = _native.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(_native.SIGNATURES) == declared_symbols()
    assert lib.fhb_version() >= 1


def test_invalid_arguments_are_rejected_without_gpu():
    from fhelium_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        pytest.skip("libfhb200.so not built")
    lib = _native.load()
    # NULL context is rejected before any CUDA call
    rc = lib.fhb_forward_ntt(None, None, None, 1, 1, 0, 0, None)
    assert rc < 0
    assert "context" in _native.last_error()
    out = ctypes.c_void_p()
    bad = (ctypes.c_uint64 * 2)(12, 13)  # not NTT primes
    rc = lib.fhb_context_create(64, 12, bad, 1, 1, 0, ctypes.byref(out))
    assert rc < 0 and "NTT prime" in _native.last_error()
    rc = lib.fhb_context_create(64, 9, bad, 1, 1, 0, ctypes.byref(out))
    assert rc < 0 and "log_n" in _native.last_error()
