"""The C-ABI library loads on a CPU-only host and exports every declared entry."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "hirensi_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hrn_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entries():
    syms = declared_symbols()
    assert "hrn_forward" in syms and "hrn_adjoint_gradient" in syms and len(syms) >= 20


def test_library_exports_all_declared_symbols():
    from hirensi_b200 import build, capi
    build.build()
    lib = C.CDLL(capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding describes every declared entry
    assert set(declared_symbols()) == set(capi.SIGNATURES)


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from hirensi_b200 import capi
    L = capi.load()
    h = C.c_void_p()
    rc = L.hrn_create(0, capi.HRN_FP64, C.byref(h))
    assert rc == capi.HRN_ECUDA and not h.value
    assert L.hrn_version() >= 100
