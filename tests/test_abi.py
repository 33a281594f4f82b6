"""The C ABI library loads and exports every symbol include/*.h declares
(CPU; no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in ("dgtd.h", "dgtd_host.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(dgtd_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from rapidfem_b200 import _native
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert len(_declared()) >= 30


def test_version_names_sm100a():
    from rapidfem_b200 import _native
    assert "sm_100a" in _native.version()


def test_no_device_fails_loudly():
    from rapidfem_b200 import _native, gpu
    n = ctypes.c_int(0)
    try:
        import torch
        has = torch.cuda.is_available()
    except Exception:
        has = False
    if has:
        pytest.skip("a CUDA device is present")
    with pytest.raises(_native.NoDeviceError):
        gpu.GpuContext(0)


def test_bad_arguments_return_error_codes():
    from rapidfem_b200 import _native
    lib = ctypes.CDLL(_native.LIB_PATH)  # raw handle: no argtypes, NULLs allowed
    assert lib.dgtd_ctx_create(0, None) == 1
    assert lib.dgtd_op_create(None, None, None) == 1
    assert "null" in _native.last_error()
    assert lib.dgtd_expmv(None, None, ctypes.c_double(0.0), 1, ctypes.c_double(0.0), None, None) == 1
