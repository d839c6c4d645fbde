"""The CUDA library loads on a machine without a GPU and exports every
symbol that include/fiberlab_gpu.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

from fiberlab_gpu import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "fiberlab_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fl_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_capi.LIB_PATH):
        pytest.fail("the CUDA library is not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(_capi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_capi.EXPORTS) == names


def test_status_strings_and_no_device_behaviour():
    lib = _capi.load()
    assert lib.fl_version().decode().startswith("fiberlab-gpu")
    assert lib.fl_status_string(0) == b"ok"
    assert b"Hermitian" not in lib.fl_status_string(1)
    # without a GPU the context cannot be created: FL_ENODEV, no fallback
    import torch
    if not torch.cuda.is_available():
        h = ctypes.c_void_p()
        assert lib.fl_ctx_create(0, None, ctypes.byref(h)) == 7
