"""The C-ABI library loads and exports every entry point that the headers
under include/ declare (no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

from helpers import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names |= set(re.findall(r"\b(ibg_[a-zA-Z0-9_]+)\s*\(", open(h).read()))
    return sorted(names)


def test_header_and_binding_agree():
    from ibpm_b200._native import SIGNATURES
    assert set(declared_symbols()) == set(SIGNATURES)


def test_library_exports_every_declared_symbol():
    from ibpm_b200 import _native
    L = ctypes.CDLL(_native.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(L, name), name
    _native.lib()  # argtypes bind


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    from ibpm_b200 import _native
    L = _native.lib()
    g = _native.ibg_grid(16, 16, 1, 1.0, -0.5, -0.5)
    xy = (ctypes.c_double * 2)(0.0, 0.0)
    b = _native.ibg_body(1, ctypes.cast(xy, ctypes.POINTER(ctypes.c_double)), 0.0, 0.0, 0)
    p = _native.ibg_params(100.0, 0.01, 2, 1e-7, 100, 1.0, 0.0, 0, -1, 0, 10, 1, 0)
    h = ctypes.c_void_p()
    st = L.ibg_create(ctypes.byref(g), 1, ctypes.byref(b), ctypes.byref(p), None, ctypes.byref(h))
    assert st < 0
    assert L.ibg_last_error(None)
