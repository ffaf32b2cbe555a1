"""The C ABI libraries load without a GPU and export every function that
include/*.h declares."""
import ctypes
import os
import re

import pytest

from dtfe_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(dtfe_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_functions():
    names = declared_functions()
    assert "dtfe_gpu_interpolate" in names and "dtfe_vertex_density_noalloc" in names
    assert len(names) >= 13


def test_gpu_library_exports_all(built):
    lib = ctypes.CDLL(build.build_gpu())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_create_without_device_fails_cleanly(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from dtfe_b200 import _native as N
    lib = N.gpu()
    h = ctypes.c_void_p()
    cfg = N.Config(0, 0, 0, 0)
    rc = lib.dtfe_gpu_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == N.ERR_NO_DEVICE
    assert b"device" in lib.dtfe_last_error()
