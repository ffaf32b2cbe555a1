"""The C ABI libraries load without a GPU and export every function that
include/*.h declares."""
import ctypes
import os
import re

import pytest

from dtfe_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header=None):
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h") or (header and f != header):
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
    missing = [n for n in declared_functions("dtfe_gpu.h") if not hasattr(lib, n)]
    assert not missing, missing


def test_host_library_exports_all(built):
    lib = ctypes.CDLL(build.build_host())
    names = declared_functions("dtfe_host.h")
    assert "dtfe_plan_build" in names and "dtfe_tessellate_batch" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_dropin_exports_reference_entry_point(built):
    """libdtfe_dropin.so defines the reference's C++ entry point
    DTFE(std::vector<Particle_data>*, std::vector<Sample_point>&,
    User_options&, Quantities*, Quantities*) (src/DTFE.h:36-40)."""
    import subprocess
    path = os.path.join(build.BUILD, "libdtfe_dropin.so")
    if not os.path.exists(path):
        pytest.skip("drop-in not built (needs the reference headers)")
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    assert "_Z4DTFEPSt6vectorI13Particle_dataSaIS0_EERS_I12Sample_pointSaIS4_EER12User_optionsP10QuantitiesSB_" in out


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


def test_tessellate_argument_errors_without_device(built):
    """dtfe_gpu_tessellate checks its arguments before any device call:
    no sets, a decreasing or non-zero-based vertex prefix and missing
    positions give DTFE_ERR_ARG and no handle."""
    assert "dtfe_gpu_tessellate" in declared_functions("dtfe_gpu.h")
    lib = ctypes.CDLL(build.build_gpu())
    lib.dtfe_gpu_tessellate.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_void_p)]
    out = ctypes.c_void_p(1)
    assert lib.dtfe_gpu_tessellate(None, 0, None, None, ctypes.byref(out)) == 1
    assert not out.value
    for pre in ((0, 5, 3), (1, 5), (0, 5)):
        arr = (ctypes.c_int64 * len(pre))(*pre)
        out = ctypes.c_void_p(1)
        assert lib.dtfe_gpu_tessellate(None, len(pre) - 1, arr, None, ctypes.byref(out)) == 1
        assert not out.value
