import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def built():
    from dtfe_b200 import build
    build.build_host()
    build.build_oracle()
    return True


@pytest.fixture(scope="session")
def gpu_built():
    from dtfe_b200 import build
    build.build_host()
    build.build_oracle()
    build.build_gpu()
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def rel_err(a, b):
    """max_i |a_i - b_i| / max(|b_i|, rms(b)) — relative error with the field's
    RMS as the floor of the denominator (components near zero)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    rms = np.sqrt(np.mean(b * b)) if b.size else 1.0
    if rms == 0:
        rms = 1.0
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), rms))) if b.size else 0.0
