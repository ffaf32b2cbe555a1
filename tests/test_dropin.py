"""The DTFE() drop-in's option checks, which run before any GPU work (CPU)."""
import numpy as np
import pytest

import dropin as D

pytestmark = pytest.mark.skipif(not D.available(), reason="drop-in driver not built (needs the reference headers)")


def _particles():
    rng = np.random.default_rng(0)
    return rng.uniform(0, 100, (500, 3)).astype(np.float32), np.ones(500, np.float32)


def test_unsupported_options_throw(built):
    pos, w = _particles()
    with pytest.raises(RuntimeError, match="averaging methods other than 1, 2, 3"):
        D.run("DTFE", pos, w, None, None, (8, 8, 8), a_fields=("density",), method=4)
    with pytest.raises(RuntimeError, match="scalar fields with NGP/CIC/TSC"):
        D.run("CIC", pos, w, None, None, (8, 8, 8), a_fields=("density", "scalar"))
