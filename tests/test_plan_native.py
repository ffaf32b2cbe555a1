"""The C++ planner (dtfe_plan_build, used by the DTFE() drop-in) against
the Python planner: identical plans, array for array."""
import ctypes as C

import numpy as np
import pytest

from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S


def _inputs(n=14, seed=3):
    pos, psi = S.zeldovich_lattice(n, 100.0, 0.9, seed=seed)
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (20 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 2)).astype(np.float32)
    return pos, w, vel, sc


def _boxes_equal(a, b, typ):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert bytes(x) == bytes(y)


@pytest.mark.parametrize("threads,periodic,avg", [(1, True, None), (4, True, 1e-3), (6, False, None)])
def test_dtfe_plan_identical(built, threads, periodic, avg):
    pos, w, vel, sc = _inputs()
    kw = dict(grid=(12, 10, 14), n_threads=threads, periodic=periodic, average_density_value=avg)
    a = P.make_plan(pos, w, vel, sc, **kw)
    b = P.native_plan("DTFE", pos, w, vel, sc, **kw)
    for f in ("tet_v", "tet_n", "xyz", "src", "weight", "velocity", "scalar", "xs", "ys", "zs", "padding"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert a.grid == b.grid and a.rho_bar == b.rho_bar
    _boxes_equal(a.boxes, b.boxes, "subbox")


@pytest.mark.parametrize("kind", ["NGP", "CIC", "TSC"])
def test_deposit_plan_identical(built, kind):
    pos, w, vel, _ = _inputs(seed=5)
    kw = dict(grid=(9, 12, 10), n_threads=4, kind=kind)
    a = P.make_deposit_plan(pos, w, vel, **kw)
    b = P.native_plan(kind, pos, w, vel, grid=(9, 12, 10), n_threads=4)
    for f in ("pos", "weight", "velocity", "src"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert a.rho_bar == b.rho_bar and a.kind == b.kind
    _boxes_equal(a.boxes, b.boxes, "deposit")
