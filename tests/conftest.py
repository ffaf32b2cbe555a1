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


def rel_err_plain(a, b, floor_frac=0.01):
    """max_i |a_i - b_i| / |b_i| over the entries with |b_i| above floor_frac
    times the field's RMS (the plain relative error; entries nearer zero are
    cancellation residues whose relative error says nothing)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    if not b.size:
        return 0.0
    rms = np.sqrt(np.mean(b * b))
    keep = np.abs(b) > floor_frac * rms
    if not keep.any():
        return 0.0
    return float(np.max(np.abs(a[keep] - b[keep]) / np.abs(b[keep])))


GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_zeldovich10.npz")


def golden():
    return dict(np.load(GOLDEN))


def golden_plan(g):
    """A single-box Plan rebuilt from the fixture's stored tessellation."""
    import ctypes as C
    from dtfe_b200 import _native as N
    from dtfe_b200.plan import Plan
    boxes = (N.Subbox * 1)()
    b = boxes[0]
    b.vert_offset, b.n_verts, b.tet_offset, b.n_tets = 0, len(g["xyz"]), 0, len(g["tet_v"])
    for a in range(3):
        b.tile_origin[a] = 0
        b.tile_dims[a] = int(g["grid"][a])
        b.dx[a] = float(g["box_dx"][a])
        b.lo[a] = float(g["box_lo"][a])
    b.coord_offset[0] = b.coord_offset[1] = b.coord_offset[2] = 0
    b.part_no = -1
    return Plan(tet_v=g["tet_v"], tet_n=g["tet_n"], xyz=g["xyz"], src=np.arange(len(g["xyz"]), dtype=np.int32),
                weight=g["weight"], velocity=g["velocity"], scalar=g["scalar"], boxes=boxes, xs=g["xs"],
                ys=g["ys"], zs=g["zs"], grid=tuple(int(x) for x in g["grid"]), rho_bar=float(g["rho_bar"]),
                padding=g["padding"], regions=g["region"].reshape(1, 6) if "region" in g else None)
