"""Fields at user sampling points on the GPU (dtfe_gpu_interpolate_points),
bit-identical to the oracle's float mode (itself bit-identical to the
reference's interpolateUserSampling, tests/test_reference_live.py): points
outside the region dropped, outside the hull zeros, on vertices (ties), with
seeds from the grid bins and from the sub-box's first tetrahedron."""
import numpy as np
import pytest

import oracle as O
from dtfe_b200 import _native as N
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu
FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear",
          "velocity_vorticity", "scalar", "scalar_gradient"]


def test_points_vs_oracle(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=51)
    rng = np.random.default_rng(52)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 1)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, sc, grid=(12, 12, 12), n_threads=1, average_density_value=float(w.sum()) / 1e6)
    pts = np.concatenate([rng.uniform(-80, 180, (3000, 3)), rng.uniform(0, 100, (5000, 3))]).astype(np.float32)
    pts[:20] = plan.xyz[:20]
    region = np.array([-70, 170, -60, 160, -70, 150], np.float32)
    d32, d64, _ = O.vertex_density(plan)
    for fix in (False, True):
        want = O.interpolate_points(plan, d32, d64, FIELDS, pts, region, mode=O.MODE_REF, fix=fix)
        with DeviceDTFE(0, 1) as d:
            d.load(plan)
            d.vertex_density(plan.rho_bar)
            for loc in (11, 3, 0):        # fused (seeded), walk (seeded), raster (no seeds)
                d.set_variants(loc, 2)
                d.vertex_density(plan.rho_bar)
                got = d.interpolate_points(FIELDS, pts, region, fix=fix)
                for f in FIELDS:
                    assert got[f].shape[0] == want[f].shape[0]
                    assert np.array_equal(got[f], want[f].astype(np.float32)), (fix, loc, f)
    assert (want["density"] == 0).any() and (want["density"] != 0).any()


def test_points_errors(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    pos, _ = S.zeldovich_lattice(8, 100.0, 0.5, seed=3)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(8, 8, 8), n_threads=2)
    with DeviceDTFE(0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        with pytest.raises(N.DTFEError, match="one sub-box"):
            d.interpolate_points(["density"], np.zeros((4, 3), np.float32), [0, 100, 0, 100, 0, 100])


def test_average_points_vs_oracle(gpu_built):
    """Monte-Carlo volume averages at user points (dtfe_gpu_average_points):
    bit-identical to the oracle's float mode with the same Philox offsets
    (the oracle's estimator matches the reference's statistically,
    tests/test_reference_live.py)."""
    from dtfe_b200.device import DeviceDTFE
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=71)
    rng = np.random.default_rng(72)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 1)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, sc, grid=(12, 12, 12), n_threads=1, average_density_value=float(w.sum()) / 1e6)
    pts = np.concatenate([rng.uniform(-60, 160, (1000, 3)), rng.uniform(0, 100, (2000, 3))]).astype(np.float32)
    delta = rng.uniform(0.5, 12, pts.shape).astype(np.float32)
    region = np.array([-50, 150, -40, 140, -50, 150], np.float32)
    d32, d64, _ = O.vertex_density(plan)
    for nn, seed in ((1, 0), (20, 7)):
        want = O.average_points(plan, d32, d64, FIELDS, pts, delta, region, nn, seed=seed, mode=O.MODE_REF)
        with DeviceDTFE(0, 1) as d:
            d.load(plan)
            for loc in (11, 0):
                d.set_variants(loc, 2)
                d.vertex_density(plan.rho_bar)
                got = d.average_points(FIELDS, pts, delta, region, nn, seed=seed)
                for f in FIELDS:
                    assert got[f].shape[0] == want[f].shape[0]
                    assert np.array_equal(got[f], want[f].astype(np.float32)), (nn, loc, f)
    assert (want["density"] == 0).any() and (want["density"] != 0).any()
