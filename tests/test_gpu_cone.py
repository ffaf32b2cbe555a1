"""Fields on a redshift-cone grid on the GPU (dtfe_gpu_interpolate_cone),
bit-identical to the oracle's float mode (itself bit-identical to the
reference's interpolateRedshiftCone, tests/test_reference_live.py): shells
leaving the padded hull (zeros), the reference's stuck psi after an outside
sample and its fix, a psi range wrapping through 360 degrees, seeds from the
grid bins and from the sub-box's first tetrahedron."""
import numpy as np
import pytest

import oracle as O
from dtfe_b200 import _native as N
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu
FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear",
          "velocity_vorticity", "scalar", "scalar_gradient"]
CONES = [((1.0, 120.0, 10.0, 170.0, 300.0, 60.0), (50.0, 50.0, 50.0), (9, 7, 45)),
         ((0.5, 60.0, 0.0, 180.0, 0.0, 359.0), (20.0, 70.0, 40.0), (6, 5, 13)),
         ((30.0, 31.0, 90.0, 90.0, 10.0, 10.0), (50.0, 50.0, 50.0), (1, 1, 1))]


def _plan(seed):
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=seed)
    rng = np.random.default_rng(seed + 1)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 1)).astype(np.float32)
    return P.make_plan(pos, w, vel, sc, grid=(12, 12, 12), n_threads=1, average_density_value=float(w.sum()) / 1e6)


def test_cone_vs_oracle(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(53)
    d32, d64, _ = O.vertex_density(plan)
    with DeviceDTFE(0, 1) as d:
        d.load(plan)
        for cone, origin, dims in CONES:
            for fix, fix_outside in ((False, False), (True, False), (False, True)):
                want = O.interpolate_cone(plan, d32, d64, FIELDS, cone, origin, dims, mode=O.MODE_REF, fix=fix,
                                          fix_outside=fix_outside)
                for loc in (11, 3, 0):        # fused (seeded), walk (seeded), raster (no seeds)
                    d.set_variants(loc, 2)
                    d.vertex_density(plan.rho_bar)
                    got = d.interpolate_cone(FIELDS, cone, origin, dims, fix=fix, fix_outside=fix_outside)
                    for f in FIELDS:
                        assert got[f].shape[0] == int(np.prod(dims))
                        assert np.array_equal(got[f], want[f].astype(np.float32)), (cone, fix, fix_outside, loc, f)
    # the first cone leaves the hull and its stuck psi zeroes inside samples
    cone, origin, dims = CONES[0]
    a = O.interpolate_cone(plan, d32, d64, ["density"], cone, origin, dims, mode=O.MODE_REF)["density"]
    b = O.interpolate_cone(plan, d32, d64, ["density"], cone, origin, dims, mode=O.MODE_REF,
                           fix_outside=True)["density"]
    assert (a == 0).any() and (a != 0).any() and ((a == 0) & (b != 0)).any()


def test_cone_device_outputs(gpu_built):
    """dtfe_gpu_interpolate_cone_dev writes the same rows into device
    buffers as the host-buffer call."""
    import torch
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(57)
    cone, origin, dims = CONES[0]
    n = int(np.prod(dims))
    with DeviceDTFE(0, 1) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        want = d.interpolate_cone(FIELDS, cone, origin, dims)
        outs = {f: torch.full((n, N.field_components(N.FIELD_SLOTS[f], 1)), float("nan"), device="cuda")
                for f in FIELDS}
        d.interpolate_cone_dev(FIELDS, cone, origin, dims, outs)
        d.synchronize()
        for f in FIELDS:
            assert np.array_equal(outs[f].cpu().numpy().reshape(want[f].shape), want[f]), f


def test_cone_errors(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(55)
    with DeviceDTFE(0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        with pytest.raises(N.DTFEError, match="theta"):
            d.interpolate_cone(["density"], (1, 10, -5, 90, 0, 90), (50, 50, 50), (2, 2, 2))
        with pytest.raises(N.DTFEError, match="360"):
            d.interpolate_cone(["density"], (1, 10, 0, 90, 0, 360), (50, 50, 50), (2, 2, 2))
        with pytest.raises(N.DTFEError, match="bins"):
            d.interpolate_cone(["density"], (1, 10, 0, 90, 0, 90), (50, 50, 50), (2, 0, 2))
    pos, _ = S.zeldovich_lattice(8, 100.0, 0.5, seed=3)
    split = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(8, 8, 8), n_threads=2)
    with DeviceDTFE(0) as d:
        d.load(split)
        d.vertex_density(split.rho_bar)
        with pytest.raises(N.DTFEError, match="one sub-box"):
            d.interpolate_cone(["density"], (1, 10, 0, 90, 0, 90), (50, 50, 50), (2, 2, 2))


def test_cone_average_vs_oracle(gpu_built):
    """Monte-Carlo bin averages on a redshift cone (dtfe_gpu_interpolate_cone
    with DTFE_METHOD_MONTE_CARLO): bit-identical to the oracle's float mode
    with the same Philox offsets."""
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(59)
    d32, d64, _ = O.vertex_density(plan)
    with DeviceDTFE(0, 1) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        for cone, origin, dims in CONES[:2]:
            for nn, seed in ((1, 0), (12, 5)):
                want = O.average_cone(plan, d32, d64, FIELDS, cone, origin, dims, nn, seed=seed, mode=O.MODE_REF)
                got = d.interpolate_cone(FIELDS, cone, origin, dims, n_samples=nn, seed=seed)
                for f in FIELDS:
                    assert np.array_equal(got[f], want[f].astype(np.float32)), (cone, nn, f)
