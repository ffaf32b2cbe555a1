"""Averaging method 1 on the GPU (dtfe_gpu_interpolate with
DTFE_METHOD_TETRAHEDRA): Sobol points inside every tetrahedron gathered per
cell in the reference's order and float arithmetic.

Bars: bit-identical to the oracle's float mode (itself bit-identical to the
reference's interpolateGrid_averaged_1, tests/test_reference_live.py and
tests/test_golden.py); against the FP64 oracle within 1e-5 for the
accumulated fields and 5e-5 for divergence, shear and vorticity (differences
of accumulated gradient components, where the reference's float sums over
up to 100 points per tetrahedron lose more digits); within 1e-6 of the
reference's stored outputs (those use the reference's float-summed vertex
densities)."""
import numpy as np
import pytest

import oracle as O
from conftest import golden, golden_plan, rel_err
from dtfe_b200 import _native as N
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu
FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear",
          "velocity_vorticity", "scalar", "scalar_gradient"]


def _plan(n_threads, n_scalars, grid=(17, 15, 19), seed=41):
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=seed)
    rng = np.random.default_rng(seed + 1)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), n_scalars)).astype(np.float32)
    return P.make_plan(pos, w, vel, sc, grid=grid, n_threads=n_threads, average_density_value=float(w.sum()) / 1e6)


@pytest.mark.parametrize("n_threads,n_scalars,nn,fix", [(1, 1, 100, False), (4, 2, 8, False), (3, 1, 27, True)])
def test_method1_vs_oracle(gpu_built, n_threads, n_scalars, nn, fix):
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(n_threads, n_scalars)
    d32, d64, _ = O.vertex_density(plan)
    want = O.method1(plan, d32, d64, FIELDS, n_points=nn, mode=O.MODE_REF, fix=fix)
    w64 = O.method1(plan, d32, d64, FIELDS, n_points=nn, mode=O.MODE_FP64, fix=fix)
    with DeviceDTFE(0, n_scalars) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        got = d.interpolate(FIELDS, method=N.METHOD_TETRAHEDRA, n_samples=nn, fix=fix)
        again = d.interpolate(FIELDS, method=N.METHOD_TETRAHEDRA, n_samples=nn, fix=fix)
    for f in FIELDS:
        g = got[f].reshape(want[f].shape)
        assert np.array_equal(g, want[f].astype(np.float32)), (f, rel_err(g, want[f]))
        bar = 5e-5 if f in ("velocity_divergence", "velocity_shear", "velocity_vorticity") else 1e-5
        assert rel_err(g, w64[f]) <= bar, (f, rel_err(g, w64[f]))
        assert np.array_equal(got[f], again[f]), f     # deterministic


def test_method1_vs_reference_golden(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    g = golden()
    plan = golden_plan(g)
    fields = ["density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"]
    with DeviceDTFE(0, 1) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        out = d.interpolate(fields, method=N.METHOD_TETRAHEDRA, n_samples=100)
    for f in fields:
        assert rel_err(out[f], g[f"ref_method1_100_{f}"].reshape(out[f].shape)) <= 1e-6, f


def test_method1_errors(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(1, 0, grid=(8, 8, 8))
    with DeviceDTFE(0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        with pytest.raises(N.DTFEError):      # not a Monte-Carlo method
            d.interpolate(["velocity_std"], method=N.METHOD_TETRAHEDRA, n_samples=8)
        bad = plan.region_array().copy()
        bad[0, 0] += 1.0
        with pytest.raises(N.DTFEError):      # lower corner must be the sub-box's lo
            d.set_regions(bad)
        G = int(np.prod(plan.grid))
        import torch
        dens = torch.empty(G, device="cuda")
        with pytest.raises(N.DTFEError, match="not capturable"):
            d.graph_build(plan.rho_bar, ["density"], {"density": dens}, method=N.METHOD_TETRAHEDRA, n_samples=8)
