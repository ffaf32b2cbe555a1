"""GPU SPH estimator (dtfe_gpu_sph) against the oracle and the reference.

The oracle's FP64 mode sums the same float terms in double, as the GPU does:
1e-6 relative (RMS floor) between the two.  Against the reference's float
accumulation (the golden fixture, made by the reference's own
SPH_interpolation): 1e-5.
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden, golden_plan, rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from dtfe_b200 import _native as N  # noqa: E402
from dtfe_b200 import plan as P  # noqa: E402
from dtfe_b200 import synthetic as S  # noqa: E402


def _plan(n, grid, threads, seed, disp=0.8, scalars=1):
    pos, psi = S.zeldovich_lattice(n, 100.0, disp, seed=seed)
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (40 * psi + rng.normal(0, 5, psi.shape)).astype(np.float32)
    sc = rng.standard_normal((len(pos), scalars)).astype(np.float32) if scalars else None
    return P.make_plan(pos, w, vel, sc, grid=grid, n_threads=threads, average_density_value=float(w.sum()) / 1e6)


@pytest.mark.parametrize("n,grid,threads,k,extensive", [(16, (16, 16, 16), 1, 32, False),
                                                        (20, (24, 20, 18), 8, 32, True),
                                                        (18, (12, 12, 12), 4, 16, False),
                                                        (18, (12, 14, 10), 2, 64, False),
                                                        (16, (10, 10, 10), 1, 100, True)])
def test_sph_matches_oracle(gpu_built, n, grid, threads, k, extensive):
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(n, grid, threads, seed=n + k)
    with DeviceDTFE(0, plan.n_scalars) as dev:
        dev.load(plan)
        out = dev.sph(plan.rho_bar, n_neighbors=k, velocity=True, scalars=True, extensive=extensive)
    d64, v64, s64 = O.sph(plan, k=k, velocity=True, scalars=True, extensive=extensive, mode=O.MODE_FP64)
    assert rel_err(out["density"], d64) < 1e-6
    assert rel_err(out["velocity"], v64) < 1e-6
    assert rel_err(out["scalar"], s64) < 1e-5
    dref, vref, _ = O.sph(plan, k=k, velocity=True, mode=O.MODE_REF)
    assert rel_err(out["density"], dref) < 1e-5
    assert rel_err(out["velocity"], vref) < 1e-5


def test_sph_vs_reference_fixture(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    g = golden()
    plan = golden_plan(g)
    plan.scalar = g["scalar"]
    with DeviceDTFE(0, 1) as dev:
        dev.load(plan)
        out = dev.sph(plan.rho_bar, n_neighbors=32, velocity=True, scalars=True)
    assert rel_err(out["density"], g["ref_sph32_density"]) < 1e-5
    assert rel_err(out["velocity"], g["ref_sph32_velocity"]) < 1e-5
    assert rel_err(out["scalar"][:, 0], g["ref_sph32_scalar"]) < 1e-5


def test_sph_device_outputs_and_errors(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    plan = _plan(12, (10, 10, 10), 2, seed=3, scalars=0)
    G = int(np.prod(plan.grid))
    cuda = torch.device("cuda", 0)
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        host = dev.sph(plan.rho_bar, velocity=True)
        d = torch.empty(G, device=cuda)
        v = torch.empty((G, 3), device=cuda)
        dev.sph_dev(plan.rho_bar, d, v)
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy(), host["density"])
        assert np.array_equal(v.cpu().numpy(), host["velocity"])
        # repeatable: FP64 sums rounded once
        again = dev.sph(plan.rho_bar, velocity=True)
        assert np.array_equal(again["density"], host["density"])
        with pytest.raises(N.DTFEError):
            dev.sph(plan.rho_bar, n_neighbors=0)
        with pytest.raises(N.DTFEError):
            dev.sph(plan.rho_bar, n_neighbors=129)
        with pytest.raises(N.DTFEError):
            dev.sph(plan.rho_bar, scalars=True)  # no scalars uploaded
