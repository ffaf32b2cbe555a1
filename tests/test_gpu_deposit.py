"""GPU NGP / CIC / TSC deposition against the oracle (through the C ABI).

Bars: relative error <= 1e-6 (denominator floored at the field RMS) against
both the oracle in the reference's float arithmetic and in FP64 — the GPU
sums the reference's float contributions exactly (64-bit fixed point), so it
is at least as close to FP64 as the reference's own float accumulation; and
two runs are bit-identical (order-independent sums).
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["NGP", "CIC", "TSC"])
@pytest.mark.parametrize("n_threads", [1, 8])
def test_deposit_matches_oracle(gpu_built, kind, n_threads):
    from dtfe_b200.device import DeviceDTFE
    pos, psi = S.zeldovich_lattice(24, 100.0, 0.8, 2)
    w = np.random.default_rng(3).uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (80 * psi).astype(np.float32)
    dp = P.make_deposit_plan(pos, w, vel, grid=(20, 24, 18), n_threads=n_threads, kind=kind,
                             average_density_value=float(w.sum()) / 1e6)
    with DeviceDTFE(0, 0) as d:
        g1 = d.deposit(dp)
        g2 = d.deposit(dp)
    assert np.array_equal(g1["density"], g2["density"]) and np.array_equal(g1["velocity"], g2["velocity"])
    rd, rv = O.deposit(dp, O.MODE_REF)
    fd, fv = O.deposit(dp, O.MODE_FP64)
    assert rel_err(g1["density"], rd) <= 1e-6
    assert rel_err(g1["density"], fd) <= 1e-6
    mask = fd != 0
    assert rel_err(g1["velocity"][mask], fv[mask]) <= (1e-4 if kind == "CIC" else 1e-6)


@pytest.mark.parametrize("kind", ["NGP", "CIC", "TSC"])
def test_deposit_resident_paths(gpu_built, kind):
    """Uniform random particles on a fine grid: a block's 512 particles span
    more cells than its shared tile holds, so they add to global memory
    directly.  Device-resident particles (dtfe_gpu_deposit_resident) give the
    same bits as host ones, and a density-only deposit the same densities as
    one with velocities; all agree with the oracle.  At 0.5 particles per
    cell the clipped, partly negative edge weights leave some cells with a
    mass near 0, where velocity = momentum / mass amplifies the float
    rounding of the reference's contributions; velocities are compared where
    the FP64 density exceeds 10% of its RMS."""
    import torch
    from dtfe_b200.device import DeviceDTFE
    rng = np.random.default_rng(11)
    n = 40000
    pos = rng.uniform(0.0, 100.0, (n, 3)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, n).astype(np.float32)
    vel = rng.normal(0.0, 100.0, (n, 3)).astype(np.float32)
    dp = P.make_deposit_plan(pos, w, vel, grid=(48, 40, 44), n_threads=2, kind=kind,
                             average_density_value=float(w.sum()) / 1e6)
    G = int(np.prod(dp.grid))
    cuda = torch.device("cuda:0")
    with DeviceDTFE(0, 0) as d:
        host = d.deposit(dp)
        dens_only = d.deposit(dp, velocity=False)
        pd, wd, vd = (torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in (dp.pos, dp.weight, dp.velocity))
        dd = torch.full((G,), -1.0, device=cuda)
        dv = torch.full((G, 3), -1.0, device=cuda)
        torch.cuda.synchronize()
        d.deposit_resident(dp, pd, wd, vd, dd, dv)
        res_d, res_v = dd.cpu().numpy(), dv.cpu().numpy()
    assert np.array_equal(res_d.view(np.int32), host["density"].view(np.int32))
    assert np.array_equal(res_v.view(np.int32), host["velocity"].view(np.int32))
    assert np.array_equal(dens_only["density"].view(np.int32), host["density"].view(np.int32))
    fd, fv = O.deposit(dp, O.MODE_FP64)
    assert rel_err(host["density"], fd) <= 1e-6
    mask = np.abs(fd) > 0.1 * np.sqrt(np.mean(fd.astype(np.float64) ** 2))
    assert mask.sum() > G // 4
    assert rel_err(host["velocity"][mask], fv[mask]) <= (1e-4 if kind == "CIC" else 1e-6)
