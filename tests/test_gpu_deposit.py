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
