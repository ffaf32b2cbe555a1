"""GPU parity on the 64^3 -> 128^3 density workload, not only on toy sizes.

Workload: 64^3 particles on a cell-centred lattice in a periodic 100 Mpc/h
box, displaced by Zel'dovich displacements (P(k) ~ k^-2, Gaussian smoothing
at 2 lattice spacings, rms 0.5 spacing, seed 0), unit weights, the default
padding of 5 particles, average density sum(w)/L^3, cell centres of a 128^3
grid, split into the reference's sub-boxes for 8 host threads
(parallelGrid / optimalPartitionSplit, src/subpartition.h:163-555).

Checked through the C ABI against the CPU oracle on every cell:
  * the tetrahedron each centre is located in equals the oracle's walk
    (canonical tie rule) — interpolateGrid's dt.locate,
    unaveraged_interpolation.cc:289;
  * vertex densities and the density field are bit-identical to the oracle
    in the reference's arithmetic (unaveraged_interpolation.cc:209-369);
  * density within 1e-5 of the FP64 oracle, both as the relative error with
    the field's RMS as the floor of the denominator and as the plain
    relative error (density is positive everywhere).
The same tessellation with velocities (100 km/s per unit displacement plus
N(0, 50 km/s)) then checks all 22 floats per cell (density, velocity, its
gradient, divergence, shear, vorticity): bit-identical to the oracle in the
reference's arithmetic, and within 1e-5 of the FP64 oracle except the shear.
The reference evaluates the gradient in float (unaveraged_interpolation.cc:
94-104), and its rounding, relative to a cell's largest gradient component,
reaches 1.28e-5 (RMS floor) on one shear component of this grid: the FP64
formulas applied to the same float gradient give the same 1.27e-5, so the
shear's bar in this arithmetic is 2e-5.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import rel_err, rel_err_plain
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu

FULL = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear",
        "velocity_vorticity"]
# FP64 bars of the reference's float arithmetic (see the module docstring)
FP64_BAR = {f: 1e-5 for f in FULL}
FP64_BAR["velocity_shear"] = 2e-5
NCPU = os.cpu_count() or 1


@pytest.fixture(scope="module")
def plan0(gpu_built):
    pos, psi = S.zeldovich_lattice(64, S.BOX, 0.5, seed=0)
    vel = (100.0 * psi / (S.BOX / 64) + np.random.default_rng(2).normal(0.0, 50.0, psi.shape)).astype(np.float32)
    w = np.ones(len(pos), np.float32)
    return P.make_plan(pos, w, vel, None, grid=(128, 128, 128), n_threads=8,
                       average_density_value=float(len(pos)) / S.BOX ** 3)


@pytest.fixture(scope="module")
def densities(plan0):
    return O.vertex_density(plan0)


def _run(plan, fields):
    from dtfe_b200.device import DeviceDTFE
    with DeviceDTFE(0, 0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        dens = d.download_vertex_density(plan.n_verts)
        out = d.interpolate(fields, method=0)
        st = d.last_status
        loc = d.download_located()
    return dens, out, loc, st


def test_config0_density(plan0, densities):
    d32, d64, _ = densities
    assert plan0.n_boxes == 8
    dens, out, loc, st = _run(plan0, ["density"])
    G = 128 ** 3
    assert st["n_samples_located"] == G and st["n_walk_failures"] == 0 and st["n_outside"] == 0
    assert np.array_equal(dens.view(np.int32), d32.view(np.int32))
    ref, oloc = O.interpolate(plan0, d32, d64, ["density"], mode=O.MODE_REF, want_loc=True, nthreads=NCPU)
    assert (oloc >= 0).all()
    bad = np.flatnonzero(loc != oloc)
    assert bad.size == 0, (bad.size, bad[:10])
    assert np.array_equal(out["density"], ref["density"].astype(np.float32))
    f64, _ = O.interpolate(plan0, d32, d64, ["density"], mode=O.MODE_FP64, nthreads=NCPU)
    assert rel_err(out["density"], f64["density"]) <= 1e-5
    assert (f64["density"] > 0).all()
    assert rel_err_plain(out["density"], f64["density"], floor_frac=0.0) <= 1e-5


def test_config0_all_fields(plan0, densities):
    d32, d64, _ = densities
    _, out, loc, st = _run(plan0, FULL)
    assert st["n_walk_failures"] == 0
    ref, oloc = O.interpolate(plan0, d32, d64, FULL, mode=O.MODE_REF, want_loc=True, nthreads=NCPU)
    assert np.array_equal(loc, oloc)
    f64, _ = O.interpolate(plan0, d32, d64, FULL, mode=O.MODE_FP64, nthreads=NCPU)
    for f in FULL:
        assert np.array_equal(out[f].reshape(ref[f].shape), ref[f].astype(np.float32)), f
        assert rel_err(out[f], f64[f]) <= FP64_BAR[f], (f, rel_err(out[f], f64[f]))
    assert rel_err_plain(out["density"], f64["density"], floor_frac=0.0) <= 1e-5
