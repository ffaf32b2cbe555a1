"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Bars:
  * point location: bit-exact tetrahedron ids (canonical tie rule);
  * vertex densities: bit-identical to the oracle's mode-"ref" values (both
    add a vertex's FP64 volumes as exact integers in units of its sub-box,
    fixed_volume.cuh);
  * interpolated fields vs the oracle in the reference's arithmetic (mode ref):
    relative error <= 1e-6;
  * interpolated fields vs the FP64 oracle: relative error <= 1e-5 (the
    north-star tolerance), denominators floored at the field's RMS.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu

FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear",
          "velocity_vorticity", "scalar", "scalar_gradient"]


def _plan(n=24, grid=(24, 24, 24), n_threads=1, rms=0.5, seed=0, n_scalars=1):
    pos, psi = S.zeldovich_lattice(n, 100.0, rms, seed)
    w = np.random.default_rng(seed + 10).uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (100 * psi / (100.0 / n)).astype(np.float32)
    sc = np.random.default_rng(seed + 20).standard_normal((len(pos), n_scalars)).astype(np.float32) \
        if n_scalars else None
    return P.make_plan(pos, w, vel, sc, grid=grid, n_threads=n_threads,
                       average_density_value=float(w.sum()) / 1e6)


@pytest.fixture(scope="module")
def plan1(gpu_built):
    return _plan()


@pytest.fixture(scope="module")
def plan8(gpu_built):
    return _plan(n=20, grid=(20, 20, 20), n_threads=8, n_scalars=2)


def _device(plan):
    from dtfe_b200.device import DeviceDTFE
    d = DeviceDTFE(0, plan.n_scalars)
    d.load(plan)
    d.vertex_density(plan.rho_bar)
    return d


def test_vertex_density(plan1):
    d = _device(plan1)
    g = d.download_vertex_density(plan1.n_verts)
    d32, d64, _ = O.vertex_density(plan1)
    assert np.array_equal(g.view(np.int32), d32.view(np.int32))
    assert rel_err(g, d64) < 1e-6
    d.close()


def test_locate_bit_exact(plan1):
    d = _device(plan1)
    rng = np.random.default_rng(3)
    pts = rng.random((20000, 3)) * 100.0
    # include exact vertex positions and face/edge midpoints (ties)
    tv = plan1.tet_v[:500]
    X = plan1.xyz.astype(np.float64)
    pts = np.concatenate([pts, X[tv[:, 0]], 0.5 * (X[tv[:, 0]] + X[tv[:, 1]]),
                          (X[tv[:, 0]] + X[tv[:, 1]] + X[tv[:, 2]]) / 3.0])
    g = d.locate_points(pts, start=0)
    o = O.locate(plan1, pts)
    assert (g == o).all(), np.flatnonzero(g != o)[:10]
    d.close()


@pytest.mark.parametrize("fix", [False, True])
def test_centre_fields(plan1, fix):
    d = _device(plan1)
    g = d.interpolate(FIELDS, method=0, fix=fix)
    assert d.last_status["n_walk_failures"] == 0
    d32, d64, _ = O.vertex_density(plan1)
    ref, _ = O.interpolate(plan1, d32, d64, FIELDS, mode=O.MODE_REF, fix=fix)
    f64, _ = O.interpolate(plan1, d32, d64, FIELDS, mode=O.MODE_FP64, fix=fix)
    for f in FIELDS:
        assert rel_err(g[f], ref[f]) <= 1e-6, f
        assert rel_err(g[f], f64[f]) <= 1e-5, f
    d.close()


@pytest.mark.parametrize("method,nn", [(2, 8), (3, 8)])
def test_averaged_fields(plan1, method, nn):
    d = _device(plan1)
    fields = FIELDS + (["velocity_std"] if method == 2 else [])
    g = d.interpolate(fields, method=method, n_samples=nn, seed=3)
    d32, d64, _ = O.vertex_density(plan1)
    ref, _ = O.interpolate(plan1, d32, d64, fields, method=method, n_samples=nn, seed=3, mode=O.MODE_REF)
    f64, _ = O.interpolate(plan1, d32, d64, fields, method=method, n_samples=nn, seed=3, mode=O.MODE_FP64)
    for f in fields:
        assert rel_err(g[f], ref[f]) <= 1e-6, f
        assert rel_err(g[f], f64[f]) <= 1e-5, f
    d.close()


def test_subboxes(plan8):
    d = _device(plan8)
    fields = FIELDS
    g = d.interpolate(fields, method=0)
    d32, d64, _ = O.vertex_density(plan8)
    ref, loc = O.interpolate(plan8, d32, d64, fields, mode=O.MODE_REF, want_loc=True)
    assert (loc >= 0).all()
    for f in fields:
        assert rel_err(g[f], ref[f]) <= 1e-6, f
    d.close()


def test_launch_variants_identical(plan8):
    """Every autotuner variant (register budget, cells per thread seeded from
    the previous hit) produces bit-identical fields."""
    d = _device(plan8)
    chosen = d.autotune(FIELDS)
    n_loc, n_ev = d.variant_counts()
    assert n_loc >= 6 and n_ev >= 3
    assert 0 <= chosen[0] < n_loc and 0 <= chosen[1] < n_ev
    d.set_variants(0, 0)
    base = d.interpolate(FIELDS, method=0)
    st0 = d.last_status
    for loc in range(n_loc):
        for ev in range(n_ev):
            d.set_variants(loc, ev)
            g = d.interpolate(FIELDS, method=0)
            for f in FIELDS:
                assert np.array_equal(g[f], base[f]), (loc, ev, f)
            assert d.last_status["n_samples_located"] == st0["n_samples_located"]
            assert d.last_status["n_outside"] == st0["n_outside"]
    d.close()


def test_centre_ties_lattice(gpu_built):
    """Particles exactly on every second sample coordinate: every cell centre
    is a vertex, an edge midpoint, a face centre or a cube centre of the
    lattice, so most centres lie on shared faces, edges or vertices.  The
    raster variants (lowest id among the tetrahedra whose closure holds the
    centre) and the walk variants (walk, then the tie rule) must both give
    the oracle's canonical tetrahedra: fields equal to the oracle's."""
    from dtfe_b200.device import DeviceDTFE
    g = (24, 24, 24)
    rng = np.random.default_rng(1)
    probe = P.make_plan(rng.random((100, 3)).astype(np.float32) * 100, np.ones(100, np.float32), None, None,
                        grid=g, n_threads=1, average_density_value=1e-3)
    X, Y, Z = np.meshgrid(probe.xs[::2], probe.ys[::2], probe.zs[::2], indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.float32)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, None, grid=g, n_threads=1, average_density_value=float(w.sum()) / 1e6)
    assert np.array_equal(plan.xs, probe.xs)
    fields = ["density", "velocity", "velocity_gradient"]
    d32, d64, _ = O.vertex_density(plan)
    ref, _ = O.interpolate(plan, d32, d64, fields, mode=O.MODE_REF)
    with DeviceDTFE(0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        n_loc, _ = d.variant_counts()
        outs = []
        for loc in (0, 1, 2, n_loc - 6):     # the three raster budgets and the first walk variant
            d.set_variants(loc, 0)
            outs.append(d.interpolate(fields, method=0))
            assert d.last_status["n_outside"] == 0
            assert d.last_status["n_samples_located"] == int(np.prod(g))
        assert d.last_status["n_ties"] > 0
    for got in outs:
        for f in fields:
            assert np.array_equal(got[f], outs[0][f]), f
            assert rel_err(got[f], ref[f]) <= 1e-6, f


def test_sparse_subboxes(gpu_built):
    """Sub-boxes without tetrahedra, one-tetrahedron sub-boxes and cell centres
    outside the hulls (the reference's stale raster after an outside sample,
    and DTFE_FLAG_FIX_OUTSIDE_RASTER): every locate variant, methods 0, 3, 1,
    bit-identical to the oracle's float mode (itself pinned to the reference
    in tests/test_reference_live.py)."""
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    rng = np.random.default_rng(1)
    pos = (rng.random((40, 3)) * 100).astype(np.float32)
    vel = rng.standard_normal((40, 3)).astype(np.float32)
    plan = P.make_plan(pos, rng.uniform(0.5, 1.5, 40).astype(np.float32), vel, None, grid=(16, 16, 16),
                       n_threads=16, periodic=False, padding=np.ones(6, np.float32), average_density_value=1e-3)
    fields = ["density", "velocity", "velocity_gradient", "velocity_divergence"]
    d32, d64, _ = O.vertex_density(plan)
    with DeviceDTFE(0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        n_loc, _ = d.variant_counts()
        for fix_outside in (False, True):
            want, _ = O.interpolate(plan, d32, d64, fields, method=0, mode=O.MODE_REF, fix_outside=fix_outside)
            for loc in range(n_loc):
                d.set_variants(loc, 0)
                got = d.interpolate(fields, method=0, fix_outside=fix_outside)
                for f in fields:
                    assert np.array_equal(got[f].reshape(want[f].shape), want[f].astype(np.float32)), \
                        (fix_outside, loc, f)
        want, _ = O.interpolate(plan, d32, d64, fields, method=3, n_samples=8, mode=O.MODE_REF)
        got = d.interpolate(fields, method=3, n_samples=8)
        for f in fields:
            assert rel_err(got[f].reshape(want[f].shape), want[f]) <= 1e-6, f
        want = O.method1(plan, d32, d64, fields, n_points=100, mode=O.MODE_REF)
        got = d.interpolate(fields, method=N.METHOD_TETRAHEDRA, n_samples=100)
        for f in fields:
            assert np.array_equal(got[f].reshape(want[f].shape), want[f].astype(np.float32)), f
