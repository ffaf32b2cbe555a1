"""The oracle against the reference's own sources, run live through the
reference-code harness (oracle/_ref, built from the reference tree where it
is available; skipped elsewhere), on fresh inputs and on a sub-box split."""
import numpy as np
import pytest

import oracle as O
import refharness as R
from conftest import rel_err
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.skipif(not R.available(), reason="reference harness not built")
FIELDS = ["density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"]


@pytest.mark.parametrize("n_threads", [1, 4])
def test_live_interpolation(built, n_threads):
    pos, psi = S.zeldovich_lattice(14, 100.0, 0.9, seed=21)
    w = np.random.default_rng(22).uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = np.random.default_rng(23).standard_normal((len(pos), 1)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, sc, grid=(12, 14, 16), n_threads=n_threads,
                       average_density_value=float(w.sum()) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    for method, nn in ((0, 1), (3, 8)):
        ora, _ = O.interpolate(plan, d32, d64, FIELDS, method=method, n_samples=nn, mode=O.MODE_REF)
        for k, b in enumerate(plan.box_list()):
            ref = R.run(plan, k, which=method, n_points=nn, dens_override=d32)
            v0 = b.vert_offset
            assert rel_err(ref["vertex_density"], d32[v0:v0 + b.n_verts]) <= 1e-6
            ox, oy, oz = b.tile_origin[0], b.tile_origin[1], b.tile_origin[2]
            dims = (b.tile_dims[0], b.tile_dims[1], b.tile_dims[2])
            for f in FIELDS:
                full = ora[f].reshape(plan.grid + ora[f].shape[1:])
                tile = full[ox:ox + dims[0], oy:oy + dims[1], oz:oz + dims[2]].reshape(ref[f].shape)
                assert np.array_equal(tile.astype(np.float32), ref[f]), (method, k, f)


@pytest.mark.parametrize("k,extensive", [(32, 0), (16, 1), (7, 0)])
def test_live_sph(built, k, extensive):
    """SPH oracle (reference float mode) against the reference's own
    SPH_interpolation and kd-tree on fresh particles in a region."""
    import ctypes as C
    L = R.lib()
    vp = C.c_void_p
    L.ref_sph.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int64, vp, vp, C.c_double, C.c_int, vp, vp, vp]
    n = 18
    pos, psi = S.zeldovich_lattice(n, 100.0, 0.8, seed=30 + k)
    rng = np.random.default_rng(k)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (12 * psi).astype(np.float32)
    sc = rng.standard_normal(len(pos)).astype(np.float32)
    region = np.array([10, 90, 5, 95, 0, 100], np.float32)
    grid = np.array([11, 9, 13], np.int32)
    G = int(np.prod(grid))
    d, v, s = np.zeros(G, np.float32), np.zeros((G, 3), np.float32), np.zeros(G, np.float32)
    avg = float(w.sum()) / 1e6
    assert L.ref_sph(pos.ctypes.data, w.ctypes.data, vel.ctypes.data, sc.ctypes.data, extensive, len(pos),
                     region.ctypes.data, grid.ctypes.data, avg, k, d.ctypes.data, v.ctypes.data, s.ctypes.data) == 0
    tabs = [P.axis_coords(region[2 * a], np.float32((region[2 * a + 1] - region[2 * a]) / np.float32(grid[a])),
                          int(grid[a])) for a in range(3)]
    od, ov, osc = O.sph_region(pos, w, vel, sc[:, None], *tabs, avg, k, extensive=bool(extensive), mode=O.MODE_REF)
    assert np.array_equal(od.astype(np.float32), d)
    assert np.array_equal(ov.astype(np.float32), v)
    assert np.array_equal(osc[:, 0].astype(np.float32), s)


def test_timed_reference_matches_untimed(built):
    """The timed harness entry the CPU baseline uses runs the same reference
    code (same outputs) and reports a positive time per sub-box."""
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.8, seed=3)
    w = np.ones(len(pos), np.float32)
    vel = (20 * psi).astype(np.float32)
    plan = P.make_plan(pos, w, vel, None, grid=(10, 10, 10), n_threads=4, average_density_value=float(len(pos)) / 1e6)
    tmax, per_box = R.time_boxes(plan, 2)
    assert len(per_box) == plan.n_boxes and all(t > 0 for t in per_box)
    assert tmax >= max(per_box) - 1e-12


@pytest.mark.parametrize("n_threads,nn", [(1, 100), (4, 8)])
def test_live_method1(built, n_threads, nn):
    """Averaging method 1 (Sobol points inside every tetrahedron scattered to
    the grid): the reference's own interpolateGrid_averaged_1, run through the
    harness on each sub-box, against the oracle's float mode bit for bit, and
    the oracle's FP64 mode within 1e-5 of it."""
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=41)
    rng = np.random.default_rng(42)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 1)).astype(np.float32)
    # grid finer than the particles: tetrahedra spanning several cells and
    # tetrahedra inside one cell both occur
    plan = P.make_plan(pos, w, vel, sc, grid=(17, 15, 19), n_threads=n_threads,
                       average_density_value=float(w.sum()) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    ora = O.method1(plan, d32, d64, FIELDS, n_points=nn, mode=O.MODE_REF)
    o64 = O.method1(plan, d32, d64, FIELDS, n_points=nn, mode=O.MODE_FP64)
    for k, b in enumerate(plan.box_list()):
        ref = R.run(plan, k, which=1, n_points=nn, dens_override=d32)
        ox, oy, oz = b.tile_origin[0], b.tile_origin[1], b.tile_origin[2]
        dims = (b.tile_dims[0], b.tile_dims[1], b.tile_dims[2])
        for f in FIELDS:
            full = ora[f].reshape(plan.grid + ora[f].shape[1:])
            tile = full[ox:ox + dims[0], oy:oy + dims[1], oz:oz + dims[2]].reshape(ref[f].shape)
            assert np.array_equal(tile.astype(np.float32), ref[f]), (k, f)
    for f in FIELDS:
        assert rel_err(ora[f], o64[f]) <= 1e-5, f
    assert np.abs(ora["density"]).max() > 0


def _sparse_plan():
    """40 particles, no periodic images, a small explicit padding, 16
    sub-boxes: several sub-boxes have no tetrahedra (fewer than 4 particles),
    others one to four, and many cell centres lie outside every hull."""
    rng = np.random.default_rng(1)
    pos = (rng.random((40, 3)) * 100).astype(np.float32)
    vel = rng.standard_normal((40, 3)).astype(np.float32)
    return P.make_plan(pos, rng.uniform(0.5, 1.5, 40).astype(np.float32), vel, None, grid=(16, 16, 16),
                       n_threads=16, periodic=False, padding=np.ones(6, np.float32), average_density_value=1e-3)


def test_live_sparse_subboxes(built):
    """Sub-boxes without tetrahedra give zeros, as the reference's triangulation
    with fewer than four vertices; after an outside sample the reference's
    cell-centre raster keeps the outside point for the rest of its z pencil
    (zeros).  The oracle reproduces both, bit for bit, for methods 0, 3, 1;
    DTFE_FLAG_FIX_OUTSIDE_RASTER evaluates those samples instead."""
    plan = _sparse_plan()
    assert min(b.n_tets for b in plan.boxes) == 0 and max(b.n_tets for b in plan.boxes) > 0
    d32, d64, _ = O.vertex_density(plan)
    fields = ["density", "velocity", "velocity_gradient"]
    for method, nn in ((0, 1), (3, 8), (1, 100)):
        if method == 1:
            ora = O.method1(plan, d32, d64, fields, n_points=nn, mode=O.MODE_REF)
        else:
            ora, _ = O.interpolate(plan, d32, d64, fields, method=method, n_samples=nn, mode=O.MODE_REF)
        for k, b in enumerate(plan.box_list()):
            ref = R.run(plan, k, which=method, n_points=nn, dens_override=d32)
            ox, oy, oz = b.tile_origin[0], b.tile_origin[1], b.tile_origin[2]
            dims = (b.tile_dims[0], b.tile_dims[1], b.tile_dims[2])
            for f in fields:
                full = ora[f].reshape(plan.grid + ora[f].shape[1:])
                tile = full[ox:ox + dims[0], oy:oy + dims[1], oz:oz + dims[2]].reshape(ref[f].shape)
                assert np.array_equal(tile.astype(np.float32), ref[f]), (method, k, f)
    fixed, _ = O.interpolate(plan, d32, d64, fields, method=0, mode=O.MODE_REF, fix_outside=True)
    compat, _ = O.interpolate(plan, d32, d64, fields, method=0, mode=O.MODE_REF)
    moved = np.abs(fixed["velocity"] - compat["velocity"]).sum(1) > 0
    assert moved.any() and not (np.abs(compat["velocity"][moved]).sum(1) > 0).any()


def test_live_user_sampling(built):
    """Fields at user sampling points: the reference's interpolateUserSampling
    (one box, as DTFE() runs user samples) against the oracle's float mode,
    bit for bit: points outside the region dropped, points outside the hull
    zeros, the rest evaluated as cell centres are."""
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=51)
    rng = np.random.default_rng(52)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 1)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, sc, grid=(12, 12, 12), n_threads=1, average_density_value=float(w.sum()) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    # the padded hull reaches about 40 beyond the box: points up to 80 beyond
    pts = np.concatenate([rng.uniform(-80, 180, (3000, 3)), rng.uniform(0, 100, (2000, 3))]).astype(np.float32)
    pts[:20] = plan.xyz[:20]                       # on vertices (ties)
    region = np.array([-70, 170, -60, 160, -70, 150], np.float32)
    fields = ["density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"]
    ora = O.interpolate_points(plan, d32, d64, fields, pts, region, mode=O.MODE_REF)
    ref = R.run_points(plan, pts, region, d32)
    keep = np.all((pts >= region[0::2]) & (pts <= region[1::2]), axis=1)
    assert len(ref["density"]) == keep.sum() == len(ora["density"])
    for f in fields:
        assert np.array_equal(ora[f].astype(np.float32), ref[f]), f
    assert (ora["density"] == 0).any() and (ora["density"] != 0).any()


def test_live_redshift_cone(built):
    """Fields on a redshift-cone grid: the reference's interpolateRedshiftCone
    (one box, as DTFE() runs cones) against the oracle's float mode, bit for
    bit, on a cone whose outer shells leave the padded hull (zeros, and the
    reference's stuck psi: the rest of such a psi pencil stays zero) and whose
    psi range wraps through 360 degrees."""
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=53)
    rng = np.random.default_rng(54)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 1)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, sc, grid=(12, 12, 12), n_threads=1, average_density_value=float(w.sum()) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    fields = ["density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"]
    for cone, origin, dims in [((1.0, 120.0, 10.0, 170.0, 300.0, 60.0), (50.0, 50.0, 50.0), (9, 7, 11)),
                               ((0.5, 60.0, 0.0, 180.0, 0.0, 359.0), (20.0, 70.0, 40.0), (6, 5, 13))]:
        ora = O.interpolate_cone(plan, d32, d64, fields, cone, origin, dims, mode=O.MODE_REF)
        ref = R.run_cone(plan, cone, origin, dims, d32)
        for f in fields:
            assert np.array_equal(ora[f].astype(np.float32), ref[f]), (cone, f)
    # the first cone reaches outside the hull, and the stuck psi zeroes samples
    # that would have been inside
    cone, origin, dims = (1.0, 120.0, 10.0, 170.0, 300.0, 60.0), (50.0, 50.0, 50.0), (9, 7, 11)
    ora = O.interpolate_cone(plan, d32, d64, ["density"], cone, origin, dims, mode=O.MODE_REF)
    fixed = O.interpolate_cone(plan, d32, d64, ["density"], cone, origin, dims, mode=O.MODE_REF, fix_outside=True)
    assert (ora["density"] == 0).any() and (ora["density"] != 0).any()
    assert ((ora["density"] == 0) & (fixed["density"] != 0)).any()


def test_live_averaged_samples_statistical(built):
    """Monte-Carlo volume averages at user points and on a redshift cone: the
    oracle (Philox offsets) against the reference's own
    interpolateUserSampling_averaged_2 / interpolateRedshiftCone_averaged_2
    (its mt19937 offsets).  The random points differ, so the check is
    statistical: the median absolute difference oracle - reference matches
    the one between two oracle seeds (the same estimator spread) within 25%
    (medians, since a rare sample in a sliver tetrahedron carries a huge
    gradient), and the mean difference lies within 4 standard errors of
    zero."""
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=61)
    rng = np.random.default_rng(62)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (60 * psi).astype(np.float32)
    plan = P.make_plan(pos, w, vel, None, grid=(12, 12, 12), n_threads=1, average_density_value=float(w.sum()) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    fields = ["density", "velocity", "velocity_gradient"]
    pts = rng.uniform(5, 95, (2000, 3)).astype(np.float32)
    delta = rng.uniform(2, 8, (2000, 3)).astype(np.float32)
    region = np.array([0, 100, 0, 100, 0, 100], np.float32)
    cone, origin, dims = (1.0, 45.0, 5.0, 175.0, 0.0, 350.0), (50.0, 50.0, 50.0), (8, 10, 25)
    NN = 16
    cases = [(O.average_points(plan, d32, d64, fields, pts, delta, region, NN, seed=1),
              O.average_points(plan, d32, d64, fields, pts, delta, region, NN, seed=2),
              R.run_average(plan, d32, NN, 3, pts=pts, delta=delta, region=region)),
             (O.average_cone(plan, d32, d64, fields, cone, origin, dims, NN, seed=1),
              O.average_cone(plan, d32, d64, fields, cone, origin, dims, NN, seed=2),
              R.run_average(plan, d32, NN, 3, cone=cone, origin=origin, dims=dims))]
    for a, b, ref in cases:
        for f in fields:
            assert len(ref[f]) == len(a[f])
            d_ref = (a[f].astype(np.float32) - ref[f]).astype(np.float64).ravel()
            d_self = (a[f] - b[f]).ravel()
            ratio = np.median(np.abs(d_ref)) / np.median(np.abs(d_self))
            assert 0.8 < ratio < 1.25, (f, ratio)
            assert abs(d_ref.mean()) < 4 * d_ref.std() / np.sqrt(d_ref.size), f


@pytest.mark.skipif(not __import__("os").path.exists(R.MAIN_LIB), reason="reference DTFE.cpp harness not built")
def test_live_divergence_shear_vorticity(built):
    """Divergence, shear and vorticity of the oracle in the reference's
    arithmetic (the GPU's fused epilogue is bit-identical to it) against the
    reference's own computeDivergenceShearVorticity (src/DTFE.cpp:436-475,
    compiled in the harness) applied to the same float gradient: bit for
    bit."""
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.9, seed=31)
    vel = (80 * psi + np.random.default_rng(32).normal(0, 20, psi.shape)).astype(np.float32)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), vel, None, grid=(14, 12, 10), n_threads=3,
                       average_density_value=len(pos) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    fields = ["velocity_gradient", "velocity_divergence", "velocity_shear", "velocity_vorticity"]
    ora, _ = O.interpolate(plan, d32, d64, fields, mode=O.MODE_REF)
    div, sh, vo, _ = R.derived(ora["velocity_gradient"].astype(np.float32))
    assert np.array_equal(div, ora["velocity_divergence"].astype(np.float32))
    assert np.array_equal(sh, ora["velocity_shear"].astype(np.float32))
    assert np.array_equal(vo, ora["velocity_vorticity"].astype(np.float32))
