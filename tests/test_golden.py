"""The oracle and the host planning against the reference's own outputs
(tests/golden/ref_zeldovich10.npz, generated by tests/golden/make_golden.py
from the reference's sources).

Bars: bit-exact for the interpolation given the reference's vertex densities,
for NGP/CIC/TSC and for the planning functions; 1e-6 relative for vertex
densities (the reference sums volumes in float, the oracle in double).
"""
import numpy as np
import pytest

import oracle as O
from conftest import golden, golden_plan, rel_err
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

FIELDS = ["density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"]


@pytest.fixture(scope="module")
def g(built):
    return golden()


def test_fixture_inputs_reproducible(g):
    pos, _ = S.zeldovich_lattice(10, 100.0, 0.5, seed=11)
    assert np.array_equal(pos, g["particles_pos"])


def test_vertex_density_vs_reference(g):
    plan = golden_plan(g)
    d32, d64, _ = O.vertex_density(plan)
    ref = g["ref_vertex_density"]
    assert rel_err(d32, ref) <= 1e-6
    assert rel_err(d64, ref) <= 1e-6


@pytest.mark.parametrize("method,nn,tag", [(0, 1, "centre"), (3, 8, "equidistant8")])
def test_interpolation_bit_exact_vs_reference(g, method, nn, tag):
    plan = golden_plan(g)
    _, d64, _ = O.vertex_density(plan)
    ref_dens = np.ascontiguousarray(g["ref_vertex_density"])
    out, _ = O.interpolate(plan, ref_dens, d64, FIELDS, method=method, n_samples=nn, mode=O.MODE_REF)
    for f in FIELDS:
        want = g[f"ref_{tag}_{f}"].reshape(out[f].shape)
        assert np.array_equal(out[f].astype(np.float32), want), f


def test_method1_bit_exact_vs_reference(g):
    """Averaging method 1 with the reference's default 100 points per cell
    (its own vertex densities): the oracle's float mode reproduces the
    reference's interpolateGrid_averaged_1 bit for bit."""
    plan = golden_plan(g)
    _, d64, _ = O.vertex_density(plan)
    ref_dens = np.ascontiguousarray(g["ref_vertex_density"])
    out = O.method1(plan, ref_dens, d64, FIELDS, n_points=100, mode=O.MODE_REF)
    for f in FIELDS:
        want = g[f"ref_method1_100_{f}"].reshape(out[f].shape)
        assert np.array_equal(out[f].astype(np.float32), want), f


@pytest.mark.parametrize("kind,name", [(0, "ngp"), (1, "cic"), (2, "tsc")])
def test_deposit_bit_exact_vs_reference(g, kind, name):
    import ctypes as C
    L = O.lib()
    pos, w, vel = g["particles_pos"], g["particles_w"], g["particles_vel"]
    region, grid = g["deposit_region"], g["deposit_grid"]
    G = int(np.prod(grid))
    d = np.zeros(G)
    v = np.zeros((G, 3))
    L.oracle_deposit(kind, O.MODE_REF, pos.ctypes.data, w.ctypes.data, vel.ctypes.data, len(pos),
                     region.ctypes.data, grid.ctypes.data, float(g["rho_bar"]), d.ctypes.data, v.ctypes.data)
    assert np.array_equal(d.astype(np.float32), g[f"ref_{name}_density"])
    assert np.array_equal(v.astype(np.float32), g[f"ref_{name}_velocity"])


def test_planning_bit_exact_vs_reference(g):
    for gi, grid in enumerate(g["pgrid_grids"]):
        for t in range(1, 65):
            assert P.parallel_grid(t, grid) == tuple(g["pgrid_table"][gi, t - 1]), (grid, t)
    sub, co = P.optimal_partition(g["particles_pos"], g["part_grid"], np.array([0, 100, 0, 100, 0, 100], np.float32),
                                  g["part_parts"])
    assert np.array_equal(sub, g["part_subgrid"])
    assert np.array_equal(co, g["part_coords"])
    _, sel = P.select_in_box(g["particles_pos"], np.array([0, 100, 0, 100, 0, 100], np.float32),
                             g["select_padded"], True)
    assert np.array_equal(sel, g["select_pos"])


def test_sph_bit_exact_vs_reference(g):
    """SPH_interpolation with 32 neighbours (density, velocity, intensive
    scalar) of the fixture's padded particle set: the oracle in the
    reference's float arithmetic equals the reference's own output."""
    plan = golden_plan(g)
    plan.scalar = g["scalar"]
    dens, vel, sc = O.sph(plan, k=32, velocity=True, scalars=True, mode=O.MODE_REF)
    assert np.array_equal(dens.astype(np.float32), g["ref_sph32_density"])
    assert np.array_equal(vel.astype(np.float32), g["ref_sph32_velocity"])
    assert np.array_equal(sc[:, 0].astype(np.float32), g["ref_sph32_scalar"])
    d64, v64, _ = O.sph(plan, k=32, velocity=True, mode=O.MODE_FP64)
    assert rel_err(d64, g["ref_sph32_density"]) < 1e-6


def test_user_points_and_cone_bit_exact_vs_reference(g):
    """interpolateUserSampling and interpolateRedshiftCone with the
    reference's own vertex densities: the oracle's float mode reproduces the
    reference's rows bit for bit (points dropped by the region, zeros beyond
    the hull, the cone's stuck psi)."""
    plan = golden_plan(g)
    _, d64, _ = O.vertex_density(plan)
    ref_dens = np.ascontiguousarray(g["ref_vertex_density"])
    pts = O.interpolate_points(plan, ref_dens, d64, FIELDS, g["points_xyz"], g["points_region"], mode=O.MODE_REF)
    cone = O.interpolate_cone(plan, ref_dens, d64, FIELDS, g["cone_limits"], g["cone_origin"], g["cone_dims"],
                              mode=O.MODE_REF)
    for f in FIELDS:
        assert np.array_equal(pts[f].astype(np.float32), g[f"ref_points_{f}"].reshape(pts[f].shape)), f
        assert np.array_equal(cone[f].astype(np.float32), g[f"ref_cone_{f}"].reshape(cone[f].shape)), f
