"""Generates tests/golden/*.npz from the reference's own code.

Runs where the reference tree is available (the harness in oracle/_ref is
built from it by ``make -C oracle ref``); the fixtures are committed so that
tests on machines without the reference (the GPU host) check against the
reference's outputs.

    python tests/golden/make_golden.py

ref_zeldovich10.npz — a 10^3 Zel'dovich lattice (rms 0.5 spacing, weights
U[0.5,1.5], velocities, one scalar) in a periodic 100 Mpc/h box, padding of 2
particle spacings, tessellated by this project's tessellator (stored, so the
fixture does not depend on it), then:
  * vertexDensity of the reference (its float accumulation);
  * interpolateGrid (cell centres) of density, velocity, gradient, scalar,
    scalar gradient on a 10^3 grid, with the reference's own vertex densities;
  * interpolateGrid_averaged_3 with 8 equidistant points per cell;
  * interpolateGrid_averaged_1 with 100 points per cell (the reference's
    default method and count; its GSL Sobol generator stood in by
    dtfe_b200/csrc/sobol.h);
  * interpolateUserSampling at 600 points (some outside the region, some
    beyond the hull, ten on vertices) and interpolateRedshiftCone on a
    7 x 6 x 9 cone whose psi range wraps and whose outer shells leave the
    hull, both with the reference's own vertex densities;
  * NGP / CIC / TSC density and velocity of the same particles in a region;
  * SPH_interpolation (32 neighbours) density, velocity and intensive scalar
    of the padded particle set on the 10^3 grid of the box;
  * parallelGrid for 1..64 threads on three grids, optimalPartitionSplit and
    findParticlesInBox on the particle set.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from dtfe_b200 import plan as P  # noqa: E402
from dtfe_b200 import synthetic as S  # noqa: E402
import refharness as R  # noqa: E402


def main():
    if not R.available():
        raise SystemExit("reference harness not built (make -C oracle ref)")
    L = R.lib()
    vp = C.c_void_p
    L.ref_parallel_grid.argtypes = [C.c_int64, vp, vp]
    L.ref_optimal_partition.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp]
    L.ref_select_in_box.argtypes = [vp, C.c_int64, vp, vp, C.c_int, vp]
    L.ref_select_in_box.restype = C.c_int64
    L.ref_deposit.argtypes = [C.c_int, vp, vp, vp, C.c_int64, vp, vp, C.c_double, vp, vp]
    L.ref_sph.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int64, vp, vp, C.c_double, C.c_int, vp, vp, vp]

    n = 10
    pos, psi = S.zeldovich_lattice(n, 100.0, 0.5, seed=11)
    w = np.random.default_rng(12).uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (100.0 * psi / (100.0 / n)).astype(np.float32)
    sc = np.random.default_rng(13).standard_normal((len(pos), 1)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, sc, grid=(n, n, n), n_threads=1, padding_particles=2.0,
                       average_density_value=float(w.sum()) / 1e6)
    out = {
        "particles_pos": pos, "particles_w": w, "particles_vel": vel, "particles_scalar": sc,
        "tet_v": plan.tet_v, "tet_n": plan.tet_n, "xyz": plan.xyz, "weight": plan.weight,
        "velocity": plan.velocity, "scalar": plan.scalar, "xs": plan.xs, "ys": plan.ys, "zs": plan.zs,
        "grid": np.array(plan.grid, np.int32), "rho_bar": np.float64(plan.rho_bar),
        "padding": plan.padding,
    }
    b = plan.boxes[0]
    out["box_lo"] = np.array(list(b.lo), np.float32)
    out["box_dx"] = np.array(list(b.dx), np.float32)
    out["region"] = plan.region_array()[0]
    centre = R.run(plan, 0, which=0)
    out["ref_vertex_density"] = centre["vertex_density"]
    for f in ("density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"):
        out["ref_centre_" + f] = centre[f]
    eq = R.run(plan, 0, which=3, n_points=8)
    for f in ("density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"):
        out["ref_equidistant8_" + f] = eq[f]
    m1 = R.run(plan, 0, which=1, n_points=100)
    for f in ("density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"):
        out["ref_method1_100_" + f] = m1[f]

    rho_ref = centre["vertex_density"]
    pts = np.random.default_rng(14).uniform(-40, 140, (600, 3)).astype(np.float32)
    pts[:10] = plan.xyz[:10]
    pregion = np.array([-30, 130, -25, 125, -30, 130], np.float32)
    up = R.run_points(plan, pts, pregion, rho_ref)
    out["points_xyz"], out["points_region"] = pts, pregion
    for f in ("density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"):
        out["ref_points_" + f] = up[f]
    cone = np.array([1.0, 95.0, 5.0, 175.0, 300.0, 60.0], np.float32)
    origin = np.array([50.0, 45.0, 55.0], np.float32)
    cdims = np.array([7, 6, 9], np.int32)
    uc = R.run_cone(plan, cone, origin, cdims, rho_ref)
    out["cone_limits"], out["cone_origin"], out["cone_dims"] = cone, origin, cdims
    for f in ("density", "velocity", "velocity_gradient", "scalar", "scalar_gradient"):
        out["ref_cone_" + f] = uc[f]

    region = np.array([10, 90, 5, 95, 0, 100], np.float32)
    dgrid = np.array([8, 9, 10], np.int32)
    out["deposit_region"], out["deposit_grid"] = region, dgrid
    G = int(np.prod(dgrid))
    for k, name in enumerate(("ngp", "cic", "tsc")):
        dd = np.zeros(G, np.float32)
        dv = np.zeros((G, 3), np.float32)
        L.ref_deposit(k, pos.ctypes.data, w.ctypes.data, vel.ctypes.data, len(pos), region.ctypes.data,
                      dgrid.ctypes.data, plan.rho_bar, dd.ctypes.data, dv.ctypes.data)
        out[f"ref_{name}_density"], out[f"ref_{name}_velocity"] = dd, dv

    box = np.array([0, 100, 0, 100, 0, 100], np.float32)
    g3 = np.array(plan.grid, np.int32)
    G3 = int(np.prod(g3))
    sd, sv, ss = np.zeros(G3, np.float32), np.zeros((G3, 3), np.float32), np.zeros(G3, np.float32)
    sc1 = np.ascontiguousarray(plan.scalar[:, 0])
    rc = L.ref_sph(plan.xyz.ctypes.data, plan.weight.ctypes.data, plan.velocity.ctypes.data, sc1.ctypes.data, 0,
                   plan.n_verts, box.ctypes.data, g3.ctypes.data, plan.rho_bar, 32, sd.ctypes.data, sv.ctypes.data,
                   ss.ctypes.data)
    assert rc == 0
    out["ref_sph32_density"], out["ref_sph32_velocity"], out["ref_sph32_scalar"] = sd, sv, ss

    grids = np.array([[256, 256, 256], [8, 8, 8], [4, 16, 2]], np.int64)
    table = np.zeros((len(grids), 64, 3), np.int64)
    for gi, g in enumerate(grids):
        for t in range(1, 65):
            o = np.zeros(3, np.int64)
            L.ref_parallel_grid(t, g.ctypes.data, o.ctypes.data)
            table[gi, t - 1] = o
    out["pgrid_grids"], out["pgrid_table"] = grids, table
    parts = np.array([2, 3, 2], np.int64)
    pg = np.array([20, 24, 16], np.int64)
    full = np.array([0, 100, 0, 100, 0, 100], np.float32)
    sub = np.zeros((12, 6), np.int64)
    co = np.zeros((12, 6), np.float32)
    L.ref_optimal_partition(pos.ctypes.data, len(pos), pg.ctypes.data, full.ctypes.data, parts.ctypes.data,
                            sub.ctypes.data, co.ctypes.data)
    out["part_parts"], out["part_grid"], out["part_subgrid"], out["part_coords"] = parts, pg, sub, co
    padded = np.array([-7.5, 108.25, -3.0, 103.0, -11.0, 100.5], np.float32)
    cnt = L.ref_select_in_box(pos.ctypes.data, len(pos), full.ctypes.data, padded.ctypes.data, 1, None)
    sel = np.zeros((cnt, 3), np.float32)
    L.ref_select_in_box(pos.ctypes.data, len(pos), full.ctypes.data, padded.ctypes.data, 1, sel.ctypes.data)
    out["select_padded"], out["select_pos"] = padded, sel
    path = os.path.join(HERE, "ref_zeldovich10.npz") if len(sys.argv) < 2 else sys.argv[1]
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
