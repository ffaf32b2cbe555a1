"""Python access to the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

Used by tests/, the smoke check and bench.py's CPU-baseline leg as the
checker; never by the product path.  See dtfe_oracle.cpp for what it
restates and in which arithmetic modes.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from dtfe_b200 import _native as N  # noqa: E402  (struct definitions only)

MODE_REF, MODE_FP64 = 0, 1
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        from dtfe_b200 import build
        path = build.build_oracle()
        L = C.CDLL(path)
        vp = C.c_void_p
        L.oracle_vertex_density.argtypes = [C.c_int64, vp, vp, C.c_int64, vp, vp, C.c_double, vp, vp, vp,
                                            C.c_int, vp, C.c_int]
        L.oracle_vertex_density_ref.argtypes = [C.c_int64, vp, vp, C.c_int64, vp, vp, C.c_double, vp, C.c_int, vp,
                                                C.c_int]
        L.oracle_locate.argtypes = [C.c_int64, vp, vp, vp, C.c_int64, C.c_int64, C.c_int64, vp, vp]
        L.oracle_interpolate.argtypes = [C.c_int64, vp, vp, C.c_int64, vp, vp, vp, C.c_int, vp, vp, C.c_int,
                                         vp, vp, vp, vp, vp, C.POINTER(N.InterpOpts), C.c_int,
                                         C.POINTER(C.c_void_p), vp, C.c_int, vp]
        L.oracle_deposit.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int64, vp, vp, C.c_double, vp, vp]
        L.oracle_dtfe_loss.argtypes = [C.c_int64, vp, C.c_int64, vp, vp, vp, vp, C.c_double, C.c_int64, vp, vp,
                                       vp, vp, vp, C.c_int]
        L.oracle_dtfe_loss.restype = C.c_double
        L.oracle_dtfe_grad.argtypes = [C.c_int64, vp, C.c_int64, vp, vp, vp, vp, C.c_double, C.c_int64, vp, vp,
                                       vp, vp, vp, C.c_int, vp, vp, vp]
        L.oracle_sph.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int64, vp, vp, vp, vp, C.c_double, C.c_int, C.c_int,
                                 C.c_int, vp, vp, vp]
        L.oracle_dtfe_fd.argtypes = [C.c_int64, vp, C.c_int64, vp, vp, vp, vp, C.c_double, C.c_int64, vp, vp,
                                     vp, vp, vp, C.c_int, C.c_int64, vp, vp, C.c_double, C.c_double, C.c_double, vp]
        L.oracle_deposit_loss_grad.argtypes = [C.c_int, vp, vp, C.c_int64, vp, vp, C.c_double, vp, vp, vp]
        L.oracle_deposit_loss_grad.restype = C.c_double
        L.oracle_method1.argtypes = [C.c_int64, vp, C.c_int64, vp, vp, vp, C.c_int, vp, vp, C.c_int, vp, vp, vp,
                                     C.c_int, C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.oracle_interpolate_points.argtypes = [C.c_int64, vp, vp, C.c_int64, vp, vp, vp, C.c_int, vp, vp,
                                                C.c_int64, C.c_int64, C.c_int64, vp, vp, C.c_uint32, C.c_int,
                                                C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
        L.oracle_cone_tables.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.oracle_interpolate_cone.argtypes = [C.c_int64, vp, vp, C.c_int64, vp, vp, vp, C.c_int, vp, vp,
                                              C.c_int64, C.c_int64, vp, vp, vp, C.c_uint32, C.c_int, C.c_int,
                                              C.c_int, C.POINTER(C.c_void_p)]
        L.oracle_average_points.argtypes = [C.c_int64, vp, vp, C.c_int64, vp, vp, vp, C.c_int, vp, vp, C.c_int64,
                                            C.c_int64, C.c_int64, vp, vp, vp, C.c_uint32, C.c_int, C.c_uint64,
                                            C.c_int, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
        L.oracle_average_cone.argtypes = [C.c_int64, vp, vp, C.c_int64, vp, vp, vp, C.c_int, vp, vp, C.c_int64,
                                          C.c_int64, vp, vp, vp, C.c_uint32, C.c_int, C.c_uint64, C.c_int, C.c_int,
                                          C.POINTER(C.c_void_p)]
        L.oracle_sobol_simplex.argtypes = [C.c_int64, vp]
        L.oracle_sobol_simplex.restype = None
        _lib = L
    return _lib


def deposit(dplan, mode: int = MODE_REF, velocity: bool = True):
    """NGP / CIC / TSC per region (NGP/CIC/TSC_interpolation_regular_grid),
    placed into the main grid: (density (G,), velocity (G, 3) or None)."""
    g = dplan.grid
    dens = np.zeros(g, np.float64)
    vel = np.zeros(g + (3,), np.float64) if velocity and dplan.velocity is not None else None
    for b in dplan.boxes:
        o, n = b.particle_offset, b.n_particles
        dims = np.array([b.tile_dims[0], b.tile_dims[1], b.tile_dims[2]], np.int32)
        region = np.array(list(b.region), np.float32)
        td = np.zeros(int(np.prod(dims)), np.float64)
        tv = np.zeros((int(np.prod(dims)), 3), np.float64) if vel is not None else None
        pos = np.ascontiguousarray(dplan.pos[o:o + n])
        w = np.ascontiguousarray(dplan.weight[o:o + n])
        v = np.ascontiguousarray(dplan.velocity[o:o + n]) if vel is not None else None
        rc = lib().oracle_deposit(dplan.kind, mode, pos.ctypes.data, w.ctypes.data,
                                  None if v is None else v.ctypes.data, n, region.ctypes.data, dims.ctypes.data,
                                  dplan.rho_bar, td.ctypes.data, None if tv is None else tv.ctypes.data)
        if rc:
            raise RuntimeError("oracle_deposit failed")
        x0, y0, z0 = b.tile_origin[0], b.tile_origin[1], b.tile_origin[2]
        dens[x0:x0 + dims[0], y0:y0 + dims[1], z0:z0 + dims[2]] = td.reshape(dims)
        if vel is not None:
            vel[x0:x0 + dims[0], y0:y0 + dims[1], z0:z0 + dims[2]] = tv.reshape(tuple(dims) + (3,))
    G = int(np.prod(g))
    return dens.reshape(G), None if vel is None else vel.reshape(G, 3)


def sph_region(pos, w, vel, scal, xs, ys, zs, avg: float, k: int = 32, extensive: bool = False,
               mode: int = MODE_REF):
    """SPH_interpolation for one region's particles and grid point tables:
    (density (G,), velocity (G, 3) or None, scalars (G, S) or None), doubles."""
    pos = np.ascontiguousarray(pos, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    S = 0 if scal is None else int(np.asarray(scal).reshape(len(pos), -1).shape[1])
    vel_a = None if vel is None else np.ascontiguousarray(vel, np.float32)
    sc_a = None if scal is None else np.ascontiguousarray(np.asarray(scal, np.float32).reshape(len(pos), S))
    xs, ys, zs = (np.ascontiguousarray(a, np.float32) for a in (xs, ys, zs))
    dims = np.array([len(xs), len(ys), len(zs)], np.int32)
    G = int(np.prod(dims))
    dens = np.zeros(G)
    vo = np.zeros((G, 3)) if vel is not None else None
    so = np.zeros((G, S)) if S else None
    rc = lib().oracle_sph(pos.ctypes.data, w.ctypes.data, None if vel_a is None else vel_a.ctypes.data,
                          None if sc_a is None else sc_a.ctypes.data, S, len(pos), xs.ctypes.data, ys.ctypes.data,
                          zs.ctypes.data, dims.ctypes.data, float(avg), int(k), int(extensive), int(mode),
                          dens.ctypes.data, None if vo is None else vo.ctypes.data,
                          None if so is None else so.ctypes.data)
    if rc:
        raise RuntimeError("oracle_sph failed")
    return dens, vo, so


def sph(plan, k: int = 32, velocity: bool = True, scalars: bool = False, extensive: bool = False,
        mode: int = MODE_REF):
    """SPH over every sub-box of a DTFE plan (its padded particle sets and
    grid tiles), placed into the main grid: (density (G,), velocity (G, 3) or
    None, scalars (G, S) or None)."""
    g = plan.grid
    G = int(np.prod(g))
    S = plan.n_scalars if scalars else 0
    dens = np.zeros(g)
    vel = np.zeros(g + (3,)) if velocity else None
    sc = np.zeros(g + (S,)) if S else None
    for b in plan.boxes:
        o, n = b.vert_offset, b.n_verts
        d = [b.tile_dims[a] for a in range(3)]
        org = [b.tile_origin[a] for a in range(3)]
        co = [b.coord_offset[a] for a in range(3)]
        xs = plan.xs[co[0]:co[0] + d[0]]
        ys = plan.ys[co[1]:co[1] + d[1]]
        zs = plan.zs[co[2]:co[2] + d[2]]
        sv = plan.scalar[o:o + n] if S else None
        dd, vv, ss = sph_region(plan.xyz[o:o + n], plan.weight[o:o + n],
                                plan.velocity[o:o + n] if velocity else None, sv, xs, ys, zs, plan.rho_bar, k,
                                extensive, mode)
        sl = (slice(org[0], org[0] + d[0]), slice(org[1], org[1] + d[1]), slice(org[2], org[2] + d[2]))
        dens[sl] = dd.reshape(d)
        if vel is not None:
            vel[sl] = vv.reshape(tuple(d) + (3,))
        if sc is not None:
            sc[sl] = ss.reshape(tuple(d) + (S,))
    return dens.reshape(G), None if vel is None else vel.reshape(G, 3), None if sc is None else sc.reshape(G, S)


def vertex_density(plan, rho_bar: float | None = None, nthreads: int = 0):
    """(dens32 float32 (V,), dens64 float64 (V,), volsum float64 (V,)).
    nthreads 0 = all host threads (parallel over sub-boxes)."""
    rb = plan.rho_bar if rho_bar is None else rho_bar
    V = plan.n_verts
    d32 = np.empty(V, np.float32)
    d64 = np.empty(V, np.float64)
    vs = np.empty(V, np.float64)
    lib().oracle_vertex_density(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, V,
                                plan.xyz.ctypes.data, plan.weight.ctypes.data, rb,
                                d32.ctypes.data, d64.ctypes.data, vs.ctypes.data,
                                plan.n_boxes, C.addressof(plan.boxes), nthreads or (os.cpu_count() or 1))
    return d32, d64, vs


def vertex_density_ref(plan, rho_bar: float | None = None, nthreads: int = 0) -> np.ndarray:
    """The reference's own vertexDensity arithmetic (float sums of the
    incident cells' float volumes in ascending cell id): float32 (V,)."""
    rb = plan.rho_bar if rho_bar is None else rho_bar
    out = np.empty(plan.n_verts, np.float32)
    lib().oracle_vertex_density_ref(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, plan.n_verts,
                                    plan.xyz.ctypes.data, plan.weight.ctypes.data, rb, out.ctypes.data,
                                    plan.n_boxes, C.addressof(plan.boxes), nthreads or (os.cpu_count() or 1))
    return out


def locate(plan, pts: np.ndarray, box: int = 0) -> np.ndarray:
    pts = np.ascontiguousarray(pts, np.float64)
    b = plan.boxes[box]
    out = np.empty(len(pts), np.int64)
    lib().oracle_locate(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, plan.xyz.ctypes.data,
                        b.tet_offset, b.tet_offset + b.n_tets, len(pts), pts.ctypes.data, out.ctypes.data)
    return out


def interpolate(plan, dens32, dens64, fields, method: int = 0, n_samples: int = 1, seed: int = 0,
                mode: int = MODE_REF, fix: bool = False, nthreads: int = 1, want_loc: bool = False,
                fix_outside: bool = False):
    """Returns (dict field -> float64 array shaped (G, ncomp) or (G,), loc or None)."""
    G = int(np.prod(plan.grid))
    S = plan.n_scalars
    mask = 0
    outs = [None] * N.NUM_FIELDS
    arrs = {}
    for f in fields:
        s = N.FIELD_SLOTS[f]
        mask |= 1 << s
        nc = N.field_components(s, S)
        a = np.zeros((G, nc) if nc > 1 else G, np.float64)
        arrs[f] = a
        outs[s] = a.ctypes.data
    optr = (C.c_void_p * N.NUM_FIELDS)(*[o if o else None for o in outs])
    o = N.InterpOpts(method, n_samples, seed, mask, (N.FLAG_FIX_VALUE_INTERP if fix else 0) |
                     (N.FLAG_FIX_OUTSIDE_RASTER if fix_outside else 0))
    loc = np.full(G, -1, np.int64) if want_loc else None
    nfail = C.c_int64(0)
    vel = plan.velocity.ctypes.data if plan.velocity is not None else None
    sc = plan.scalar.ctypes.data if plan.scalar is not None else None
    grid = np.asarray(plan.grid, np.int32)
    rc = lib().oracle_interpolate(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, plan.n_verts,
                                  plan.xyz.ctypes.data, vel, sc, S,
                                  None if dens32 is None else dens32.ctypes.data,
                                  None if dens64 is None else dens64.ctypes.data,
                                  plan.n_boxes, C.addressof(plan.boxes), plan.xs.ctypes.data, plan.ys.ctypes.data,
                                  plan.zs.ctypes.data, grid.ctypes.data, C.byref(o), mode, optr,
                                  None if loc is None else loc.ctypes.data, nthreads, C.byref(nfail))
    if rc not in (0, 5):
        raise RuntimeError(f"oracle_interpolate failed with status {rc}")
    if nfail.value:
        raise RuntimeError(f"oracle walk failed on {nfail.value} samples")
    return arrs, loc


def method1(plan, dens32, dens64, fields, n_points: int = 100, mode: int = MODE_REF, fix: bool = False):
    """Averaging method 1 (points inside each tetrahedron scattered to the
    grid, interpolateGrid_averaged_1): dict field -> float64 array."""
    G = int(np.prod(plan.grid))
    S = plan.n_scalars
    mask = 0
    outs = [None] * N.NUM_FIELDS
    arrs = {}
    for f in fields:
        s = N.FIELD_SLOTS[f]
        mask |= 1 << s
        nc = N.field_components(s, S)
        a = np.zeros((G, nc) if nc > 1 else G, np.float64)
        arrs[f] = a
        outs[s] = a.ctypes.data
    optr = (C.c_void_p * N.NUM_FIELDS)(*[o if o else None for o in outs])
    vel = plan.velocity.ctypes.data if plan.velocity is not None else None
    sc = plan.scalar.ctypes.data if plan.scalar is not None else None
    grid = np.asarray(plan.grid, np.int32)
    regions = plan.region_array()
    rc = lib().oracle_method1(plan.n_tets, plan.tet_v.ctypes.data, plan.n_verts, plan.xyz.ctypes.data, vel, sc, S,
                              dens32.ctypes.data, dens64.ctypes.data, plan.n_boxes, C.addressof(plan.boxes),
                              regions.ctypes.data, grid.ctypes.data, n_points, mask, 1 if fix else 0, mode, optr)
    if rc:
        raise RuntimeError(f"oracle_method1 failed with status {rc}")
    return arrs


def interpolate_points(plan, dens32, dens64, fields, pts, region, mode: int = MODE_REF, fix: bool = False,
                       box: int = 0):
    """Fields at user sampling points (interpolateUserSampling) in the
    tessellation of sub-box `box`: dict field -> float64 array of the points
    inside `region`, in order."""
    pts = np.ascontiguousarray(pts, np.float32)
    n = len(pts)
    S = plan.n_scalars
    mask = 0
    outs = [None] * N.NUM_FIELDS
    arrs = {}
    for f in fields:
        s = N.FIELD_SLOTS[f]
        mask |= 1 << s
        nc = N.field_components(s, S)
        a = np.zeros((n, nc) if nc > 1 else n, np.float64)
        arrs[f] = a
        outs[s] = a.ctypes.data
    optr = (C.c_void_p * N.NUM_FIELDS)(*[o if o else None for o in outs])
    vel = plan.velocity.ctypes.data if plan.velocity is not None else None
    sc = plan.scalar.ctypes.data if plan.scalar is not None else None
    b = plan.boxes[box]
    reg = np.ascontiguousarray(region, np.float32)
    n_out = C.c_int64(0)
    rc = lib().oracle_interpolate_points(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, plan.n_verts,
                                         plan.xyz.ctypes.data, vel, sc, S, dens32.ctypes.data, dens64.ctypes.data,
                                         b.tet_offset, b.tet_offset + b.n_tets, n, pts.ctypes.data,
                                         reg.ctypes.data, mask, mode, 1 if fix else 0, optr, C.byref(n_out))
    if rc:
        raise RuntimeError(f"oracle_interpolate_points failed with status {rc}")
    return {f: a[:n_out.value] for f, a in arrs.items()}


def cone_tables(cone, dims):
    """Per-axis tables of a redshift-cone grid: r, sin(theta), cos(theta),
    cos(psi), sin(psi) as float32 arrays, in the reference's arithmetic."""
    c = np.ascontiguousarray(cone, np.float32)
    d = np.ascontiguousarray(dims, np.int32)
    r = np.zeros(max(int(d[0]), 1), np.float32)
    st, ct = np.zeros(max(int(d[1]), 1), np.float32), np.zeros(max(int(d[1]), 1), np.float32)
    cp, sp = np.zeros(max(int(d[2]), 1), np.float32), np.zeros(max(int(d[2]), 1), np.float32)
    rc = lib().oracle_cone_tables(c.ctypes.data, d.ctypes.data, r.ctypes.data, st.ctypes.data, ct.ctypes.data,
                                  cp.ctypes.data, sp.ctypes.data)
    if rc:
        raise ValueError(f"oracle_cone_tables refused the cone {list(cone)} (status {rc})")
    return r, st, ct, cp, sp


def interpolate_cone(plan, dens32, dens64, fields, cone, origin, dims, mode: int = MODE_REF, fix: bool = False,
                     fix_outside: bool = False, box: int = 0):
    """Fields on a redshift-cone grid (interpolateRedshiftCone) in the
    tessellation of sub-box `box`: dict field -> float64 array of
    dims[0] * dims[1] * dims[2] rows, r slowest and psi fastest."""
    n = int(np.prod(dims))
    S = plan.n_scalars
    mask = 0
    outs = [None] * N.NUM_FIELDS
    arrs = {}
    for f in fields:
        s = N.FIELD_SLOTS[f]
        mask |= 1 << s
        nc = N.field_components(s, S)
        a = np.zeros((n, nc) if nc > 1 else n, np.float64)
        arrs[f] = a
        outs[s] = a.ctypes.data
    optr = (C.c_void_p * N.NUM_FIELDS)(*[o if o else None for o in outs])
    vel = plan.velocity.ctypes.data if plan.velocity is not None else None
    sc = plan.scalar.ctypes.data if plan.scalar is not None else None
    b = plan.boxes[box]
    c = np.ascontiguousarray(cone, np.float32)
    o = np.ascontiguousarray(origin, np.float32)
    d = np.ascontiguousarray(dims, np.int32)
    rc = lib().oracle_interpolate_cone(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, plan.n_verts,
                                       plan.xyz.ctypes.data, vel, sc, S, dens32.ctypes.data, dens64.ctypes.data,
                                       b.tet_offset, b.tet_offset + b.n_tets, c.ctypes.data, o.ctypes.data,
                                       d.ctypes.data, mask, mode, 1 if fix else 0, 1 if fix_outside else 0, optr)
    if rc:
        raise RuntimeError(f"oracle_interpolate_cone failed with status {rc}")
    return arrs


def _outputs(fields, n, S):
    mask = 0
    outs = [None] * N.NUM_FIELDS
    arrs = {}
    for f in fields:
        s = N.FIELD_SLOTS[f]
        mask |= 1 << s
        nc = N.field_components(s, S)
        a = np.zeros((n, nc) if nc > 1 else n, np.float64)
        arrs[f] = a
        outs[s] = a.ctypes.data
    return mask, (C.c_void_p * N.NUM_FIELDS)(*[o if o else None for o in outs]), arrs


def average_points(plan, dens32, dens64, fields, pts, delta, region, n_samples: int, seed: int = 0,
                   mode: int = MODE_REF, fix: bool = False, box: int = 0):
    """Monte-Carlo volume averages at user sampling points
    (interpolateUserSampling_averaged_2) with the Philox offsets: dict field
    -> float64 array of the points inside `region`, in order."""
    pts = np.ascontiguousarray(pts, np.float32)
    delta = np.ascontiguousarray(delta, np.float32)
    n = len(pts)
    mask, optr, arrs = _outputs(fields, n, plan.n_scalars)
    vel = plan.velocity.ctypes.data if plan.velocity is not None else None
    sc = plan.scalar.ctypes.data if plan.scalar is not None else None
    b = plan.boxes[box]
    reg = np.ascontiguousarray(region, np.float32)
    n_out = C.c_int64(0)
    rc = lib().oracle_average_points(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, plan.n_verts,
                                     plan.xyz.ctypes.data, vel, sc, plan.n_scalars, dens32.ctypes.data,
                                     dens64.ctypes.data, b.tet_offset, b.tet_offset + b.n_tets, n, pts.ctypes.data,
                                     delta.ctypes.data, reg.ctypes.data, mask, n_samples, seed, mode,
                                     1 if fix else 0, optr, C.byref(n_out))
    if rc:
        raise RuntimeError(f"oracle_average_points failed with status {rc}")
    return {f: a[:n_out.value] for f, a in arrs.items()}


def average_cone(plan, dens32, dens64, fields, cone, origin, dims, n_samples: int, seed: int = 0,
                 mode: int = MODE_REF, fix: bool = False, box: int = 0):
    """Monte-Carlo bin averages on a redshift-cone grid
    (interpolateRedshiftCone_averaged_2) with the Philox offsets: dict field
    -> float64 array of dims[0] * dims[1] * dims[2] rows."""
    n = int(np.prod(dims))
    mask, optr, arrs = _outputs(fields, n, plan.n_scalars)
    vel = plan.velocity.ctypes.data if plan.velocity is not None else None
    sc = plan.scalar.ctypes.data if plan.scalar is not None else None
    b = plan.boxes[box]
    c = np.ascontiguousarray(cone, np.float32)
    o = np.ascontiguousarray(origin, np.float32)
    d = np.ascontiguousarray(dims, np.int32)
    rc = lib().oracle_average_cone(plan.n_tets, plan.tet_v.ctypes.data, plan.tet_n.ctypes.data, plan.n_verts,
                                   plan.xyz.ctypes.data, vel, sc, plan.n_scalars, dens32.ctypes.data,
                                   dens64.ctypes.data, b.tet_offset, b.tet_offset + b.n_tets, c.ctypes.data,
                                   o.ctypes.data, d.ctypes.data, mask, n_samples, seed, mode, 1 if fix else 0, optr)
    if rc:
        raise RuntimeError(f"oracle_average_cone failed with status {rc}")
    return arrs


def sobol_simplex(n: int) -> np.ndarray:
    """(n, 3) float32: the method-1 quasi-random table."""
    out = np.zeros((n, 3), np.float32)
    lib().oracle_sobol_simplex(n, out.ctypes.data)
    return out


# ---- adjoint checker -------------------------------------------------------

def cell_points(plan) -> np.ndarray:
    """(G, 3) float64 sample point of every main-grid cell (zeros outside
    every tile), as the interpolation evaluates them."""
    G1, G2 = plan.grid[1], plan.grid[2]
    pts = np.zeros((int(np.prod(plan.grid)), 3), np.float64)
    for b in plan.boxes:
        d = [b.tile_dims[a] for a in range(3)]
        i, j, k = np.meshgrid(np.arange(d[0]), np.arange(d[1]), np.arange(d[2]), indexing="ij")
        cell = ((b.tile_origin[0] + i) * G1 + (b.tile_origin[1] + j)) * G2 + (b.tile_origin[2] + k)
        pts[cell.ravel(), 0] = plan.xs[b.coord_offset[0] + i.ravel()]
        pts[cell.ravel(), 1] = plan.ys[b.coord_offset[1] + j.ravel()]
        pts[cell.ravel(), 2] = plan.zs[b.coord_offset[2] + k.ravel()]
    return pts


def hull_marks(plan) -> np.ndarray:
    """(V,) int32: 1 for vertices of a hull face (a face without neighbour)."""
    h = np.zeros(plan.n_verts, np.int32)
    tv, tn = plan.tet_v, plan.tet_n
    for f in range(4):
        faces = tn[:, f] < 0
        for a in range(4):
            if a != f:
                h[tv[faces, a]] = 1
    return h


class AdjointProblem:
    """FP64 loss L = sum a*density + c.velocity + b*divergence over the cell
    centres of a plan at frozen topology and frozen cell -> tetrahedron
    assignment ``loc``; ``factor`` = 4 / rho_bar as the forward rounds it."""

    def __init__(self, plan, loc, a=None, c=None, b=None, full_value: bool = False):
        self.plan = plan
        self.tv = np.ascontiguousarray(plan.tet_v, np.int32)
        self.hull = hull_marks(plan)
        self.pts = cell_points(plan)
        self.loc = np.ascontiguousarray(loc, np.int64)
        self.a = None if a is None else np.ascontiguousarray(a, np.float64)
        self.c = None if c is None else np.ascontiguousarray(c, np.float64)
        self.b = None if b is None else np.ascontiguousarray(b, np.float64)
        self.full = 1 if full_value else 0
        self.factor = float(np.float32(4.0 / float(np.float32(plan.rho_bar))))

    def _args(self, x, w, v):
        p = self.plan
        return (p.n_tets, self.tv.ctypes.data, p.n_verts, x.ctypes.data, w.ctypes.data, v.ctypes.data,
                self.hull.ctypes.data, self.factor, len(self.loc), self.loc.ctypes.data, self.pts.ctypes.data,
                None if self.a is None else self.a.ctypes.data, None if self.c is None else self.c.ctypes.data,
                None if self.b is None else self.b.ctypes.data, self.full)

    def loss(self, x, w, v) -> float:
        x, w, v = (np.ascontiguousarray(t, np.float64) for t in (x, w, v))
        return float(lib().oracle_dtfe_loss(*self._args(x, w, v)))

    def grad(self, x, w, v):
        """(gx (V,3), gv (V,3), gw (V,)) float64."""
        x, w, v = (np.ascontiguousarray(t, np.float64) for t in (x, w, v))
        V = self.plan.n_verts
        gx, gv, gw = np.zeros((V, 3)), np.zeros((V, 3)), np.zeros(V)
        lib().oracle_dtfe_grad(*self._args(x, w, v), gx.ctypes.data, gv.ctypes.data, gw.ctypes.data)
        return gx, gv, gw


def images_of(src: np.ndarray, particles: np.ndarray):
    """CSR (offsets, vertices) of the vertices that are images of each
    selected particle."""
    order = np.argsort(src, kind="stable")
    ss = src[order]
    lo = np.searchsorted(ss, particles, "left")
    hi = np.searchsorted(ss, particles, "right")
    off = np.zeros(len(particles) + 1, np.int64)
    off[1:] = np.cumsum(hi - lo)
    verts = np.concatenate([order[l:h] for l, h in zip(lo, hi)]).astype(np.int32) if len(particles) else \
        np.zeros(0, np.int32)
    return off, verts


def dtfe_fd(prob: "AdjointProblem", x, w, v, particles, h_pos: float, h_vel: float = 1e-3, h_w: float = 1e-4):
    """FP64 central differences of prob's loss for the selected particles:
    (n, 7) = d/d(x, y, z, vx, vy, vz, w), every image of a particle moved."""
    x, w, v = (np.ascontiguousarray(t, np.float64) for t in (x, w, v))
    off, verts = images_of(np.asarray(prob.plan.src), np.asarray(particles))
    out = np.zeros((len(particles), 7))
    lib().oracle_dtfe_fd(*prob._args(x, w, v), len(particles), off.ctypes.data, verts.ctypes.data,
                         float(h_pos), float(h_vel), float(h_w), out.ctypes.data)
    return out


def deposit_loss_grad(kind: int, pos, w, region, grid, rho_bar, a, want_grad: bool = True):
    """FP64 L = sum a*density of one region's NGP/CIC/TSC deposition and its
    gradient: (L, gx (n,3) or None, gw (n,) or None)."""
    pos = np.ascontiguousarray(pos, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    region = np.ascontiguousarray(region, np.float32)
    grid = np.ascontiguousarray(grid, np.int32)
    a = np.ascontiguousarray(a, np.float64)
    gx = np.zeros((len(pos), 3)) if want_grad else None
    gw = np.zeros(len(pos)) if want_grad else None
    L = lib().oracle_deposit_loss_grad(kind, pos.ctypes.data, w.ctypes.data, len(pos), region.ctypes.data,
                                       grid.ctypes.data, float(rho_bar), a.ctypes.data,
                                       None if gx is None else gx.ctypes.data,
                                       None if gw is None else gw.ctypes.data)
    return float(L), gx, gw
