"""Python access to the reference-code harness (oracle/_ref/libdtfe_ref.so) —
TEST INFRASTRUCTURE ONLY.

The harness runs the reference's own interpolation sources
(src/CGAL_triangulation/triangulation.cpp, compiled from the reference tree
by oracle/Makefile) on a flat tessellation through a CGAL-API facade.  It is
built only where the reference tree exists; ``available()`` says whether it
was built.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libdtfe_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.ref_interpolate.argtypes = [C.c_int64, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp, C.c_int, C.c_int,
                                      C.c_uint64, C.c_double, vp, vp, vp, vp, vp, vp, vp, vp]
        L.ref_interpolate.restype = C.c_int
        L.ref_interpolate_timed.argtypes = L.ref_interpolate.argtypes + [C.c_uint32, C.POINTER(C.c_double)]
        L.ref_interpolate_timed.restype = C.c_int
        _lib = L
    return _lib


def run(plan, box: int = 0, which: int = 0, n_points: int = 1, seed: int = 0, dens_override=None):
    """Reference fields of one sub-box tile (tile-local grid, x slowest).

    Returns dict with 'vertex_density' (local vertices) and the fields."""
    b = plan.boxes[box]
    v0, nv, t0, nt = b.vert_offset, b.n_verts, b.tet_offset, b.n_tets
    xyz = np.ascontiguousarray(plan.xyz[v0:v0 + nv])
    w = np.ascontiguousarray(plan.weight[v0:v0 + nv])
    vel = None if plan.velocity is None else np.ascontiguousarray(plan.velocity[v0:v0 + nv])
    sc = None if plan.scalar is None else np.ascontiguousarray(plan.scalar[v0:v0 + nv, 0])
    tv = np.ascontiguousarray(plan.tet_v[t0:t0 + nt] - v0, dtype=np.int32)
    tn = plan.tet_n[t0:t0 + nt]
    tn = np.ascontiguousarray(np.where(tn >= 0, tn - t0, -1), dtype=np.int32)
    dims = np.array([b.tile_dims[0], b.tile_dims[1], b.tile_dims[2]], np.int32)
    region = np.ascontiguousarray(plan.region_array()[box])
    G = int(np.prod(dims))
    out = {"vertex_density": np.zeros(nv, np.float32), "density": np.zeros(G, np.float32),
           "velocity": np.zeros((G, 3), np.float32), "velocity_gradient": np.zeros((G, 9), np.float32),
           "scalar": np.zeros(G, np.float32), "scalar_gradient": np.zeros((G, 3), np.float32),
           "velocity_std": np.zeros(G, np.float32)}
    dov = None if dens_override is None else np.ascontiguousarray(dens_override[v0:v0 + nv], np.float32)
    p = lambda a: None if a is None else a.ctypes.data
    rc = lib().ref_interpolate(nv, p(xyz), p(w), p(vel), p(sc), nt, p(tv), p(tn), p(region), p(dims), which,
                               n_points, seed, plan.rho_bar, p(dov), p(out["vertex_density"]),
                               p(out["density"]), p(out["velocity"]), p(out["velocity_gradient"]),
                               p(out["scalar"]) if sc is not None else None,
                               p(out["scalar_gradient"]) if sc is not None else None,
                               p(out["velocity_std"]) if which == 2 else None)
    if rc:
        raise RuntimeError(f"ref_interpolate failed ({rc})")
    return out


def run_points(plan, pts, region, dens, box: int = 0, timing: bool = False):
    """The reference's interpolateUserSampling on sub-box `box`'s
    tessellation with vertex densities `dens`: density, velocity, gradient,
    scalar, scalar gradient of the points inside `region`, in order.  With
    `timing`, (that dict, seconds of the interpolateUserSampling call)."""
    xyz, w, vel, tv, tn, dims, _ = _box_args(plan, box)
    b = plan.boxes[box]
    v0, nv = b.vert_offset, b.n_verts
    sc = None if plan.scalar is None else np.ascontiguousarray(plan.scalar[v0:v0 + nv, 0])
    d = np.ascontiguousarray(dens[v0:v0 + nv], np.float32)
    pts = np.ascontiguousarray(pts, np.float32)
    n = len(pts)
    out = {"density": np.zeros(n, np.float32), "velocity": np.zeros((n, 3), np.float32),
           "velocity_gradient": np.zeros((n, 9), np.float32), "scalar": np.zeros(n, np.float32),
           "scalar_gradient": np.zeros((n, 3), np.float32)}
    reg = np.ascontiguousarray(region, np.float32)
    L = lib()
    vp = C.c_void_p
    L.ref_interpolate_points.argtypes = [C.c_int64, vp, vp, vp, vp, C.c_int64, vp, vp, vp, C.c_int64, vp, vp,
                                         vp, vp, vp, vp, vp, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    p = lambda a: None if a is None else a.ctypes.data
    m = C.c_int64(0)
    secs = C.c_double(0.0)
    rc = L.ref_interpolate_points(len(xyz), p(xyz), p(w), p(vel), p(sc), len(tv), p(tv), p(tn), p(reg), n,
                                  p(pts), p(d), p(out["density"]), p(out["velocity"]), p(out["velocity_gradient"]),
                                  p(out["scalar"]) if sc is not None else None,
                                  p(out["scalar_gradient"]) if sc is not None else None, C.byref(m), C.byref(secs))
    if rc:
        raise RuntimeError(f"ref_interpolate_points failed ({rc})")
    res = {k: a[:m.value] for k, a in out.items()}
    return (res, secs.value) if timing else res


def run_cone(plan, cone, origin, dims, dens, box: int = 0, timing: bool = False):
    """The reference's interpolateRedshiftCone on sub-box `box`'s
    tessellation with vertex densities `dens`: density, velocity, gradient,
    scalar, scalar gradient of the dims[0] * dims[1] * dims[2] cone samples.
    With `timing`, (that dict, seconds of the interpolateRedshiftCone call)."""
    xyz, w, vel, tv, tn, _, _ = _box_args(plan, box)
    b = plan.boxes[box]
    v0, nv = b.vert_offset, b.n_verts
    sc = None if plan.scalar is None else np.ascontiguousarray(plan.scalar[v0:v0 + nv, 0])
    d = np.ascontiguousarray(dens[v0:v0 + nv], np.float32)
    n = int(np.prod(dims))
    out = {"density": np.zeros(n, np.float32), "velocity": np.zeros((n, 3), np.float32),
           "velocity_gradient": np.zeros((n, 9), np.float32), "scalar": np.zeros(n, np.float32),
           "scalar_gradient": np.zeros((n, 3), np.float32)}
    c = np.ascontiguousarray(cone, np.float32)
    o = np.ascontiguousarray(origin, np.float32)
    dd = np.ascontiguousarray(dims, np.int32)
    L = lib()
    vp = C.c_void_p
    L.ref_interpolate_cone.argtypes = [C.c_int64, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                       vp, vp, C.POINTER(C.c_double)]
    p = lambda a: None if a is None else a.ctypes.data
    secs = C.c_double(0.0)
    rc = L.ref_interpolate_cone(len(xyz), p(xyz), p(w), p(vel), p(sc), len(tv), p(tv), p(tn), p(c), p(o), p(dd),
                                p(d), p(out["density"]), p(out["velocity"]), p(out["velocity_gradient"]),
                                p(out["scalar"]) if sc is not None else None,
                                p(out["scalar_gradient"]) if sc is not None else None, C.byref(secs))
    if rc:
        raise RuntimeError(f"ref_interpolate_cone failed ({rc})")
    return (out, secs.value) if timing else out


def run_average(plan, dens, n_samples: int, seed: int, pts=None, delta=None, region=None, cone=None, origin=None,
                dims=None, box: int = 0):
    """The reference's Monte-Carlo averages (its own mt19937 stream): at user
    points (interpolateUserSampling_averaged_2; pts, delta, region) or on a
    redshift cone (interpolateRedshiftCone_averaged_2; cone, origin, dims).
    Dict of density, velocity, gradient, scalar, scalar gradient rows."""
    xyz, w, vel, tv, tn, _, _ = _box_args(plan, box)
    b = plan.boxes[box]
    v0, nv = b.vert_offset, b.n_verts
    sc = None if plan.scalar is None else np.ascontiguousarray(plan.scalar[v0:v0 + nv, 0])
    d = np.ascontiguousarray(dens[v0:v0 + nv], np.float32)
    which = 0 if pts is not None else 1
    n = len(pts) if which == 0 else int(np.prod(dims))
    out = {"density": np.zeros(n, np.float32), "velocity": np.zeros((n, 3), np.float32),
           "velocity_gradient": np.zeros((n, 9), np.float32), "scalar": np.zeros(n, np.float32),
           "scalar_gradient": np.zeros((n, 3), np.float32)}
    f32 = lambda a, k: np.ascontiguousarray(a if a is not None else np.zeros(k), np.float32)
    P = f32(pts, 3)
    D = f32(delta, 3)
    R = f32(region, 6)
    Cn = f32(cone, 6)
    O = f32(origin, 3)
    Dm = np.ascontiguousarray(dims if dims is not None else (1, 1, 1), np.int32)
    L = lib()
    vp = C.c_void_p
    L.ref_average_samples.argtypes = [C.c_int, C.c_int64, vp, vp, vp, vp, C.c_int64, vp, vp, vp, C.c_int64, vp, vp,
                                      vp, vp, vp, C.c_int, C.c_uint64, vp, vp, vp, vp, vp, vp,
                                      C.POINTER(C.c_int64)]
    p = lambda a: None if a is None else a.ctypes.data
    m = C.c_int64(0)
    rc = L.ref_average_samples(which, len(xyz), p(xyz), p(w), p(vel), p(sc), len(tv), p(tv), p(tn), p(R),
                               n if which == 0 else 0, p(P), p(D), p(Cn), p(O), p(Dm), n_samples, seed, p(d),
                               p(out["density"]), p(out["velocity"]), p(out["velocity_gradient"]),
                               p(out["scalar"]) if sc is not None else None,
                               p(out["scalar_gradient"]) if sc is not None else None, C.byref(m))
    if rc:
        raise RuntimeError(f"ref_average_samples failed ({rc})")
    return {k: a[:m.value] for k, a in out.items()}


def _box_args(plan, box):
    b = plan.boxes[box]
    v0, nv, t0, nt = b.vert_offset, b.n_verts, b.tet_offset, b.n_tets
    xyz = np.ascontiguousarray(plan.xyz[v0:v0 + nv])
    w = np.ascontiguousarray(plan.weight[v0:v0 + nv])
    vel = None if plan.velocity is None else np.ascontiguousarray(plan.velocity[v0:v0 + nv])
    tv = np.ascontiguousarray(plan.tet_v[t0:t0 + nt] - v0, dtype=np.int32)
    tn = plan.tet_n[t0:t0 + nt]
    tn = np.ascontiguousarray(np.where(tn >= 0, tn - t0, -1), dtype=np.int32)
    dims = np.array([b.tile_dims[0], b.tile_dims[1], b.tile_dims[2]], np.int32)
    region = np.ascontiguousarray(plan.region_array()[box])
    return xyz, w, vel, tv, tn, dims, region


MAIN_LIB = os.path.join(_HERE, "_ref", "libdtfe_refmain.so")
_main = None


def main_lib() -> C.CDLL:
    """The reference's own src/DTFE.cpp in the harness (libdtfe_refmain.so)."""
    global _main
    if _main is None:
        L = C.CDLL(MAIN_LIB)
        vp = C.c_void_p
        L.ref_derived_timed.argtypes = [C.c_int64, vp, vp, vp, vp, C.POINTER(C.c_double)]
        L.ref_derived_timed.restype = C.c_int
        _main = L
    return _main


def derived(grad: np.ndarray):
    """The reference's computeDivergenceShearVorticity (src/DTFE.cpp:436-475)
    on a gradient grid (G, 9): (divergence, shear, vorticity, seconds of the
    call alone)."""
    g = np.ascontiguousarray(grad, np.float32).reshape(-1, 9)
    G = len(g)
    div = np.empty(G, np.float32)
    sh = np.empty((G, 5), np.float32)
    vo = np.empty((G, 3), np.float32)
    sec = C.c_double(0.0)
    if main_lib().ref_derived_timed(G, g.ctypes.data, div.ctypes.data, sh.ctypes.data, vo.ctypes.data,
                                    C.byref(sec)):
        raise RuntimeError("ref_derived_timed failed")
    return div, sh, vo, sec.value


def time_boxes(plan, threads: int, which: int = 0, n_points: int = 1, with_derived: bool = False):
    """Times the reference's own per-thread work of DTFE_parallel
    (src/DTFE.cpp:331-356): vertexDensity + the interpolation ``which``
    (0 interpolateGrid, 1/2/3 the averaging methods with ``n_points``) of
    density, velocity and velocity gradient on every sub-box, the sub-boxes
    spread over ``threads`` host threads as the reference's OpenMP team would.
    with_derived adds, after the threads, DTFE()'s one serial
    computeDivergenceShearVorticity on the main grid's gradient
    (src/DTFE.cpp:248-249, the reference's own code from
    libdtfe_refmain.so).  Returns (seconds: the slowest thread plus the
    derived pass, per-box seconds); only the reference's calls are timed, not
    loading the tessellation."""
    from concurrent.futures import ThreadPoolExecutor
    L = lib()
    G1, G2 = plan.grid[1], plan.grid[2]
    main_grad = np.zeros((int(np.prod(plan.grid)), 9), np.float32) if with_derived else None

    def one(box):
        xyz, w, vel, tv, tn, dims, region = _box_args(plan, box)
        G = int(np.prod(dims))
        dens = np.zeros(G, np.float32)
        velo = np.zeros((G, 3), np.float32)
        grad = np.zeros((G, 9), np.float32)
        sec = C.c_double(0.0)
        p = lambda a: None if a is None else a.ctypes.data
        rc = L.ref_interpolate_timed(len(xyz), p(xyz), p(w), p(vel), None, len(tv), p(tv), p(tn), p(region),
                                     p(dims), which, n_points, 0, plan.rho_bar, None, None, p(dens), p(velo),
                                     p(grad),
                                     None, None, None, 7, C.byref(sec))
        if rc:
            raise RuntimeError(f"ref_interpolate_timed failed ({rc})")
        if main_grad is not None:
            # copySubgridResultsToMain (src/subpartition.h:399-432), untimed
            b = plan.boxes[box]
            o = [b.tile_origin[a] for a in range(3)]
            d = [int(x) for x in dims]
            view = main_grad.reshape(plan.grid[0], G1, G2, 9)
            view[o[0]:o[0] + d[0], o[1]:o[1] + d[1], o[2]:o[2] + d[2]] = grad.reshape(d[0], d[1], d[2], 9)
        return sec.value
    K = plan.n_boxes
    with ThreadPoolExecutor(max_workers=max(1, min(threads, K))) as ex:
        per_box = list(ex.map(one, range(K)))
    # the reference gives each OpenMP thread one sub-box; with more boxes than
    # threads, boxes are dealt round-robin
    loads = [0.0] * max(1, min(threads, K))
    for k, t in enumerate(per_box):
        loads[k % len(loads)] += t
    t_derived = derived(main_grad)[3] if main_grad is not None else 0.0
    return max(loads) + t_derived, per_box


def _time_sample(fn, n_items: int, threads: int):
    """Runs fn(k) for the first min(threads, n_items) items concurrently, one
    host thread each (the reference's OpenMP team gives each thread one
    sub-box); returns (wall seconds, items run)."""
    from concurrent.futures import ThreadPoolExecutor
    m = max(1, min(threads, n_items))
    with ThreadPoolExecutor(max_workers=m) as ex:
        t0 = time.perf_counter()
        list(ex.map(fn, range(m)))
        return time.perf_counter() - t0, m


def time_deposit_boxes(dplan, threads: int, velocity: bool = True):
    """Times the reference's own NGP/CIC/TSC_interpolation_regular_grid
    (src/CIC_interpolation.cc:67-273, src/TSC_interpolation.cc:67-254) on a
    sample of the deposit plan's sub-boxes, one per host thread, each with its
    region's particles and grid tile.  Returns (grid cells of the sampled
    tiles per second of wall time, sampled boxes, particles in them); the
    wall time includes the harness copying the arrays into the reference's
    Particle_data records."""
    L = lib()
    vp = C.c_void_p
    L.ref_deposit.argtypes = [C.c_int, vp, vp, vp, C.c_int64, vp, vp, C.c_double, vp, vp]
    boxes = list(dplan.boxes)
    cells = [int(b.tile_dims[0]) * int(b.tile_dims[1]) * int(b.tile_dims[2]) for b in boxes]

    def one(k):
        b = boxes[k]
        o, n = int(b.particle_offset), int(b.n_particles)
        pos = np.ascontiguousarray(dplan.pos[o:o + n])
        w = np.ascontiguousarray(dplan.weight[o:o + n])
        vel = np.ascontiguousarray(dplan.velocity[o:o + n]) if velocity and dplan.velocity is not None else None
        region = np.array([b.region[a] for a in range(6)], np.float32)
        dims = np.array([b.tile_dims[a] for a in range(3)], np.int32)
        dens = np.zeros(cells[k], np.float32)
        velo = np.zeros((cells[k], 3), np.float32) if vel is not None else None
        rc = L.ref_deposit(int(dplan.kind), pos.ctypes.data, w.ctypes.data, None if vel is None else vel.ctypes.data,
                           n, region.ctypes.data, dims.ctypes.data, float(dplan.rho_bar), dens.ctypes.data,
                           None if velo is None else velo.ctypes.data)
        if rc:
            raise RuntimeError(f"ref_deposit failed ({rc})")
    wall, m = _time_sample(one, len(boxes), threads)
    return sum(cells[:m]) / wall, m, int(sum(int(b.n_particles) for b in boxes[:m]))


def time_sph_boxes(plan, threads: int, n_neighbors: int = 32):
    """Times the reference's own SPH_interpolation (src/SPH_interpolation.cc:
    47-146 and 252-474, with its kd-tree) of density and velocity on a sample
    of the plan's padded sub-boxes, one per host thread, each on its grid
    tile.  Returns (grid cells of the sampled tiles per second of wall time,
    sampled boxes)."""
    L = lib()
    vp = C.c_void_p
    L.ref_sph.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int64, vp, vp, C.c_double, C.c_int, vp, vp, vp]
    K = plan.n_boxes
    cells = []
    for k in range(K):
        b = plan.boxes[k]
        cells.append(int(b.tile_dims[0]) * int(b.tile_dims[1]) * int(b.tile_dims[2]))

    def one(k):
        xyz, w, vel, _tv, _tn, dims, region = _box_args(plan, k)
        dens = np.zeros(cells[k], np.float32)
        velo = np.zeros((cells[k], 3), np.float32)
        rc = L.ref_sph(xyz.ctypes.data, w.ctypes.data, None if vel is None else vel.ctypes.data, None, 0, len(xyz),
                       region.ctypes.data, dims.ctypes.data, float(plan.rho_bar), n_neighbors, dens.ctypes.data,
                       None if vel is None else velo.ctypes.data, None)
        if rc:
            raise RuntimeError(f"ref_sph failed ({rc})")
    wall, m = _time_sample(one, K, threads)
    return sum(cells[:m]) / wall, m


def write_binary(path: str, data, ncomp: int) -> None:
    """The reference's writeBinaryFile of rows x ncomp floats (a std::vector
    of Real for 1, of Pvector<Real, ncomp> for 3, 5, 9) into `path`."""
    a = np.ascontiguousarray(data, np.float32)
    L = lib()
    L.ref_write_binary.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_int]
    rc = L.ref_write_binary(path.encode(), a.ctypes.data, a.size // ncomp, ncomp)
    if rc:
        raise RuntimeError(f"ref_write_binary failed ({rc})")


_SLOTS = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear",
          "velocity_vorticity", "velocity_std", "scalar", "scalar_gradient"]


def write_output(base: str, n: int, u: dict, a: dict) -> None:
    """The reference's writeOutputData (binary output) of n rows per field:
    u / a map field names to float arrays (uQuantities / aQuantities)."""
    keep = []

    def table(d):
        ptrs = (C.c_void_p * 9)()
        mask = 0
        for s, f in enumerate(_SLOTS):
            if f in d:
                arr = np.ascontiguousarray(d[f], np.float32)
                keep.append(arr)
                ptrs[s] = arr.ctypes.data
                mask |= 1 << s
        return ptrs, mask

    up, um = table(u)
    ap, am = table(a)
    L = lib()
    L.ref_write_output.argtypes = [C.c_char_p, C.c_int64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
    rc = L.ref_write_output(base.encode(), n, um, am, C.cast(up, C.c_void_p), C.cast(ap, C.c_void_p))
    if rc:
        raise RuntimeError(f"ref_write_output failed ({rc})")
