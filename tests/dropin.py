"""ctypes access to the DTFE() test driver — test infrastructure shared by
test_dropin.py, test_reference_flow.py and test_gpu_dropin.py.

The same driver source (oracle/refharness/dropin_driver.cpp) is built twice
where the reference's headers exist: against this project's drop-in
(oracle/_ref/libdropin_driver.so, GPU) and against the reference's own
src/DTFE.cpp (oracle/_ref/libdtfe_refmain.so, CPU).  ``which`` picks one:
"dropin" or "reference"."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATHS = {"dropin": os.path.join(ROOT, "oracle", "_ref", "libdropin_driver.so"),
         "reference": os.path.join(ROOT, "oracle", "_ref", "libdtfe_refmain.so")}
PATH = PATHS["dropin"]
NCOMP = [1, 3, 9, 1, 5, 3, 1, 1, 3]
SLOTS = {"density": 0, "velocity": 1, "velocity_gradient": 2, "velocity_divergence": 3, "velocity_shear": 4,
         "velocity_vorticity": 5, "velocity_std": 6, "scalar": 7, "scalar_gradient": 8}
ESTIMATORS = {"DTFE": 0, "NGP": 1, "CIC": 2, "TSC": 3, "SPH": 4}
_libs = {}


class DriverOptions(C.Structure):
    """DriverOptions of dropin_driver.cpp: DTFE()'s planning options."""
    _fields_ = [("region_on", C.c_int32), ("region_mpc", C.c_int32), ("region", C.c_float * 6),
                ("partition_on", C.c_int32), ("partition", C.c_int32 * 3), ("part_no", C.c_int32),
                ("padding_mode", C.c_int32), ("padding_particles", C.c_float), ("padding", C.c_float * 6)]


def available(which: str = "dropin") -> bool:
    return os.path.exists(PATHS[which])


def lib(which: str = "dropin"):
    if which not in _libs:
        L = C.CDLL(PATHS[which])
        vp = C.c_void_p
        L.dropin_run.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int64, vp, C.c_int, vp, C.c_double, C.c_uint32,
                                 C.c_uint32, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, vp, vp,
                                 C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.dropin_run_points.argtypes = [vp, vp, vp, vp, C.c_int64, vp, C.c_int, vp, C.c_double, C.c_uint32,
                                        C.c_int64, vp, C.c_int, vp, C.POINTER(C.c_int64), C.c_uint32, vp, C.c_int,
                                        C.c_uint64, vp]
        L.dropin_run_cone.argtypes = [vp, vp, vp, vp, C.c_int64, vp, C.c_int, vp, C.c_double, C.c_uint32, vp, vp,
                                      C.c_int, vp, C.c_uint32, C.c_int, C.c_uint64, vp]
        L.dropin_run_ex.argtypes = [C.c_int, vp, vp, vp, vp, C.c_int64, vp, C.c_int, vp, C.c_double, C.c_uint32,
                                    C.c_uint32, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, vp, vp,
                                    C.POINTER(DriverOptions), C.c_int64, C.POINTER(C.c_int64), vp]
        L.dropin_error.restype = C.c_char_p
        _libs[which] = L
    return _libs[which]


def run(estimator, pos, w, vel, scal, grid, box=(0, 100, 0, 100, 0, 100), periodic=True, average_density=-1.0,
        u_fields=(), a_fields=(), method=3, n_points=8, seed=0, sph_neighbors=32, n_threads=4, which="dropin"):
    """Calls DTFE() through the driver: (u dict, a dict, average density used,
    particles left in the input vector).  Raises RuntimeError with DTFE()'s
    message when it throws."""
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    G = int(np.prod(grid))
    arrs = []

    def outs(fields):
        d = {f: np.full((G, NCOMP[SLOTS[f]]), np.nan, np.float32) for f in fields}
        arrs.append(d)
        ptrs = (C.c_void_p * 9)(*[d[f].ctypes.data if f in d else None for f in SLOTS])
        return d, ptrs, sum(1 << SLOTS[f] for f in fields)
    ud, up, um = outs(u_fields)
    ad, ap, am = outs(a_fields)
    g = np.ascontiguousarray(grid, np.int32)
    bx = np.ascontiguousarray(box, np.float32)
    keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (w, vel, scal)]
    avg = C.c_double()
    left = C.c_int64()
    L = lib(which)
    rc = L.dropin_run(ESTIMATORS[estimator], pos.ctypes.data, *[a.ctypes.data if a is not None else None
                                                                for a in keep], n, bx.ctypes.data, int(periodic),
                      g.ctypes.data, float(average_density), um, am, method, n_points, seed, sph_neighbors,
                      n_threads, up, ap, C.byref(avg), C.byref(left))
    if rc:
        raise RuntimeError(L.dropin_error().decode())
    return ud, ad, avg.value, left.value


def run_ex(estimator, pos, w, vel, scal, grid, box=(0, 100, 0, 100, 0, 100), periodic=True, average_density=-1.0,
           u_fields=(), a_fields=(), method=3, n_points=8, seed=0, sph_neighbors=32, n_threads=4, which="dropin",
           region=None, region_mpc=False, partition=None, part_no=-1, padding=None, padding_mode=1,
           padding_particles=5.0):
    """DTFE() with its planning options (--region in box fractions, or
    absolute with region_mpc; --partition with --partNo; --padding
    l1..l6 with padding_mode 1 or --paddingMpc with 2): (u dict, a dict,
    userOptions.region after the call), each field holding the rows of the
    grid the results cover."""
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    G = int(np.prod(grid))
    x = DriverOptions()
    if region is not None:
        x.region_on, x.region_mpc = 1, int(region_mpc)
        x.region[:] = [float(r) for r in np.asarray(region, np.float32)]
    if partition is not None:
        x.partition_on = 1
        x.partition[:] = [int(q) for q in partition]
        x.part_no = int(part_no)
    x.padding_particles = float(padding_particles)
    if padding is not None:
        x.padding_mode = int(padding_mode)
        x.padding[:] = [float(q) for q in np.asarray(padding, np.float32)]
    ud = {f: np.full((G, NCOMP[SLOTS[f]]), np.nan, np.float32) for f in u_fields}
    ad = {f: np.full((G, NCOMP[SLOTS[f]]), np.nan, np.float32) for f in a_fields}
    up = (C.c_void_p * 9)(*[ud[f].ctypes.data if f in ud else None for f in SLOTS])
    ap = (C.c_void_p * 9)(*[ad[f].ctypes.data if f in ad else None for f in SLOTS])
    um = sum(1 << SLOTS[f] for f in u_fields)
    am = sum(1 << SLOTS[f] for f in a_fields)
    g = np.ascontiguousarray(grid, np.int32)
    bx = np.ascontiguousarray(box, np.float32)
    keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (w, vel, scal)]
    rows = C.c_int64()
    reg = np.zeros(6, np.float32)
    L = lib(which)
    rc = L.dropin_run_ex(ESTIMATORS[estimator], pos.ctypes.data, *[a.ctypes.data if a is not None else None
                                                                   for a in keep], n, bx.ctypes.data, int(periodic),
                         g.ctypes.data, float(average_density), um, am, method, n_points, seed, sph_neighbors,
                         n_threads, up, ap, C.byref(x), G, C.byref(rows), reg.ctypes.data)
    if rc:
        raise RuntimeError(L.dropin_error().decode())
    m = rows.value
    return {f: a[:m] for f, a in ud.items()}, {f: a[:m] for f, a in ad.items()}, reg


def run_points(pos, w, vel, scal, grid, samples, box=(0, 100, 0, 100, 0, 100), periodic=True,
               average_density=-1.0, u_fields=("density",), n_threads=4, a_fields=(), delta=None, n_points=-1,
               seed=0):
    """DTFE() with user sampling points: dict field -> rows of the samples
    inside the box, in order (with a_fields: (u dict, a dict))."""
    pos = np.ascontiguousarray(pos, np.float32)
    samples = np.ascontiguousarray(samples, np.float32)
    m = len(samples)
    d = {f: np.full((m, NCOMP[SLOTS[f]]), np.nan, np.float32) for f in u_fields}
    da = {f: np.full((m, NCOMP[SLOTS[f]]), np.nan, np.float32) for f in a_fields}
    ptrs = (C.c_void_p * 9)(*[d[f].ctypes.data if f in d else None for f in SLOTS])
    aptrs = (C.c_void_p * 9)(*[da[f].ctypes.data if f in da else None for f in SLOTS])
    mask = sum(1 << SLOTS[f] for f in u_fields)
    amask = sum(1 << SLOTS[f] for f in a_fields)
    g = np.ascontiguousarray(grid, np.int32)
    bx = np.ascontiguousarray(box, np.float32)
    dl = np.ascontiguousarray(delta, np.float32) if delta is not None else None
    keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (w, vel, scal)]
    kept = C.c_int64()
    rc = lib().dropin_run_points(pos.ctypes.data, *[a.ctypes.data if a is not None else None for a in keep],
                                 len(pos), bx.ctypes.data, int(periodic), g.ctypes.data, float(average_density),
                                 mask, m, samples.ctypes.data, n_threads, ptrs, C.byref(kept), amask,
                                 dl.ctypes.data if dl is not None else None, n_points, seed, aptrs)
    if rc:
        raise RuntimeError(lib().dropin_error().decode())
    u = {f: a[:kept.value] for f, a in d.items()}
    if a_fields:
        return u, {f: a[:kept.value] for f, a in da.items()}
    return u


def run_cone(pos, w, vel, scal, grid, cone, origin, box=(0, 100, 0, 100, 0, 100), periodic=True,
             average_density=-1.0, u_fields=("density",), n_threads=4, a_fields=(), n_points=-1, seed=0):
    """DTFE() on a redshift-cone grid: dict field -> grid[0] grid[1] grid[2]
    rows, r slowest and psi fastest (with a_fields: (u dict, a dict))."""
    pos = np.ascontiguousarray(pos, np.float32)
    G = int(np.prod(grid))
    d = {f: np.full((G, NCOMP[SLOTS[f]]), np.nan, np.float32) for f in u_fields}
    da = {f: np.full((G, NCOMP[SLOTS[f]]), np.nan, np.float32) for f in a_fields}
    ptrs = (C.c_void_p * 9)(*[d[f].ctypes.data if f in d else None for f in SLOTS])
    aptrs = (C.c_void_p * 9)(*[da[f].ctypes.data if f in da else None for f in SLOTS])
    mask = sum(1 << SLOTS[f] for f in u_fields)
    amask = sum(1 << SLOTS[f] for f in a_fields)
    g = np.ascontiguousarray(grid, np.int32)
    bx = np.ascontiguousarray(box, np.float32)
    c = np.ascontiguousarray(cone, np.float32)
    o = np.ascontiguousarray(origin, np.float32)
    keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (w, vel, scal)]
    rc = lib().dropin_run_cone(pos.ctypes.data, *[a.ctypes.data if a is not None else None for a in keep],
                               len(pos), bx.ctypes.data, int(periodic), g.ctypes.data, float(average_density),
                               mask, c.ctypes.data, o.ctypes.data, n_threads, ptrs, amask, n_points, seed, aptrs)
    if rc:
        raise RuntimeError(lib().dropin_error().decode())
    if a_fields:
        return d, da
    return d
