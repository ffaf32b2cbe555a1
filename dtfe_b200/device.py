"""Python handle over the C ABI of include/dtfe_gpu.h (libdtfe_gpu.so)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def _mask(fields) -> int:
    m = 0
    for f in fields:
        m |= 1 << N.FIELD_SLOTS[f]
    return m


class DeviceDTFE:
    """One device handle: uploaded multi-tessellation, sub-boxes, vertex data."""

    def __init__(self, device: int = 0, n_scalars: int = 0, max_walk_steps: int = 0):
        self.lib = N.gpu()
        self.h = C.c_void_p()
        cfg = N.Config(device, n_scalars, max_walk_steps, 0)
        N.check(self.lib.dtfe_gpu_create(C.byref(cfg), C.byref(self.h)))
        self.n_scalars = n_scalars
        self.grid = None
        self.last_status = None

    def close(self) -> None:
        if self.h:
            self.lib.dtfe_gpu_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self) -> int:
        return int(self.lib.dtfe_gpu_stream(self.h) or 0)

    def synchronize(self) -> None:
        N.check(self.lib.dtfe_gpu_synchronize(self.h))

    def upload(self, plan, neighbours: bool = True) -> None:
        """Plain upload; neighbours=False sends tet_v alone and the device
        derives the neighbours."""
        N.check(self.lib.dtfe_gpu_upload(
            self.h, N.ptr(plan.tet_v), N.ptr(plan.tet_n) if neighbours else None, plan.n_tets, N.ptr(plan.xyz),
            N.ptr(plan.weight), N.ptr(plan.velocity), N.ptr(plan.scalar), plan.n_verts))

    def upload_packed(self, plan, packed: np.ndarray) -> None:
        """Upload with the tetrahedra in packed form (plan.pack_tets)."""
        N.check(self.lib.dtfe_gpu_upload_packed(
            self.h, packed.ctypes.data, packed.nbytes, N.ptr(plan.xyz), N.ptr(plan.weight), N.ptr(plan.velocity),
            N.ptr(plan.scalar), plan.n_verts))

    def upload_packed_particles(self, plan, packed: np.ndarray, particles: dict) -> None:
        """Packed tetrahedra plus the input particles once
        (dtfe_gpu_upload_packed_particles): ``particles`` holds ``pos``,
        ``weight``, ``velocity`` (or None), ``scalar`` (or None) of the n input
        particles, ``codes`` (plan.vertex_codes) and ``box_length`` (3 floats)."""
        L = np.ascontiguousarray(particles["box_length"], np.float32)
        codes = particles["codes"]
        N.check(self.lib.dtfe_gpu_upload_packed_particles(
            self.h, packed.ctypes.data, packed.nbytes, N.ptr(particles["pos"]), N.ptr(particles["weight"]),
            N.ptr(particles.get("velocity")), N.ptr(particles.get("scalar")), len(particles["pos"]),
            N.ptr(codes), len(codes), L.ctypes.data))

    def chain_uploads(self, after: "DeviceDTFE | None") -> None:
        """Uploads on this handle wait for ``after``'s latest transfers
        (dtfe_gpu_chain_uploads); None removes the link."""
        N.check(self.lib.dtfe_gpu_chain_uploads(self.h, after.h if after is not None else None))

    def set_subboxes(self, plan) -> None:
        grid = np.asarray(plan.grid, np.int32)
        N.check(self.lib.dtfe_gpu_set_subboxes(
            self.h, plan.n_boxes, C.addressof(plan.boxes), N.ptr(plan.xs), len(plan.xs),
            N.ptr(plan.ys), len(plan.ys), N.ptr(plan.zs), len(plan.zs), grid.ctypes.data))
        self.grid = tuple(plan.grid)
        if getattr(plan, "regions", None) is not None:
            self.set_regions(plan.regions)

    def set_regions(self, regions: np.ndarray) -> None:
        """Tile regions (K, 6) for averaging method 1 (dtfe_gpu_set_regions)."""
        r = np.ascontiguousarray(regions, np.float32).reshape(-1, 6)
        N.check(self.lib.dtfe_gpu_set_regions(self.h, len(r), r.ctypes.data))

    def load(self, plan) -> None:
        self.upload(plan)
        self.set_subboxes(plan)

    def vertex_density(self, rho_bar: float) -> None:
        N.check(self.lib.dtfe_gpu_vertex_density(self.h, float(rho_bar)))

    def download_vertex_density(self, n_verts: int) -> np.ndarray:
        out = np.empty(n_verts, np.float32)
        N.check(self.lib.dtfe_gpu_download_vertex_density(self.h, out.ctypes.data))
        return out

    def _opts(self, fields, method, n_samples, seed, fix, fix_outside=False):
        flags = (N.FLAG_FIX_VALUE_INTERP if fix else 0) | (N.FLAG_FIX_OUTSIDE_RASTER if fix_outside else 0)
        return N.InterpOpts(method, n_samples, seed, _mask(fields), flags)

    def interpolate(self, fields, method: int = 0, n_samples: int = 1, seed: int = 0, fix: bool = False,
                    out: dict | None = None, fix_outside: bool = False) -> dict:
        """Host outputs: dict field -> float32 array (G, ncomp) or (G,)."""
        G = int(np.prod(self.grid))
        outs = [None] * N.NUM_FIELDS
        res = {}
        for f in fields:
            s = N.FIELD_SLOTS[f]
            nc = N.field_components(s, self.n_scalars)
            a = out[f] if out and f in out else np.empty((G, nc) if nc > 1 else G, np.float32)
            res[f] = a
            outs[s] = N.ptr(a)
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        st = N.Status()
        o = self._opts(fields, method, n_samples, seed, fix, fix_outside)
        rc = self.lib.dtfe_gpu_interpolate(self.h, C.byref(o), optr, C.byref(st))
        self.last_status = st.as_dict()  # also when the call reports a walk failure
        N.check(rc)
        return res

    def interpolate_async(self, fields, out: dict, method: int = 0, n_samples: int = 1, seed: int = 0,
                          fix: bool = False) -> None:
        """Queues the interpolation and the copies into the host arrays of
        ``out`` (field -> float32 array, best pinned); valid after
        synchronize()."""
        outs = [None] * N.NUM_FIELDS
        for f in fields:
            outs[N.FIELD_SLOTS[f]] = N.ptr(out[f])
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        o = self._opts(fields, method, n_samples, seed, fix)
        N.check(self.lib.dtfe_gpu_interpolate_async(self.h, C.byref(o), optr))

    def interpolate_dev(self, fields, outs_dev: dict, method: int = 0, n_samples: int = 1, seed: int = 0,
                        fix: bool = False) -> dict:
        """Device outputs: dict field -> device pointer or tensor."""
        outs = [None] * N.NUM_FIELDS
        for f in fields:
            outs[N.FIELD_SLOTS[f]] = N.ptr(outs_dev[f]) if not isinstance(outs_dev[f], int) else outs_dev[f]
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        st = N.Status()
        o = self._opts(fields, method, n_samples, seed, fix)
        N.check(self.lib.dtfe_gpu_interpolate_dev(self.h, C.byref(o), optr, C.byref(st)))
        self.last_status = st.as_dict()
        return self.last_status

    def interpolate_points(self, fields, pts: np.ndarray, region, fix: bool = False) -> dict:
        """Fields at user sampling points (dtfe_gpu_interpolate_points): dict
        field -> float32 array of the points inside `region`, in order."""
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        n = len(pts)
        reg = np.ascontiguousarray(region, np.float32)
        outs = [None] * N.NUM_FIELDS
        res = {}
        for f in fields:
            s = N.FIELD_SLOTS[f]
            nc = N.field_components(s, self.n_scalars)
            a = np.zeros((n, nc) if nc > 1 else n, np.float32)
            res[f] = a
            outs[s] = N.ptr(a)
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        o = self._opts(fields, N.METHOD_CENTRE, 1, 0, fix)
        m = C.c_int64(0)
        N.check(self.lib.dtfe_gpu_interpolate_points(self.h, n, pts.ctypes.data, reg.ctypes.data, C.byref(o), optr,
                                                     C.byref(m)))
        return {f: a[:m.value] for f, a in res.items()}

    def average_points(self, fields, pts: np.ndarray, delta: np.ndarray, region, n_samples: int, seed: int = 0,
                       fix: bool = False) -> dict:
        """Monte-Carlo volume averages at user sampling points
        (dtfe_gpu_average_points): dict field -> float32 array of the points
        inside `region`, in order."""
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        delta = np.ascontiguousarray(delta, np.float32).reshape(-1, 3)
        if delta.shape != pts.shape:
            raise ValueError("one delta (3 floats) per point")
        n = len(pts)
        reg = np.ascontiguousarray(region, np.float32)
        outs = [None] * N.NUM_FIELDS
        res = {}
        for f in fields:
            s = N.FIELD_SLOTS[f]
            nc = N.field_components(s, self.n_scalars)
            a = np.zeros((n, nc) if nc > 1 else n, np.float32)
            res[f] = a
            outs[s] = N.ptr(a)
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        o = self._opts(fields, N.METHOD_MONTE_CARLO, n_samples, seed, fix)
        m = C.c_int64(0)
        N.check(self.lib.dtfe_gpu_average_points(self.h, n, pts.ctypes.data, delta.ctypes.data, reg.ctypes.data,
                                                 C.byref(o), optr, C.byref(m)))
        return {f: a[:m.value] for f, a in res.items()}

    def interpolate_cone(self, fields, cone, origin, dims, fix: bool = False, fix_outside: bool = False,
                         n_samples: int = 0, seed: int = 0) -> dict:
        """Fields on a redshift-cone grid (dtfe_gpu_interpolate_cone): dict
        field -> float32 array of dims[0] * dims[1] * dims[2] rows, r slowest
        and psi fastest; n_samples > 0 gives the Monte-Carlo bin averages."""
        d = np.ascontiguousarray(dims, np.int32)
        c = np.ascontiguousarray(cone, np.float32)
        org = np.ascontiguousarray(origin, np.float32)
        n = int(np.prod(d.astype(np.int64)))
        outs = [None] * N.NUM_FIELDS
        res = {}
        for f in fields:
            s = N.FIELD_SLOTS[f]
            nc = N.field_components(s, self.n_scalars)
            a = np.zeros((n, nc) if nc > 1 else n, np.float32)
            res[f] = a
            outs[s] = N.ptr(a)
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        if n_samples > 0:
            o = self._opts(fields, N.METHOD_MONTE_CARLO, n_samples, seed, fix)
        else:
            o = self._opts(fields, N.METHOD_CENTRE, 1, 0, fix, fix_outside)
        N.check(self.lib.dtfe_gpu_interpolate_cone(self.h, c.ctypes.data, org.ctypes.data, d.ctypes.data, C.byref(o),
                                                   optr))
        return res

    def interpolate_cone_dev(self, fields, cone, origin, dims, outs_dev: dict, fix: bool = False,
                             fix_outside: bool = False) -> None:
        """Same as interpolate_cone into device outputs (torch tensors or
        device pointers) of dims[0] * dims[1] * dims[2] rows."""
        d = np.ascontiguousarray(dims, np.int32)
        c = np.ascontiguousarray(cone, np.float32)
        org = np.ascontiguousarray(origin, np.float32)
        outs = [None] * N.NUM_FIELDS
        for f in fields:
            outs[N.FIELD_SLOTS[f]] = N.ptr(outs_dev[f]) if not isinstance(outs_dev[f], int) else outs_dev[f]
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        o = self._opts(fields, N.METHOD_CENTRE, 1, 0, fix, fix_outside)
        N.check(self.lib.dtfe_gpu_interpolate_cone_dev(self.h, c.ctypes.data, org.ctypes.data, d.ctypes.data,
                                                       C.byref(o), optr))

    def select_in_box(self, pos, full_box, padded, periodic: bool = True):
        """Particles of the padded box on the device (dtfe_gpu_select_in_box_dev):
        pos a (n, 3) float32 CUDA tensor; returns (int32 source indices,
        (m, 3) shifted positions) as CUDA tensors."""
        import torch
        if not pos.is_cuda or not pos.is_contiguous() or pos.dtype != torch.float32:
            raise ValueError("select_in_box takes a contiguous float32 CUDA tensor")
        fb = np.ascontiguousarray(full_box, np.float32)
        pb = np.ascontiguousarray(padded, np.float32)
        n = pos.shape[0]
        cnt = C.c_int64(0)
        N.check(self.lib.dtfe_gpu_select_in_box_dev(self.h, pos.data_ptr(), n, fb.ctypes.data, pb.ctypes.data,
                                                    1 if periodic else 0, None, None, 0, C.byref(cnt)))
        idx = torch.empty(cnt.value, dtype=torch.int32, device=pos.device)
        out = torch.empty((cnt.value, 3), dtype=torch.float32, device=pos.device)
        N.check(self.lib.dtfe_gpu_select_in_box_dev(self.h, pos.data_ptr(), n, fb.ctypes.data, pb.ctypes.data,
                                                    1 if periodic else 0, idx.data_ptr(), out.data_ptr(),
                                                    cnt.value, C.byref(cnt)))
        return idx, out

    def write_binary_dev(self, path: str, tensor) -> None:
        """Streams a contiguous float32 CUDA tensor to `path` in the
        reference's binary output format (dtfe_gpu_write_binary_dev)."""
        if not tensor.is_contiguous() or str(tensor.dtype) != "torch.float32":
            raise ValueError("write_binary_dev takes a contiguous float32 tensor")
        N.check(self.lib.dtfe_gpu_write_binary_dev(self.h, path.encode(), tensor.data_ptr(), tensor.numel()))

    def interpolate_dev_async(self, fields, outs_dev: dict, method: int = 0, n_samples: int = 1, seed: int = 0,
                              fix: bool = False) -> None:
        """Queues the interpolation into device outputs without waiting
        (dtfe_gpu_interpolate_dev_async); read_status() reports it."""
        outs = [None] * N.NUM_FIELDS
        for f in fields:
            outs[N.FIELD_SLOTS[f]] = N.ptr(outs_dev[f]) if not isinstance(outs_dev[f], int) else outs_dev[f]
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        o = self._opts(fields, method, n_samples, seed, fix)
        N.check(self.lib.dtfe_gpu_interpolate_dev_async(self.h, C.byref(o), optr))

    def graph_build(self, rho_bar: float, fields, outs_dev: dict, method: int = 0, n_samples: int = 1,
                    seed: int = 0, fix: bool = False) -> None:
        """Captures one step (vertex densities + interpolation into outs_dev)
        as a CUDA graph; graph_launch replays it."""
        outs = [None] * N.NUM_FIELDS
        for f in fields:
            outs[N.FIELD_SLOTS[f]] = N.ptr(outs_dev[f]) if not isinstance(outs_dev[f], int) else outs_dev[f]
        self._graph_outs = outs_dev  # keep the buffers alive with the graph
        optr = (C.c_void_p * N.NUM_FIELDS)(*outs)
        o = self._opts(fields, method, n_samples, seed, fix)
        N.check(self.lib.dtfe_gpu_graph_build(self.h, float(rho_bar), C.byref(o), optr))

    def graph_launch(self) -> None:
        N.check(self.lib.dtfe_gpu_graph_launch(self.h))

    def read_status(self) -> dict:
        st = N.Status()
        N.check(self.lib.dtfe_gpu_read_status(self.h, C.byref(st)))
        self.last_status = st.as_dict()
        return self.last_status

    def deposit(self, dplan, velocity: bool = True) -> dict:
        """NGP / CIC / TSC density (and velocity) on the host."""
        G = int(np.prod(dplan.grid))
        dens = np.empty(G, np.float32)
        vel = np.empty((G, 3), np.float32) if velocity and dplan.velocity is not None else None
        grid = np.asarray(dplan.grid, np.int32)
        N.check(self.lib.dtfe_gpu_deposit(self.h, dplan.kind, N.ptr(dplan.pos), N.ptr(dplan.weight),
                                          N.ptr(dplan.velocity) if vel is not None else None, dplan.n,
                                          len(dplan.boxes), C.addressof(dplan.boxes), grid.ctypes.data,
                                          dplan.rho_bar, dens.ctypes.data, N.ptr(vel)))
        return {"density": dens, "velocity": vel}

    def deposit_dev(self, dplan, density_dev, velocity_dev=None) -> None:
        grid = np.asarray(dplan.grid, np.int32)
        N.check(self.lib.dtfe_gpu_deposit_dev(self.h, dplan.kind, N.ptr(dplan.pos), N.ptr(dplan.weight),
                                              N.ptr(dplan.velocity) if velocity_dev is not None else None,
                                              dplan.n, len(dplan.boxes), C.addressof(dplan.boxes),
                                              grid.ctypes.data, dplan.rho_bar, N.ptr(density_dev),
                                              N.ptr(velocity_dev)))

    def deposit_resident(self, dplan, pos_dev, weight_dev, velocity_in_dev, density_dev, velocity_dev=None) -> None:
        """Deposit with the particles already on the device (dtfe_gpu_deposit_resident):
        pos_dev (n, 3), weight_dev (n,) or None, velocity_in_dev (n, 3) or None."""
        grid = np.asarray(dplan.grid, np.int32)
        N.check(self.lib.dtfe_gpu_deposit_resident(self.h, dplan.kind, N.ptr(pos_dev), N.ptr(weight_dev),
                                                   N.ptr(velocity_in_dev) if velocity_dev is not None else None,
                                                   dplan.n, len(dplan.boxes), C.addressof(dplan.boxes),
                                                   grid.ctypes.data, dplan.rho_bar, N.ptr(density_dev),
                                                   N.ptr(velocity_dev)))

    def sph(self, rho_bar: float, n_neighbors: int = 32, velocity: bool = True, scalars: bool = False,
            extensive: bool = False) -> dict:
        """SPH density (and velocity, scalars) on the host."""
        G = int(np.prod(self.grid))
        fields = ["density"] + (["velocity"] if velocity else []) + (["scalar"] if scalars else [])
        dens = np.empty(G, np.float32)
        vel = np.empty((G, 3), np.float32) if velocity else None
        sc = np.empty((G, self.n_scalars), np.float32) if scalars else None
        N.check(self.lib.dtfe_gpu_sph(self.h, int(n_neighbors), _mask(fields), int(extensive), float(rho_bar),
                                      N.ptr(dens), N.ptr(vel), N.ptr(sc)))
        return {"density": dens, "velocity": vel, "scalar": sc}

    def sph_dev(self, rho_bar: float, density_dev, velocity_dev=None, scalar_dev=None, n_neighbors: int = 32,
                extensive: bool = False) -> None:
        fields = ["density"] + (["velocity"] if velocity_dev is not None else []) + \
            (["scalar"] if scalar_dev is not None else [])
        N.check(self.lib.dtfe_gpu_sph_dev(self.h, int(n_neighbors), _mask(fields), int(extensive), float(rho_bar),
                                          N.ptr(density_dev), N.ptr(velocity_dev), N.ptr(scalar_dev)))

    def adjoint_dev(self, grad_xyz, grad_density=None, grad_velocity=None, grad_divergence=None,
                    grad_vel=None, grad_w=None) -> None:
        """Vertex gradients of sum(a*density + c.velocity + b*divergence) of the
        last centre interpolation (device tensors: a, b (G,), c (G, 3);
        outputs grad_xyz (V, 3), grad_vel (V, 3), grad_w (V,))."""
        N.check(self.lib.dtfe_gpu_adjoint_dev(self.h, N.ptr(grad_density), N.ptr(grad_velocity),
                                              N.ptr(grad_divergence), N.ptr(grad_xyz), N.ptr(grad_vel),
                                              N.ptr(grad_w)))

    def deposit_adjoint_dev(self, grad_density, grad_xyz, grad_w=None) -> None:
        """Particle gradients of sum(a*density) of the last deposit on this
        handle (device tensors: a (G,); outputs grad_xyz (n, 3), grad_w (n,))."""
        N.check(self.lib.dtfe_gpu_deposit_adjoint_dev(self.h, N.ptr(grad_density), N.ptr(grad_xyz),
                                                      N.ptr(grad_w)))

    def autotune(self, fields) -> tuple:
        chosen = (C.c_int32 * 2)()
        N.check(self.lib.dtfe_gpu_autotune(self.h, _mask(fields), chosen))
        return int(chosen[0]), int(chosen[1])

    def variant_counts(self) -> tuple:
        counts = (C.c_int32 * 2)()
        N.check(self.lib.dtfe_gpu_variant_counts(counts))
        return int(counts[0]), int(counts[1])

    def set_variants(self, locate: int, evaluate: int) -> None:
        N.check(self.lib.dtfe_gpu_set_variants(self.h, locate, evaluate))

    def download_located(self) -> np.ndarray:
        """Per grid cell the tetrahedron of the last cell-centre interpolation
        (dtfe_gpu_download_located): int32 (G,), -1 outside the hull."""
        out = np.empty(int(np.prod(self.grid)), np.int32)
        N.check(self.lib.dtfe_gpu_download_located(self.h, out.ctypes.data))
        return out

    def download_tets(self, n_tets: int):
        """The device's (tet_v, tet_n) arrays, (T, 4) int32 each."""
        tv = np.empty((n_tets, 4), np.int32)
        tn = np.empty((n_tets, 4), np.int32)
        N.check(self.lib.dtfe_gpu_download_tets(self.h, tv.ctypes.data, tn.ctypes.data))
        return tv, tn

    def tiles_gather_dev(self, tiles: np.ndarray, grid, field, packed) -> None:
        """Copies the tiles (K, 6 int: origin, dims) of a main-grid field
        (CUDA tensor, cells x components) into ``packed`` (CUDA tensor), tile
        after tile (dtfe_gpu_tiles_gather_dev)."""
        t = np.ascontiguousarray(tiles, np.int32).reshape(-1, 6)
        g = np.ascontiguousarray(grid, np.int32)
        nc = int(field.numel() // int(np.prod(g))) if field.numel() else 1
        N.check(self.lib.dtfe_gpu_tiles_gather_dev(self.h, len(t), t.ctypes.data, g.ctypes.data, nc,
                                                   N.ptr(field), N.ptr(packed)))

    def tiles_scatter_dev(self, tiles: np.ndarray, grid, packed, field) -> None:
        """Writes a packed buffer back into the tiles of a main-grid field
        (dtfe_gpu_tiles_scatter_dev)."""
        t = np.ascontiguousarray(tiles, np.int32).reshape(-1, 6)
        g = np.ascontiguousarray(grid, np.int32)
        nc = int(field.numel() // int(np.prod(g))) if field.numel() else 1
        N.check(self.lib.dtfe_gpu_tiles_scatter_dev(self.h, len(t), t.ctypes.data, g.ctypes.data, nc,
                                                    N.ptr(packed), N.ptr(field)))

    def set_max_walk_steps(self, n: int) -> None:
        """Step limit of the point-location walks (0 = default)."""
        N.check(self.lib.dtfe_gpu_set_max_walk_steps(self.h, int(n)))

    def locate_points(self, pts: np.ndarray, start: int = 0) -> np.ndarray:
        pts = np.ascontiguousarray(pts, np.float64)
        out = np.empty(len(pts), np.int32)
        N.check(self.lib.dtfe_gpu_locate_points(self.h, len(pts), pts.ctypes.data, int(start), out.ctypes.data))
        return out


TESS_REASONS = ("duplicate", "candidates", "star", "no_start", "flat", "undecided", "tie", "not_delaunay",
                "link", "open", "overflow", "run")


def tessellate(point_sets: list, device: int = 0, return_ms: bool = False, return_stats: bool = False):
    """Delaunay tessellations of float32 point sets on the GPU
    (dtfe_gpu_tessellate), in the host tessellator's canonical order.

    Returns [(tet_v (T,4) int32 with indices local to the set, status)];
    status 0 means the set was certified on the device, any other value
    (flag bits of dtfe_gpu_tess_sizes) that the set needs the host
    tessellator (co-spherical or coplanar points, capacity limits) and its
    tet_v is empty.  With return_ms, also the device time of the call in ms
    (CUDA events around it on its stream); with return_stats, the number of
    vertex stars that failed for each of TESS_REASONS."""
    import torch

    lib = N.gpu()
    k = len(point_sets)
    sizes = [len(p) for p in point_sets]
    vpre = np.zeros(k + 1, np.int64)
    vpre[1:] = np.cumsum(sizes)
    xyz = np.ascontiguousarray(np.concatenate([np.asarray(p, np.float32).reshape(-1, 3) for p in point_sets]))
    dev = torch.device("cuda", device)
    with torch.cuda.device(dev):
        xyz_d = torch.from_numpy(xyz).to(dev)
        stream = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        handle = C.c_void_p()
        e0.record(stream)
        N.check(lib.dtfe_gpu_tessellate(C.c_void_p(stream.cuda_stream), k, vpre.ctypes.data,
                                        C.c_void_p(xyz_d.data_ptr()), C.byref(handle)))
        e1.record(stream)
        try:
            tpre = np.zeros(k + 1, np.int64)
            status = np.zeros(k, np.int32)
            N.check(lib.dtfe_gpu_tess_sizes(handle, tpre.ctypes.data, status.ctypes.data))
            why = np.zeros(len(TESS_REASONS) + 2, np.int64)
            N.check(lib.dtfe_gpu_tess_stats(handle, why.ctypes.data, len(why)))
            tv = np.empty((int(tpre[-1]), 4), np.int32)
            if len(tv):
                N.check(lib.dtfe_gpu_tess_export(handle, tv.ctypes.data, 0))
        finally:
            lib.dtfe_gpu_tess_release(handle)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
    out = [(tv[tpre[s]:tpre[s + 1]] - np.int32(vpre[s]), int(status[s])) for s in range(k)]
    res = [out]
    if return_ms:
        res.append(ms)
    if return_stats:
        d = dict(zip(TESS_REASONS, (int(x) for x in why)))
        d["first_vertex"], d["first_reason"] = int(why[-2]), int(why[-1])
        res.append(d)
    return res[0] if len(res) == 1 else tuple(res)
