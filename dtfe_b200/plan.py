"""Host planning of a DTFE run (the part of DTFE() before the device work).

``make_plan`` follows the reference's control flow
(src/DTFE.cpp:76-251 and DTFE_parallel, src/DTFE.cpp:287-385):

1. padding length from the particle count (User_options::updatePadding,
   src/user_options.cc:1062-1089) and the average density
   (averageDensity, src/subpartition.h:437-449) unless given;
2. for a periodic box, the particles of the padded box from the 27 periodic
   images (findParticlesInBox, src/subpartition.h:79-154);
3. the sub-box split — a 2^a 3^b processor grid (parallelGrid) balanced by NGP
   particle counts (optimalPartitionSplit) — each sub-box with its own padded
   particle set;
4. one Delaunay tessellation per sub-box (host, in parallel);
5. per-tile sample coordinates with the reference's float raster.

The result is a multi-tessellation in the flat format of include/dtfe_gpu.h:
vertex and tetrahedron arrays of all sub-boxes concatenated, with global
indices, plus one dtfe_subbox record per tile.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


@dataclass
class Plan:
    tet_v: np.ndarray          # (T, 4) int32, global vertex ids
    tet_n: np.ndarray          # (T, 4) int32, global tetrahedron ids or -1
    xyz: np.ndarray            # (V, 3) float32 vertex positions
    src: np.ndarray            # (V,) int32 source particle of each vertex
    weight: np.ndarray         # (V,) float32
    velocity: np.ndarray | None
    scalar: np.ndarray | None
    boxes: C.Array             # dtfe_subbox[K]
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    grid: tuple
    rho_bar: float
    padding: np.ndarray        # (6,) float32
    timings: dict = field(default_factory=dict)
    regions: np.ndarray | None = None  # (K, 6) float32 tile regions (xmin, xmax, ymin, ymax, zmin, zmax)
    covered_region: np.ndarray | None = None  # (6,) float32 the region the grid covers

    @property
    def n_tets(self) -> int:
        return int(self.tet_v.shape[0])

    @property
    def n_verts(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def n_boxes(self) -> int:
        return len(self.boxes)

    def region_array(self) -> np.ndarray:
        """(K, 6) float32 tile regions; without stored regions, the upper
        corners lo + dx * dims of each tile."""
        if self.regions is not None:
            return np.ascontiguousarray(self.regions, np.float32).reshape(-1, 6)
        out = np.empty((self.n_boxes, 6), np.float32)
        for k, b in enumerate(self.boxes):
            for a in range(3):
                out[k, 2 * a] = b.lo[a]
                out[k, 2 * a + 1] = np.float32(b.lo[a] + b.dx[a] * b.tile_dims[a])
        return out

    @property
    def n_scalars(self) -> int:
        return 0 if self.scalar is None else int(self.scalar.shape[1])

    def box_list(self) -> list:
        return [self.boxes[i] for i in range(len(self.boxes))]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def padding_length(n_total: int, box_length, grid, padding_particles: float = 5.0, kind: int = 0) -> np.ndarray:
    out = np.zeros(6, np.float32)
    bl = _f32(box_length)
    g = np.ascontiguousarray(grid, dtype=np.int64)
    N.host().dtfe_padding_length(kind, padding_particles, n_total, bl.ctypes.data, g.ctypes.data, out.ctypes.data)
    return out


def average_density(weight: np.ndarray) -> float:
    w = _f32(weight)
    return float(N.host().dtfe_average_density(w.ctypes.data, len(w)))


def select_in_box(pos: np.ndarray, full_box, padded_box, periodic: bool):
    pos = _f32(pos)
    fb = _f32(full_box)
    pb = _f32(padded_box)
    lib = N.host()
    n = lib.dtfe_select_in_box(pos.ctypes.data, len(pos), fb.ctypes.data, pb.ctypes.data, int(periodic), None, None)
    idx = np.empty(n, np.int32)
    out = np.empty((n, 3), np.float32)
    lib.dtfe_select_in_box(pos.ctypes.data, len(pos), fb.ctypes.data, pb.ctypes.data, int(periodic),
                           idx.ctypes.data, out.ctypes.data)
    return idx, out


def parallel_grid(n_threads: int, grid) -> tuple:
    g = np.ascontiguousarray(grid, dtype=np.int64)
    out = np.zeros(3, np.int64)
    N.host().dtfe_parallel_grid(int(n_threads), g.ctypes.data, out.ctypes.data)
    return tuple(int(x) for x in out)


def optimal_partition(pos: np.ndarray, grid, region, parts):
    pos = _f32(pos)
    g = np.ascontiguousarray(grid, dtype=np.int64)
    r = _f32(region)
    p = np.ascontiguousarray(parts, dtype=np.int64)
    n = int(np.prod(p))
    sub = np.zeros((n, 6), np.int64)
    coords = np.zeros((n, 6), np.float32)
    rc = N.host().dtfe_optimal_partition(pos.ctypes.data, len(pos), g.ctypes.data, r.ctypes.data, p.ctypes.data,
                                         sub.ctypes.data, coords.ctypes.data)
    if rc:
        raise ValueError("more partitions than grid cells along an axis")
    return sub, coords


def axis_coords(lo: float, dx: float, n: int) -> np.ndarray:
    out = np.empty(n, np.float32)
    N.host().dtfe_axis_coords(float(np.float32(lo)), float(np.float32(dx)), n, out.ctypes.data)
    return out


def tessellate_many_gpu(point_sets: list, device: int = 0):
    """The same tessellations as tessellate_many, built on the GPU
    (dtfe_gpu_tessellate, which reproduces the host tessellator's arrays):
    a set the device reports (exact ties such as lattice inputs, capacity
    limits) is tessellated on the host instead; the neighbours of all sets
    are derived on the device (dtfe_gpu_upload without tet_n)."""
    from . import device as D
    out = D.tessellate(point_sets, device=device)
    redo = [i for i, (_, st) in enumerate(out) if st != 0]
    host = dict(zip(redo, tessellate_many([point_sets[i] for i in redo]))) if redo else {}
    tvs = [host[i][0] if i in host else tv for i, (tv, _) in enumerate(out)]
    voff = np.concatenate([[0], np.cumsum([len(p) for p in point_sets])]).astype(np.int64)
    toff = np.concatenate([[0], np.cumsum([len(t) for t in tvs])]).astype(np.int64)
    tv_all = np.ascontiguousarray(np.concatenate([t + np.int32(voff[i]) for i, t in enumerate(tvs)]).astype(np.int32))
    xyz = np.ascontiguousarray(np.concatenate([np.asarray(p, np.float32).reshape(-1, 3) for p in point_sets]))
    tn_all = np.empty_like(tv_all)
    if len(tv_all):
        class _Flat:  # the arrays dtfe_gpu_upload reads
            pass
        f = _Flat()
        f.tet_v, f.tet_n, f.n_tets, f.xyz, f.n_verts = tv_all, None, len(tv_all), xyz, len(xyz)
        f.weight, f.velocity, f.scalar = np.ones(len(xyz), np.float32), None, None
        with D.DeviceDTFE(device) as dev:
            dev.upload(f, neighbours=False)
            _, tn_all = dev.download_tets(len(tv_all))
    res = []
    for i, tv in enumerate(tvs):
        if i in host:
            res.append(host[i])
            continue
        tn = tn_all[toff[i]:toff[i + 1]]
        res.append((tv, np.where(tn >= 0, tn - np.int32(toff[i]), -1).astype(np.int32),
                    np.arange(len(point_sets[i]), dtype=np.int32)))
    return res


def tessellate_many(point_sets: list, seed: int = 12345, sort_tets: bool = True):
    """Delaunay tessellations of several float32 point sets in parallel.

    Returns [(tet_v (T,4) int32, tet_n (T,4) int32, vmap (n,) int32)]."""
    lib = N.host()
    k = len(point_sets)
    xyz64 = [np.ascontiguousarray(p, dtype=np.float64) for p in point_sets]
    ptrs = (C.c_void_p * k)(*[a.ctypes.data for a in xyz64])
    ns = (C.c_int64 * k)(*[len(a) for a in xyz64])
    handles = (C.c_void_p * k)()
    rcs = (C.c_int * k)()
    lib.dtfe_tessellate_batch(k, ptrs, ns, seed, int(sort_tets), handles, rcs)
    out = []
    for i in range(k):
        nt, npt, nd = C.c_int64(), C.c_int64(), C.c_int64()
        lib.dtfe_tess_sizes(handles[i], C.byref(nt), C.byref(npt), C.byref(nd))
        tv = np.empty((nt.value, 4), np.int32)
        tn = np.empty((nt.value, 4), np.int32)
        vm = np.empty(npt.value, np.int32)
        lib.dtfe_tess_export(handles[i], tv.ctypes.data, tn.ctypes.data, vm.ctypes.data)
        lib.dtfe_tess_release(handles[i])
        if rcs[i] not in (0, 1):
            raise RuntimeError(f"tessellation of point set {i} failed (status {rcs[i]})")
        out.append((tv, tn, vm))
    return out


def _spread21(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64) & np.uint64(0x1FFFFF)
    x = (x | (x << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    x = (x | (x << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    x = (x | (x << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    x = (x | (x << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    x = (x | (x << np.uint64(2))) & np.uint64(0x1249249249249249)
    return x


def morton_order(pos: np.ndarray) -> np.ndarray:
    """Permutation sorting points along a Morton (Z-order) curve."""
    if len(pos) == 0:
        return np.zeros(0, np.int64)
    lo = pos.min(axis=0).astype(np.float64)
    ext = np.maximum(pos.max(axis=0).astype(np.float64) - lo, 1e-30)
    q = np.clip(((pos - lo) / ext * ((1 << 21) - 1)), 0, (1 << 21) - 1).astype(np.uint64)
    key = _spread21(q[:, 0]) | (_spread21(q[:, 1]) << np.uint64(1)) | (_spread21(q[:, 2]) << np.uint64(2))
    return np.argsort(key, kind="stable")


def _make_box(voff, nv, toff, nt, origin, dims, coff, dx, lo, part_no):
    b = N.Subbox()
    b.vert_offset, b.n_verts, b.tet_offset, b.n_tets = voff, nv, toff, nt
    for a in range(3):
        b.tile_origin[a] = int(origin[a])
        b.tile_dims[a] = int(dims[a])
        b.coord_offset[a] = int(coff[a])
        b.dx[a] = float(dx[a])
        b.lo[a] = float(lo[a])
    b.part_no = int(part_no)
    return b


def assemble(sets: list, tiles: list, weight, velocity, scalar, grid, rho_bar, padding, timings,
             tessellator: str = "host") -> Plan:
    """Concatenates per-sub-box (positions, source ids) and their tessellations.

    sets:  [(src_idx int32, pos float32 (n,3))]
    tiles: [(origin(3), dims(3), region(6) float32, part_no)]"""
    t0 = time.time()
    # vertices of each sub-box in Morton order: neighbouring tetrahedra then
    # reference neighbouring vertex records
    sets = [(src[o], pos[o]) for src, pos in sets for o in [morton_order(pos)]]
    timings["vertex_sort_s"] = time.time() - t0
    t0 = time.time()
    if tessellator == "gpu":
        tess = tessellate_many_gpu([p for _, p in sets])
    elif tessellator == "host":
        tess = tessellate_many([p for _, p in sets])
    else:
        raise ValueError("tessellator must be 'host' or 'gpu'")
    timings["tessellation_s"] = time.time() - t0
    tv_all, tn_all, xyz_all, src_all = [], [], [], []
    xs, ys, zs, regions = [], [], [], []
    boxes = (N.Subbox * len(sets))()
    voff = toff = 0
    coff = [0, 0, 0]
    for k, ((src, pos), (tv, tn, _vm), (origin, dims, region, part_no)) in enumerate(zip(sets, tess, tiles)):
        nv, nt = len(pos), len(tv)
        tv_all.append(tv + voff)
        tn_all.append(np.where(tn >= 0, tn + toff, -1).astype(np.int32))
        xyz_all.append(pos)
        src_all.append(src)
        region = np.asarray(region, np.float32)
        regions.append(region)
        dx = np.empty(3, np.float32)
        for a in range(3):
            length = np.float32(region[2 * a + 1] - region[2 * a])
            dx[a] = np.float32(length / np.float32(dims[a]))
        xs.append(axis_coords(region[0], dx[0], dims[0]))
        ys.append(axis_coords(region[2], dx[1], dims[1]))
        zs.append(axis_coords(region[4], dx[2], dims[2]))
        boxes[k] = _make_box(voff, nv, toff, nt, origin, dims, coff, dx, region[0::2], part_no)
        coff = [coff[0] + dims[0], coff[1] + dims[1], coff[2] + dims[2]]
        voff += nv
        toff += nt
    src = np.concatenate(src_all).astype(np.int32)
    return Plan(
        tet_v=np.ascontiguousarray(np.concatenate(tv_all)),
        tet_n=np.ascontiguousarray(np.concatenate(tn_all)),
        xyz=np.ascontiguousarray(np.concatenate(xyz_all)),
        src=src,
        weight=np.ascontiguousarray(weight[src], np.float32),
        velocity=None if velocity is None else np.ascontiguousarray(velocity[src], np.float32),
        scalar=None if scalar is None else np.ascontiguousarray(scalar[src], np.float32),
        boxes=boxes,
        xs=np.concatenate(xs), ys=np.concatenate(ys), zs=np.concatenate(zs),
        grid=tuple(int(g) for g in grid), rho_bar=float(rho_bar),
        padding=np.asarray(padding, np.float32), timings=timings,
        regions=np.ascontiguousarray(np.stack(regions), np.float32) if regions else None)


def decompose(pos, weight, grid, box, periodic: bool, n_threads: int, pad):
    """The reference's particle selection and sub-box split (DTFE(),
    src/DTFE.cpp:219-243, and DTFE_parallel, src/DTFE.cpp:298-356).

    Returns ([(source index, positions)], [(origin, dims, region, part_no)])."""
    pos = _f32(pos)
    box = np.asarray(box, np.float32)
    padded = np.array([box[0] - pad[0], box[1] + pad[1], box[2] - pad[2], box[3] + pad[3],
                       box[4] - pad[4], box[5] + pad[5]], np.float32)
    if periodic:
        src, ppos = select_in_box(pos, box, padded, True)
    else:
        src, ppos = np.arange(len(pos), dtype=np.int32), pos
    pgrid = parallel_grid(n_threads, grid)
    sets, tiles = [], []
    if np.prod(pgrid) == 1:
        sets.append((src, ppos))
        tiles.append(((0, 0, 0), tuple(grid), box, -1))
    else:
        sub, coords = optimal_partition(ppos, grid, box, pgrid)
        for k in range(len(sub)):
            region = coords[k]
            pb = np.array([region[0] - pad[0], region[1] + pad[1], region[2] - pad[2], region[3] + pad[3],
                           region[4] - pad[4], region[5] + pad[5]], np.float32)
            ki, kp = select_in_box(ppos, region, pb, False)
            sets.append((src[ki], kp))
            origin = (sub[k, 0], sub[k, 2], sub[k, 4])
            dims = (sub[k, 1] - sub[k, 0], sub[k, 3] - sub[k, 2], sub[k, 5] - sub[k, 4])
            tiles.append((origin, dims, region, k))
    return sets, tiles


def make_plan(pos, weight, velocity=None, scalar=None, grid=(64, 64, 64), box=(0, 100, 0, 100, 0, 100),
              periodic: bool = True, n_threads: int = 1, padding_particles: float = 5.0,
              padding=None, average_density_value: float | None = None, tessellator: str = "host") -> Plan:
    """Plans a single-box DTFE run split into parallelGrid(n_threads) sub-boxes.

    average_density_value=None reproduces the reference's automatic value
    (sum of weights / 35000^3); pass sum(w)/L^3 for the physical normalisation.
    tessellator="gpu" builds the sub-box tessellations on the GPU (the same
    arrays as the host tessellator's; sets with exact ties go to the host)."""
    timings = {}
    t0 = time.time()
    pos = _f32(pos)
    weight = _f32(weight) if weight is not None else np.ones(len(pos), np.float32)
    box = np.asarray(box, np.float32)
    blen = np.array([box[1] - box[0], box[3] - box[2], box[5] - box[4]], np.float32)
    pad = padding_length(len(pos), blen, grid, padding_particles) if padding is None else np.asarray(padding, np.float32)
    rho_bar = average_density(weight) if average_density_value is None else float(np.float32(average_density_value))
    sets, tiles = decompose(pos, weight, grid, box, periodic, n_threads, pad)
    timings["selection_s"] = time.time() - t0
    return assemble(sets, tiles, weight, velocity, scalar, grid, rho_bar, pad, timings, tessellator)


@dataclass
class DepositPlan:
    """Particles of every region for the NGP / CIC / TSC estimators."""
    pos: np.ndarray             # (n, 3) float32, regions concatenated
    weight: np.ndarray          # (n,) float32
    velocity: np.ndarray | None
    boxes: C.Array              # dtfe_deposit_box[K]
    grid: tuple
    rho_bar: float
    kind: int
    src: np.ndarray | None = None  # (n,) int64 input particle of each deposited copy

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


DEPOSIT_KINDS = {"NGP": 0, "CIC": 1, "TSC": 2}


def make_deposit_plan(pos, weight, velocity=None, grid=(64, 64, 64), box=(0, 100, 0, 100, 0, 100),
                      periodic: bool = True, n_threads: int = 1, kind: str = "TSC",
                      average_density_value: float | None = None) -> DepositPlan:
    """The reference's flow for a grid-deposition run: padding of one cell for
    NGP/TSC and none for CIC (updatePadding, src/user_options.cc:1073-1078),
    periodic images, sub-box split; each region's particles Morton-ordered."""
    k = DEPOSIT_KINDS[kind]
    pos = _f32(pos)
    weight = _f32(weight) if weight is not None else np.ones(len(pos), np.float32)
    box = np.asarray(box, np.float32)
    blen = np.array([box[1] - box[0], box[3] - box[2], box[5] - box[4]], np.float32)
    pad = padding_length(len(pos), blen, grid, 5.0, kind=2 if k == 1 else 1)
    rho_bar = average_density(weight) if average_density_value is None else float(np.float32(average_density_value))
    sets, tiles = decompose(pos, weight, grid, box, periodic, n_threads, pad)
    boxes = (N.DepositBox * len(sets))()
    allp, srcs = [], []
    off = 0
    for i, ((src, p), (origin, dims, region, _)) in enumerate(zip(sets, tiles)):
        o = morton_order(p)
        allp.append(p[o])
        srcs.append(src[o])
        b = boxes[i]
        b.particle_offset, b.n_particles = off, len(p)
        for a in range(6):
            b.region[a] = float(region[a])
        for a in range(3):
            b.tile_origin[a] = int(origin[a])
            b.tile_dims[a] = int(dims[a])
        off += len(p)
    src = np.concatenate(srcs).astype(np.int64)
    return DepositPlan(pos=np.ascontiguousarray(np.concatenate(allp)), weight=np.ascontiguousarray(weight[src]),
                       velocity=None if velocity is None else np.ascontiguousarray(np.asarray(velocity, np.float32)[src]),
                       boxes=boxes, grid=tuple(int(g) for g in grid), rho_bar=rho_bar, kind=k, src=src)


def make_subbox_plan(subboxes: list, grid=(64, 64, 64), padding_fraction: float = 0.1,
                     velocity_key: str = "velocity") -> Plan:
    """Plans independent periodic boxes, each interpolated to its own grid,
    stacked along x in one main grid of (K*gx, gy, gz) cells."""
    timings = {}
    t0 = time.time()
    sets, tiles = [], []
    ws, vs, ss = [], [], []
    base = 0
    for k, p in enumerate(subboxes):
        box = np.asarray(p.box, np.float32)
        side = np.float32(box[1] - box[0])
        pad = np.full(6, np.float32(padding_fraction) * side, np.float32)
        padded = np.array([box[0] - pad[0], box[1] + pad[1], box[2] - pad[2], box[3] + pad[3],
                           box[4] - pad[4], box[5] + pad[5]], np.float32)
        src, ppos = select_in_box(p.pos, box, padded, True)
        sets.append((src + base, ppos))
        tiles.append(((k * grid[0], 0, 0), tuple(grid), box, -1))
        ws.append(p.weight)
        vs.append(p.velocity if p.velocity is not None else np.zeros((p.n, 3), np.float32))
        base += p.n
    timings["selection_s"] = time.time() - t0
    weight = np.concatenate(ws)
    velocity = np.concatenate(vs)
    side = float(subboxes[0].box[1] - subboxes[0].box[0])
    rho_bar = float(np.float32(sum(float(p.weight.sum()) for p in subboxes) / (len(subboxes) * side ** 3)))
    main = (len(subboxes) * grid[0], grid[1], grid[2])
    return assemble(sets, tiles, weight, velocity, None, main, rho_bar, np.zeros(6, np.float32), timings)


def split_boxes(plan: Plan) -> list:
    """One single-box Plan per sub-box of ``plan`` (its vertices, tetrahedra
    with re-based ids, its grid tile as the whole grid): the unbatched form,
    one handle and one launch sequence per sub-box."""
    out = []
    regions = plan.region_array()
    for k, b in enumerate(plan.box_list()):
        vo, nv, to, nt = int(b.vert_offset), int(b.n_verts), int(b.tet_offset), int(b.n_tets)
        tv = np.ascontiguousarray(plan.tet_v[to:to + nt] - vo, np.int32)
        tn = plan.tet_n[to:to + nt]
        tn = np.ascontiguousarray(np.where(tn >= 0, tn - to, tn), np.int32)
        one = (N.Subbox * 1)()
        o = one[0]
        C.memmove(C.addressof(o), C.addressof(b), C.sizeof(N.Subbox))
        o.vert_offset, o.tet_offset = 0, 0
        d = [int(b.tile_dims[a]) for a in range(3)]
        co = [int(b.coord_offset[a]) for a in range(3)]
        for a in range(3):
            o.tile_origin[a] = 0
            o.coord_offset[a] = 0
        sl = slice(vo, vo + nv)
        out.append(Plan(tet_v=tv, tet_n=tn, xyz=np.ascontiguousarray(plan.xyz[sl]), src=plan.src[sl],
                        weight=np.ascontiguousarray(plan.weight[sl]),
                        velocity=None if plan.velocity is None else np.ascontiguousarray(plan.velocity[sl]),
                        scalar=None if plan.scalar is None else np.ascontiguousarray(plan.scalar[sl]),
                        boxes=one, xs=np.ascontiguousarray(plan.xs[co[0]:co[0] + d[0]]),
                        ys=np.ascontiguousarray(plan.ys[co[1]:co[1] + d[1]]),
                        zs=np.ascontiguousarray(plan.zs[co[2]:co[2] + d[2]]), grid=tuple(d),
                        rho_bar=plan.rho_bar, padding=plan.padding, regions=regions[k:k + 1].copy()))
    return out


def _view_array(ptr, dtype, shape):
    if not ptr or int(np.prod(shape)) == 0:
        return np.zeros(shape, dtype)
    n = int(np.prod(shape))
    buf = (C.c_byte * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=n).reshape(shape).copy()


def native_plan(kind: str, pos, weight, velocity=None, scalar=None, grid=(64, 64, 64),
                box=(0, 100, 0, 100, 0, 100), periodic: bool = True, n_threads: int = 1,
                padding_particles: float = 5.0, average_density_value: float | None = None,
                region=None, partition=None, part_no: int = -1, padding=None, padding_absolute: bool = False):
    """The same plan built by the C++ planner (dtfe_plan_build_ex,
    include/dtfe_host.h): a Plan for "DTFE", a DepositPlan for "NGP", "CIC",
    "TSC".  DTFE()'s options: region (6 absolute coordinates, --region),
    partition (3 chunk counts, --partition) with part_no (--partNo, -1 all
    chunks), padding (6 lengths, in box lengths or absolute with
    padding_absolute: --padding l1..l6 / --paddingMpc).  The plan's grid
    and .covered_region are what the results cover (one chunk's with
    part_no >= 0)."""
    kinds = {"DTFE": 0, "NGP": 1, "CIC": 2, "TSC": 3}
    k = kinds[kind]
    pos = _f32(pos)
    w = None if weight is None else _f32(weight)
    vel = None if velocity is None else _f32(velocity)
    S = 0 if scalar is None else int(np.asarray(scalar).reshape(len(pos), -1).shape[1])
    sc = None if scalar is None else np.ascontiguousarray(np.asarray(scalar, np.float32).reshape(len(pos), S))
    bx = _f32(box)
    g = np.ascontiguousarray(grid, np.int32)
    lib = N.host()
    h = C.c_void_p()
    o = N.PlanOptions()
    o.n_parts = int(n_threads)
    o.padding_particles = float(padding_particles)
    o.padding_mode = N.PAD_PARTICLES
    if padding is not None:
        o.padding_mode = N.PAD_ABSOLUTE if padding_absolute else N.PAD_RELATIVE
        o.padding[:] = [float(x) for x in np.asarray(padding, np.float32)]
    if region is not None:
        o.region_on = 1
        o.region[:] = [float(x) for x in np.asarray(region, np.float32)]
    if partition is not None:
        o.partition_on = 1
        o.partition[:] = [int(x) for x in partition]
    o.part_no = int(part_no)
    o.average_density = float(np.float32(average_density_value)) if average_density_value is not None else 0.0
    rc = lib.dtfe_plan_build_ex(k, pos.ctypes.data, None if w is None else w.ctypes.data,
                                None if vel is None else vel.ctypes.data, None if sc is None else sc.ctypes.data, S,
                                len(pos), bx.ctypes.data, int(periodic), g.ctypes.data, C.byref(o), C.byref(h))
    if rc:
        raise RuntimeError(f"dtfe_plan_build_ex failed with status {rc}")
    try:
        v = N.PlanView()
        lib.dtfe_plan_get(h, C.byref(v))
        if k == 0:
            V, T, K = v.n_verts, v.n_tets, v.n_boxes
            boxes = (N.Subbox * K)()
            C.memmove(C.addressof(boxes), v.boxes, C.sizeof(N.Subbox) * K)
            return Plan(tet_v=_view_array(v.tet_v, np.int32, (T, 4)), tet_n=_view_array(v.tet_n, np.int32, (T, 4)),
                        xyz=_view_array(v.xyz, np.float32, (V, 3)), src=_view_array(v.src, np.int32, (V,)),
                        weight=_view_array(v.weight, np.float32, (V,)),
                        velocity=_view_array(v.velocity, np.float32, (V, 3)) if v.velocity else None,
                        scalar=_view_array(v.scalar, np.float32, (V, v.n_scalars)) if v.scalar else None,
                        boxes=boxes, xs=_view_array(v.xs, np.float32, (v.n_xs,)),
                        ys=_view_array(v.ys, np.float32, (v.n_ys,)), zs=_view_array(v.zs, np.float32, (v.n_zs,)),
                        grid=tuple(int(x) for x in v.grid), rho_bar=float(v.rho_bar),
                        padding=np.array(list(v.padding), np.float32),
                        regions=_view_array(v.regions, np.float32, (K, 6)) if v.regions else None,
                        covered_region=np.array(list(v.region), np.float32))
        n, K = v.n_particles, v.n_dep_boxes
        boxes = (N.DepositBox * K)()
        C.memmove(C.addressof(boxes), v.dep_boxes, C.sizeof(N.DepositBox) * K)
        return DepositPlan(pos=_view_array(v.dep_pos, np.float32, (n, 3)),
                           weight=_view_array(v.dep_weight, np.float32, (n,)),
                           velocity=_view_array(v.dep_velocity, np.float32, (n, 3)) if v.dep_velocity else None,
                           boxes=boxes, grid=tuple(int(x) for x in v.grid), rho_bar=float(v.rho_bar), kind=k - 1,
                           src=_view_array(v.dep_src, np.int64, (n,)))
    finally:
        lib.dtfe_plan_release(h)


def pack_tets(tet_v: np.ndarray, tet_n: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
    """The packed form of a tessellation (dtfe_tets_pack): uint8 bytes,
    about 16 per tetrahedron.  ``out`` (e.g. pinned memory) is used when it
    is large enough."""
    tv = np.ascontiguousarray(tet_v, np.int32)
    tn = np.ascontiguousarray(tet_n, np.int32)
    lib = N.host()
    n = int(lib.dtfe_tets_pack(tv.ctypes.data, tn.ctypes.data, len(tv), None))
    if n < 0:
        raise ValueError("cannot pack these arrays")
    buf = out[:n] if out is not None and out.nbytes >= n else np.empty(n, np.uint8)
    lib.dtfe_tets_pack(tv.ctypes.data, tn.ctypes.data, len(tv), buf.ctypes.data)
    return buf


def vertex_codes(plan, pos: np.ndarray, box=(0.0, 100.0, 0.0, 100.0, 0.0, 100.0)):
    """Per vertex its source particle and periodic image as one uint32
    (dtfe_gpu_upload_packed_particles): bits 0-26 plan.src, bits 27-31
    i1 * 9 + i2 * 3 + i3 where vertex = pos[src] - (i - 1) * box length per
    axis in float32, the padded-box selection's arithmetic.  Returns
    (codes, box_length float32[3]); raises if a vertex is not such an image
    of its particle."""
    pos = np.asarray(pos, np.float32)
    if len(pos) > (1 << 27):
        raise ValueError("more than 2^27 particles")
    b = np.asarray(box, np.float32)
    L = np.array([b[1] - b[0], b[3] - b[2], b[5] - b[4]], np.float32)
    p = pos[plan.src]
    img = np.zeros(plan.n_verts, np.uint32)
    for k in range(3):
        found = np.zeros(plan.n_verts, bool)
        ik = np.full(plan.n_verts, 1, np.uint32)
        for i in (1, 0, 2):
            shifted = (p[:, k] - np.float32(i - 1) * L[k]).astype(np.float32)
            hit = ~found & (shifted == plan.xyz[:, k])
            ik[hit] = i
            found |= hit
        if not found.all():
            raise ValueError("vertices that are not periodic images of their particles")
        img = img * 3 + ik
    codes = (plan.src.astype(np.uint32) | (img << np.uint32(27))).astype(np.uint32)
    return codes, L


def pack_tet_vertices(tet_v: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
    """The vertex-only packed form of a tessellation
    (dtfe_tets_pack_vertices, about 5 bytes per tetrahedron): the device
    derives the neighbours.  ``out`` (e.g. pinned memory) is used when it is
    large enough."""
    tv = np.ascontiguousarray(tet_v, np.int32)
    lib = N.host()
    n = int(lib.dtfe_tets_pack_vertices(tv.ctypes.data, len(tv), None))
    if n < 0:
        raise ValueError("cannot pack these arrays (tetrahedra not in canonical vertex order)")
    buf = out[:n] if out is not None and out.nbytes >= n else np.empty(n, np.uint8)
    lib.dtfe_tets_pack_vertices(tv.ctypes.data, len(tv), buf.ctypes.data)
    return buf


def unpack_tet_vertices(packed: np.ndarray, n_tets: int) -> np.ndarray:
    tv = np.empty((n_tets, 4), np.int32)
    if N.host().dtfe_tets_unpack_vertices(packed.ctypes.data, packed.nbytes, tv.ctypes.data):
        raise ValueError("malformed packed tessellation")
    return tv


def unpack_tets(packed: np.ndarray, n_tets: int):
    tv = np.empty((n_tets, 4), np.int32)
    tn = np.empty((n_tets, 4), np.int32)
    if N.host().dtfe_tets_unpack(packed.ctypes.data, packed.nbytes, tv.ctypes.data, tn.ctypes.data):
        raise ValueError("malformed packed tessellation")
    return tv, tn
