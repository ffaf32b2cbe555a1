"""Sharding a box's sub-boxes over ranks (one process per GPU).

The reference splits a box into independent padded sub-boxes, one per
OpenMP thread (DTFE_parallel, src/DTFE.cpp:287-385; optimalPartitionSplit,
src/subpartition.h:215-372), and copies every thread's tile into the main
grid (copySubgridResultsToMain, src/subpartition.h:399-432).  Here the same
split is made for ``world * parts_per_rank`` parts; each rank tessellates and
interpolates only the parts assigned to it (greedy by particle count, so the
heaviest part goes to the least loaded rank) and the disjoint grid tiles are
exchanged once with an all-gather (or a gather to one rank) of packed
tiles.  No collective runs inside the interpolation itself.

``gather_fields_dev`` exchanges device fields: the tiles are packed and
unpacked by kernels (dtfe_gpu_tiles_gather_dev / _scatter_dev) and, with
NCCL, never leave the GPUs; ``gather_fields`` is the host form for numpy
fields.  Every rank must call them (collectives) in the same order.

Grid deposition (NGP / CIC / TSC) needs no halo exchange here: the reference
deposits every region's own padded particles into the region's own tile
with stencils clipped at its edges (src/CIC_interpolation.cc:119-264), so
ranks holding different regions write disjoint tiles and the same tile
exchange assembles the grid.
"""
from __future__ import annotations

import numpy as np

from . import plan as P


def assign_parts(costs, world: int) -> list:
    """Parts per rank: longest-processing-time greedy over ``costs``
    (ties to the lower rank), each rank's parts in ascending order."""
    order = sorted(range(len(costs)), key=lambda k: (-int(costs[k]), k))
    load = [0] * world
    out = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += int(costs[k])
    return [sorted(o) for o in out]


def make_rank_plan(pos, weight, velocity=None, scalar=None, grid=(64, 64, 64), box=(0, 100, 0, 100, 0, 100),
                   world: int = 1, rank: int = 0, parts_per_rank: int = 1, periodic: bool = True,
                   padding_particles: float = 5.0, average_density_value: float | None = None):
    """This rank's share of the reference's split of one box into
    ``world * parts_per_rank`` sub-boxes.  Returns (plan, parts): ``plan``
    covers only this rank's sub-boxes (their tiles sit at their place in the
    full grid ``grid``), ``parts`` the sub-box numbers it holds."""
    pos = np.ascontiguousarray(pos, np.float32)
    weight = np.ones(len(pos), np.float32) if weight is None else np.ascontiguousarray(weight, np.float32)
    boxa = np.asarray(box, np.float32)
    blen = np.array([boxa[1] - boxa[0], boxa[3] - boxa[2], boxa[5] - boxa[4]], np.float32)
    pad = P.padding_length(len(pos), blen, grid, padding_particles)
    rho_bar = P.average_density(weight) if average_density_value is None else \
        float(np.float32(average_density_value))
    sets, tiles = P.decompose(pos, weight, grid, boxa, periodic, world * parts_per_rank, pad)
    mine = assign_parts([len(s[1]) for s in sets], world)[rank]
    if not mine:
        raise ValueError(f"the split made {len(sets)} sub-boxes, fewer than {world} ranks")
    plan = P.assemble([sets[k] for k in mine], [tiles[k] for k in mine], weight, velocity, scalar, grid, rho_bar,
                      pad, {})
    return plan, mine


def pack_tiles(plan, field: np.ndarray) -> np.ndarray:
    """The values of ``field`` (main-grid layout, shape (G,) or (G, c)) on
    the plan's tiles, concatenated tile by tile (x, y, z order inside)."""
    g = plan.grid
    f = field.reshape(g + field.shape[1:])
    parts = []
    for b in plan.box_list():
        o = [b.tile_origin[a] for a in range(3)]
        d = [b.tile_dims[a] for a in range(3)]
        parts.append(f[o[0]:o[0] + d[0], o[1]:o[1] + d[1], o[2]:o[2] + d[2]].reshape((-1,) + field.shape[1:]))
    return np.concatenate(parts) if parts else np.zeros((0,) + field.shape[1:], field.dtype)


def tile_table(plan) -> np.ndarray:
    """(K, 6) int64 origin and dims of the plan's tiles."""
    return np.array([[b.tile_origin[0], b.tile_origin[1], b.tile_origin[2], b.tile_dims[0], b.tile_dims[1],
                      b.tile_dims[2]] for b in plan.box_list()], np.int64).reshape(-1, 6)


def gather_fields(plan, fields: dict, group=None, device=None) -> dict:
    """All-gathers every rank's tiles of ``fields`` (name -> array in the
    main-grid layout, only this rank's tiles meaningful) into the full grid
    on every rank.  Two collectives: tile tables (sizes), then one padded
    all-gather per field.  ``device``: the torch device the exchange runs
    on ("cuda:<local rank>" with NCCL, None = CPU with gloo)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    tables = _exchange_tables(plan, group, device)
    sizes = [int(np.prod(t[:, 3:6], axis=1).sum()) if len(t) else 0 for t in tables]
    smax = max(max(sizes), 1)
    g = plan.grid
    out = {}
    for name, arr in fields.items():
        comp = arr.shape[1:] if arr.ndim > 1 else ()
        packed = pack_tiles(plan, arr)
        buf = torch.zeros((smax,) + comp, dtype=torch.float32, device=device)
        if len(packed):
            buf[:len(packed)] = torch.from_numpy(np.ascontiguousarray(packed, np.float32)).to(buf.device)
        bufs = [torch.zeros_like(buf) for _ in range(world)]
        dist.all_gather(bufs, buf, group=group)
        full = np.zeros(g + comp, np.float32)
        for t, b, n in zip(tables, bufs, sizes):
            vals = b[:n].cpu().numpy()
            pos = 0
            for o0, o1, o2, d0, d1, d2 in t:
                m = int(d0 * d1 * d2)
                full[o0:o0 + d0, o1:o1 + d1, o2:o2 + d2] = vals[pos:pos + m].reshape((d0, d1, d2) + comp)
                pos += m
        out[name] = full.reshape((-1,) + comp)
    return out


def _exchange_tables(plan, group, device):
    """Every rank's tile table: list of (K_r, 6) int64 arrays, rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    table = tile_table(plan)
    counts = torch.tensor([table.shape[0]], dtype=torch.int64, device=device)
    all_counts = [torch.zeros_like(counts) for _ in range(world)]
    dist.all_gather(all_counts, counts, group=group)
    kmax = int(max(int(c.item()) for c in all_counts))
    tpad = torch.full((max(kmax, 1), 6), -1, dtype=torch.int64, device=device)
    if table.shape[0]:
        tpad[:table.shape[0]] = torch.from_numpy(table).to(tpad.device)
    tables = [torch.zeros_like(tpad) for _ in range(world)]
    dist.all_gather(tables, tpad, group=group)
    return [t[:int(c.item())].cpu().numpy() for t, c in zip(tables, all_counts)]


def gather_fields_dev(dev, plan, fields: dict, group=None, root: int | None = None, tables=None) -> dict:
    """The tile exchange on device fields: ``fields`` maps names to CUDA
    tensors in the main-grid layout (cells x components; only this rank's
    tiles meaningful).  This rank's tiles are packed on the device, one
    all-gather per field (or one gather to ``root``) moves the packed
    buffers, and each rank's buffer is scattered into a full-grid tensor on
    the device.  With NCCL the buffers stay in device memory; with gloo (CPU
    collectives) they are staged through host memory.  Returns name -> full
    grid (CUDA tensor) on every rank, or on ``root`` only (None elsewhere).
    ``tables`` (every rank's tile table) may be passed to skip their
    exchange on repeated calls."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    on_gpu = dist.get_backend(group) == "nccl"
    any_field = next(iter(fields.values()))
    cdev = any_field.device
    tables = tables if tables is not None else _exchange_tables(plan, group, cdev if on_gpu else None)
    sizes = [int(np.prod(t[:, 3:6], axis=1).sum()) if len(t) else 0 for t in tables]
    smax = max(max(sizes), 1)
    grid = tuple(int(x) for x in plan.grid)
    G = int(np.prod(grid))
    mine = tile_table(plan)
    out = {}
    for name, arr in fields.items():
        nc = int(arr.numel() // G)
        buf = torch.zeros(smax * nc, dtype=torch.float32, device=cdev)
        # buffers are filled on torch's stream, packed and unpacked on the
        # handle's (each of those calls returns when its copy is done)
        torch.cuda.current_stream(cdev).synchronize()
        if sizes[rank]:
            dev.tiles_gather_dev(mine, grid, arr, buf)
        send = buf if on_gpu else buf.cpu()
        if root is None:
            bufs = [torch.empty_like(send) for _ in range(world)]
            dist.all_gather(bufs, send, group=group)
        else:
            bufs = [torch.empty_like(send) for _ in range(world)] if rank == root else None
            dist.gather(send, bufs, dst=root, group=group)
        if root is not None and rank != root:
            out[name] = None
            continue
        if not on_gpu:
            bufs = [b.to(cdev) for b in bufs]
        full = torch.zeros(arr.shape, dtype=torch.float32, device=cdev)
        torch.cuda.current_stream(cdev).synchronize()  # the collective, copies and fill, before the unpacking
        for t, b, n in zip(tables, bufs, sizes):
            if n:
                dev.tiles_scatter_dev(t, grid, b, full)
        out[name] = full
    return out
