"""Sharding a box's sub-boxes over ranks (one process per GPU).

The reference splits a box into independent padded sub-boxes, one per
OpenMP thread (DTFE_parallel, src/DTFE.cpp:287-385; optimalPartitionSplit,
src/subpartition.h:215-372), and copies every thread's tile into the main
grid (copySubgridResultsToMain, src/subpartition.h:399-432).  Here the same
split is made for ``world * parts_per_rank`` parts; each rank tessellates and
interpolates only the parts assigned to it (greedy by particle count, so the
heaviest part goes to the least loaded rank) and the disjoint grid tiles are
exchanged once with an all-gather of packed tiles.  No collective runs
inside the interpolation itself.

Every rank must call ``gather_fields`` (a collective) in the same order.
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
    tables = [t[:int(c.item())].cpu().numpy() for t, c in zip(tables, all_counts)]
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
