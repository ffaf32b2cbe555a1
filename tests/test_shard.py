"""Sharding sub-boxes over ranks, on the CPU with gloo (world size 2).

Each rank takes its share of the reference's split of one box into
world x parts_per_rank sub-boxes, interpolates it (here with the oracle, as
the GPU box is not needed for the host logic) and all-gathers the tiles: the
gathered grid equals the single-process run with the same split, bit for bit.
"""
import os
import socket

import numpy as np
import pytest

from dtfe_b200 import shard


def test_assign_parts_balanced():
    costs = [50, 10, 40, 30, 20, 60]
    parts = shard.assign_parts(costs, 2)
    assert sorted(parts[0] + parts[1]) == list(range(6))
    loads = [sum(costs[k] for k in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= 10
    assert shard.assign_parts([5], 1) == [[0]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    import oracle as O
    from dtfe_b200 import shard as SH
    from dtfe_b200 import synthetic as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pos, psi = S.zeldovich_lattice(12, 100.0, 0.8, seed=4)
        w = np.random.default_rng(5).uniform(0.5, 1.5, len(pos)).astype(np.float32)
        vel = (30 * psi).astype(np.float32)
        plan, parts = SH.make_rank_plan(pos, w, vel, None, grid=(12, 10, 14), world=world, rank=rank,
                                        parts_per_rank=2, average_density_value=float(w.sum()) / 1e6)
        d32, d64, _ = O.vertex_density(plan)
        f, _ = O.interpolate(plan, d32, d64, ["density", "velocity"], mode=O.MODE_REF)
        full = SH.gather_fields(plan, {"density": f["density"].astype(np.float32),
                                       "velocity": f["velocity"].astype(np.float32)})
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), density=full["density"], velocity=full["velocity"],
                 parts=np.array(parts))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_gather_equals_single_process(built, tmp_path):
    import multiprocessing as mp
    import oracle as O
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in range(2))
    assert sorted(list(r0["parts"]) + list(r1["parts"])) == [0, 1, 2, 3]
    pos, psi = S.zeldovich_lattice(12, 100.0, 0.8, seed=4)
    w = np.random.default_rng(5).uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (30 * psi).astype(np.float32)
    plan = P.make_plan(pos, w, vel, None, grid=(12, 10, 14), n_threads=4,
                       average_density_value=float(w.sum()) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    ref, _ = O.interpolate(plan, d32, d64, ["density", "velocity"], mode=O.MODE_REF)
    for r in (r0, r1):
        assert np.array_equal(r["density"], ref["density"].astype(np.float32))
        assert np.array_equal(r["velocity"], ref["velocity"].astype(np.float32))
