"""One box split over two ranks, run through the product on the GPU.

Two processes on one GPU in a gloo group (this pool gives one GPU per run;
the ranks' kernels never wait on one another): each rank plans its share of
the reference's split of one box into 2 x 2 sub-boxes (make_rank_plan),
interpolates it with the CUDA kernels into device tensors, and the tiles are
exchanged with gather_fields_dev (packed and unpacked by device kernels,
staged through host memory by gloo; NCCL keeps them on the GPUs).  Every
rank's gathered grid equals the single-process GPU run of the same split,
bit for bit, and a gather to rank 0 gives rank 0 the same grid.
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence"]
GRID = (16, 14, 18)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs():
    from dtfe_b200 import synthetic as S
    pos, psi = S.zeldovich_lattice(16, 100.0, 0.8, seed=40)
    w = np.random.default_rng(41).uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (30 * psi).astype(np.float32)
    return pos, w, vel


def _worker(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import datetime
    import torch
    import torch.distributed as dist
    from dtfe_b200 import _native as NF
    from dtfe_b200 import shard as SH
    from dtfe_b200.device import DeviceDTFE
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        pos, w, vel = _inputs()
        plan, parts = SH.make_rank_plan(pos, w, vel, None, grid=GRID, world=world, rank=rank, parts_per_rank=2,
                                        average_density_value=float(w.sum()) / 1e6)
        G = int(np.prod(GRID))
        outs = {f: torch.zeros((G, NF.field_components(NF.FIELD_SLOTS[f], 0)), dtype=torch.float32,
                               device="cuda:0") for f in FIELDS}
        with DeviceDTFE(0) as dev:
            dev.load(plan)
            dev.vertex_density(plan.rho_bar)
            dev.interpolate_dev(FIELDS, outs, method=0)
            dev.synchronize()
            full = SH.gather_fields_dev(dev, plan, outs)
            to_root = SH.gather_fields_dev(dev, plan, outs, root=0)
            res = {f: full[f].cpu().numpy() for f in FIELDS}
            if rank == 0:
                res.update({"root_" + f: to_root[f].cpu().numpy() for f in FIELDS})
            else:
                assert all(v is None for v in to_root.values())
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), parts=np.array(parts), **res)
    finally:
        dist.destroy_process_group()


def test_two_ranks_one_gpu_gather_equals_single_process(gpu_built, tmp_path):
    import multiprocessing as mp
    from dtfe_b200 import plan as P
    from dtfe_b200.device import DeviceDTFE
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in range(2))
    assert sorted(list(r0["parts"]) + list(r1["parts"])) == [0, 1, 2, 3]
    pos, w, vel = _inputs()
    plan = P.make_plan(pos, w, vel, None, grid=GRID, n_threads=4, average_density_value=float(w.sum()) / 1e6)
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        ref = dev.interpolate(FIELDS, method=0)
    for f in FIELDS:
        want = ref[f].reshape(r0[f].shape)
        assert np.array_equal(r0[f], want), f
        assert np.array_equal(r1[f], want), f
        assert np.array_equal(r0["root_" + f], want), f
