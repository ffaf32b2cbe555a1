"""Batched sub-boxes in one launch per kernel, replayed as a CUDA graph.

Uneven periodic sub-boxes (a Zel'dovich lattice plus an NFW cluster each,
padding 10% of the side), every one interpolated to its own grid tile:
the graph replay equals the plain call bit for bit, both equal the oracle
within the 1e-6 bar of the other parity tests, and a new upload drops the
graph.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from dtfe_b200 import _native as N  # noqa: E402
from dtfe_b200 import plan as P  # noqa: E402
from dtfe_b200 import synthetic as S  # noqa: E402

FIELDS = ["density", "velocity", "velocity_gradient"]
NCOMP = {"density": 1, "velocity": 3, "velocity_gradient": 9}


@pytest.fixture(scope="module")
def bplan(gpu_built):
    boxes = S.subbox_set([3000, 12000, 800, 20000, 5000, 1500], 25.0, seed0=77)
    return P.make_subbox_plan(boxes, grid=(16, 16, 16), padding_fraction=0.1)


def test_graph_replay_matches_plain_and_oracle(bplan):
    from dtfe_b200.device import DeviceDTFE
    plan = bplan
    assert plan.n_boxes == 6 and plan.grid == (96, 16, 16)
    G = int(np.prod(plan.grid))
    cuda = torch.device("cuda", 0)
    outs = {f: torch.empty((G, NCOMP[f]), device=cuda) for f in FIELDS}
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        dev.autotune(FIELDS)
        st = dev.interpolate_dev(FIELDS, outs)
        plain = {f: outs[f].cpu().numpy().copy() for f in FIELDS}
        assert st["n_walk_failures"] == 0
        dev.graph_build(plan.rho_bar, FIELDS, outs)
        for f in FIELDS:
            outs[f].zero_()
        torch.cuda.synchronize()
        for _ in range(2):
            dev.graph_launch()
        st2 = dev.read_status()
        for f in FIELDS:
            assert np.array_equal(outs[f].cpu().numpy(), plain[f]), f
        assert st2["n_samples_located"] == st["n_samples_located"]
        # a new upload invalidates the captured buffers
        dev.upload(plan)
        with pytest.raises(N.DTFEError):
            dev.graph_launch()
    d32, d64, _ = O.vertex_density(plan)
    ref, _ = O.interpolate(plan, d32, d64, FIELDS, mode=O.MODE_REF)
    for f in FIELDS:
        assert rel_err(plain[f].reshape(ref[f].shape), ref[f]) <= 1e-6, f
