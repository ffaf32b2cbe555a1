"""The allocation-free vertex-density entry point (dtfe_vertex_density_noalloc).

It serves callers that cannot let a library allocate device memory (their
own fixed-budget pool owns it, or an allocation's possible synchronisation is
unacceptable in their loop).  Its scratch is a static device array, so this
test checks, through the C ABI, that two calls in a row give the same
densities as the handle-based dtfe_gpu_vertex_density (within the 1-ulp
bar of the vertex-density parity test), that a call on a different input in
between does not leak state into the next, and that inputs above the stated
maximum are refused.  The file name sorts last so a run that stops at the
first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

from dtfe_b200 import _native as N
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _plan(n, seed):
    pos, psi = S.zeldovich_lattice(n, 100.0, 0.5, seed)
    w = np.random.default_rng(seed + 1).uniform(0.5, 1.5, len(pos)).astype(np.float32)
    return P.make_plan(pos, w, None, None, grid=(n, n, n), n_threads=1,
                       average_density_value=float(w.sum()) / 1e6)


def _handle_path(plan):
    from dtfe_b200.device import DeviceDTFE
    with DeviceDTFE(0, 0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        return d.download_vertex_density(plan.n_verts)


def _noalloc(plan):
    import torch
    dev = torch.device("cuda:0")
    tv = torch.from_numpy(plan.tet_v).to(dev)
    tn = torch.from_numpy(plan.tet_n).to(dev)
    xyz = torch.from_numpy(plan.xyz).to(dev)
    w = torch.from_numpy(plan.weight).to(dev)
    out = torch.full((plan.n_verts,), -1.0, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    rc = N.gpu().dtfe_vertex_density_noalloc(tv.data_ptr(), tn.data_ptr(), plan.n_tets, xyz.data_ptr(),
                                             w.data_ptr(), plan.n_verts, plan.rho_bar, out.data_ptr(), None)
    N.check(rc)
    return out.cpu().numpy()


def _ulps(a, b):
    return int(np.max(np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))))


def test_noalloc_matches_handle_path(gpu_built):
    import torch
    torch.cuda.set_device(0)
    big = _plan(20, 0)
    small = _plan(12, 5)
    assert big.n_verts <= N.NOALLOC_MAX_VERTS
    ref_big = _handle_path(big)
    ref_small = _handle_path(small)
    first = _noalloc(big)
    second = _noalloc(big)
    assert _ulps(first, ref_big) <= 1
    assert _ulps(second, ref_big) <= 1
    # a smaller input in between, then the larger one again
    assert _ulps(_noalloc(small), ref_small) <= 1
    assert _ulps(_noalloc(big), ref_big) <= 1


def test_noalloc_rejects_oversize(gpu_built):
    import torch
    torch.cuda.set_device(0)
    lib = N.gpu()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda:0")
    p = buf.data_ptr()
    rc = lib.dtfe_vertex_density_noalloc(p, p, 1, p, p, N.NOALLOC_MAX_VERTS + 1, 1.0, p, None)
    assert rc == N.ERR_TOO_LARGE
    assert b"DTFE_NOALLOC_MAX_VERTS" in lib.dtfe_last_error()
