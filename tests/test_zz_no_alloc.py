"""The allocation-free vertex-density entry point (dtfe_vertex_density_noalloc).

It serves callers that cannot let a library allocate device memory (their
own fixed-budget pool owns it, or an allocation's possible synchronisation is
unacceptable in their loop).  Its scratch is a static device array, so this
test checks, through the C ABI, that two calls in a row give the same
densities, bit for bit, as the handle-based dtfe_gpu_vertex_density (both
add the volumes as exact integers in units of the vertices' bounding box,
so the order the GPU adds in does not matter), that a call on a different
input in between does not leak state into the next, that a call on a
non-default stream and one without tetrahedra behave, that vertex ids out of range are refused with the output
left untouched and the next call still right, and that inputs above the
stated maximum are refused.  The file name sorts last so a run that stops at
the first failure has run every other test first.
"""
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


def _noalloc(plan, tet_v=None, stream=None, fill=-1.0, n_tets=None):
    """Runs the entry point; returns (status, densities on the host)."""
    import torch
    dev = torch.device("cuda:0")
    tv = torch.from_numpy(plan.tet_v if tet_v is None else tet_v).to(dev)
    tn = torch.from_numpy(plan.tet_n).to(dev)
    xyz = torch.from_numpy(plan.xyz).to(dev)
    w = torch.from_numpy(plan.weight).to(dev)
    out = torch.full((plan.n_verts,), fill, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    rc = N.gpu().dtfe_vertex_density_noalloc(tv.data_ptr(), tn.data_ptr(), plan.n_tets if n_tets is None else n_tets,
                                             xyz.data_ptr(), w.data_ptr(), plan.n_verts, plan.rho_bar,
                                             out.data_ptr(), stream)
    return rc, out.cpu().numpy()


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
    rc1, first = _noalloc(big)
    rc2, second = _noalloc(big)
    assert rc1 == rc2 == N.OK
    assert np.array_equal(first.view(np.int32), second.view(np.int32))
    assert np.array_equal(first.view(np.int32), ref_big.view(np.int32)), _ulps(first, ref_big)
    # a smaller input in between, then the larger one again
    rc, got_small = _noalloc(small)
    assert rc == N.OK and np.array_equal(got_small.view(np.int32), ref_small.view(np.int32))
    rc, again = _noalloc(big)
    assert rc == N.OK and np.array_equal(again.view(np.int32), first.view(np.int32))


def test_noalloc_stream_and_empty(gpu_built):
    """On a non-default stream the call gives the same bits; without
    tetrahedra every density is 0."""
    import torch
    torch.cuda.set_device(0)
    plan = _plan(14, 3)
    rc, ref = _noalloc(plan)
    assert rc == N.OK
    s = torch.cuda.Stream()
    rc, got = _noalloc(plan, stream=s.cuda_stream)
    assert rc == N.OK and np.array_equal(got.view(np.int32), ref.view(np.int32))
    rc, empty = _noalloc(plan, n_tets=0, fill=7.0)
    assert rc == N.OK and not empty.any()


def test_noalloc_bad_ids(gpu_built):
    """A vertex id outside [0, n_verts) is refused (DTFE_ERR_ARG) before any
    kernel indexes with it; the output keeps its contents and the next call
    on good input is right."""
    import torch
    torch.cuda.set_device(0)
    plan = _plan(12, 7)
    rc, ref = _noalloc(plan)
    assert rc == N.OK
    for v in (-1, plan.n_verts):
        bad = plan.tet_v.copy()
        bad[plan.n_tets // 3, 2] = v
        rc, got = _noalloc(plan, tet_v=bad, fill=5.0)
        assert rc == N.ERR_ARG
        assert b"n_verts" in N.gpu().dtfe_last_error()
        assert np.all(got == 5.0)
    rc, got = _noalloc(plan)
    assert rc == N.OK and np.array_equal(got.view(np.int32), ref.view(np.int32))


def test_noalloc_rejects_oversize(gpu_built):
    import torch
    torch.cuda.set_device(0)
    lib = N.gpu()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda:0")
    p = buf.data_ptr()
    rc = lib.dtfe_vertex_density_noalloc(p, p, 1, p, p, N.NOALLOC_MAX_VERTS + 1, 1.0, p, None)
    assert rc == N.ERR_TOO_LARGE
    assert b"DTFE_NOALLOC_MAX_VERTS" in lib.dtfe_last_error()
