"""Padded-box particle selection on the GPU (dtfe_gpu_select_in_box_dev):
bit-identical to the host restatement (dtfe_select_in_box, itself
bit-identical to the reference's findParticlesInBox,
tests/test_golden.py::test_planning_bit_exact_vs_reference) and to the
reference's own selection stored in the golden fixture: same particles, same
translation-major order, same shifted float positions."""
import numpy as np
import pytest

from conftest import golden
from dtfe_b200 import plan as P

pytestmark = pytest.mark.gpu


def _gpu(d, pos, full, padded, periodic):
    import torch
    idx, out = d.select_in_box(torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda(), full, padded,
                               periodic)
    return idx.cpu().numpy(), out.cpu().numpy()


def test_select_vs_host_and_reference(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    g = golden()
    full = np.array([0, 100, 0, 100, 0, 100], np.float32)
    rng = np.random.default_rng(31)
    big = rng.uniform(0, 100, (1_000_003, 3)).astype(np.float32)
    big[:50] = np.array([0, 100, 50], np.float32)            # on the box faces
    big[50:100] = np.array([-7.5, 108.25, 100.5], np.float32)  # on the padded faces
    with DeviceDTFE(0) as d:
        idx, out = _gpu(d, g["particles_pos"], full, g["select_padded"], True)
        assert np.array_equal(out, g["select_pos"])
        for pos, padded in ((g["particles_pos"], g["select_padded"]), (big, [-7.5, 108.25, -3, 103, -11, 100.5]),
                            (big[:1000], [20, 30, 0, 100, 40, 41])):
            for periodic in (True, False):
                want_i, want_p = P.select_in_box(pos, full, padded, periodic)
                got_i, got_p = _gpu(d, pos, full, padded, periodic)
                assert np.array_equal(got_i, want_i) and np.array_equal(got_p, want_p), (len(pos), periodic)
        empty_i, empty_p = _gpu(d, np.zeros((0, 3), np.float32), full, [0, 1, 0, 1, 0, 1], True)
        assert len(empty_i) == 0 and empty_p.shape == (0, 3)


def test_select_capacity_and_arguments(gpu_built):
    """A capacity below the selection is refused with the count returned and
    nothing written; 2^31 particles and more are refused."""
    import ctypes as C
    import torch
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    pos = torch.rand(5000, 3, device="cuda") * 100
    full = np.array([0, 100, 0, 100, 0, 100], np.float32)
    padded = np.array([-5, 105, -5, 105, -5, 105], np.float32)
    idx = torch.full((10,), -7, dtype=torch.int32, device="cuda")
    with DeviceDTFE(0) as d:
        cnt = C.c_int64(0)
        rc = d.lib.dtfe_gpu_select_in_box_dev(d.h, pos.data_ptr(), 5000, full.ctypes.data, padded.ctypes.data, 1,
                                              idx.data_ptr(), None, 10, C.byref(cnt))
        assert rc == N.ERR_TOO_LARGE and cnt.value > 5000
        assert (idx.cpu().numpy() == -7).all()
        rc = d.lib.dtfe_gpu_select_in_box_dev(d.h, pos.data_ptr(), 1 << 31, full.ctypes.data, padded.ctypes.data, 1,
                                              None, None, 0, C.byref(cnt))
        assert rc == N.ERR_TOO_LARGE
