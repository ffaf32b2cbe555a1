"""Packed upload (dtfe_gpu_upload_packed) gives the device exactly the
tessellation of the plain upload: every field bit-identical."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from dtfe_b200 import plan as P  # noqa: E402
from dtfe_b200 import synthetic as S  # noqa: E402

FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence"]


def test_packed_upload_identical(gpu_built):
    from dtfe_b200.device import DeviceDTFE
    pos, psi = S.zeldovich_lattice(20, 100.0, 1.0, seed=12)
    vel = (50 * psi).astype(np.float32)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), vel, None, grid=(20, 20, 20), n_threads=8)
    packed = P.pack_tets(plan.tet_v, plan.tet_n)
    out = []
    for use_packed in (False, True):
        with DeviceDTFE(0) as dev:
            if use_packed:
                dev.upload_packed(plan, packed)
            else:
                dev.upload(plan)
            dev.set_subboxes(plan)
            dev.vertex_density(plan.rho_bar)
            out.append((dev.interpolate(FIELDS, method=0), dev.download_vertex_density(plan.n_verts)))
    for f in FIELDS:
        assert np.array_equal(out[0][0][f], out[1][0][f]), f
    assert np.array_equal(out[0][1], out[1][1])
