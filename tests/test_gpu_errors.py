"""Error paths of the C ABI that must not fault the GPU or poison the handle.

* A plain upload (dtfe_gpu_upload) whose tet_v holds a vertex id outside
  [0, n_verts), or whose tet_n holds a neighbour id outside [-1, n_tets), is
  refused with DTFE_ERR_ARG: a device kernel checks every id before any
  kernel indexes with them.  The handle holds nothing afterwards and takes the
  next valid upload.
* The point-location walk's step limit: with a limit of one step every walk
  that has to cross a face fails; the call reports DTFE_ERR_WALK with
  n_walk_failures > 0 (the reference exits the process on its errors,
  src/message.h:57-64), and the same handle, limit restored, interpolates
  the fields of a fresh handle bit for bit.
"""
import numpy as np
import pytest

from dtfe_b200 import _native as N
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu

FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence"]


@pytest.fixture(scope="module")
def plan(gpu_built):
    pos, psi = S.zeldovich_lattice(16, 100.0, 0.5, seed=21)
    vel = (50 * psi).astype(np.float32)
    return P.make_plan(pos, np.ones(len(pos), np.float32), vel, None, grid=(16, 16, 16), n_threads=4,
                       average_density_value=len(pos) / 1e6)


def _reference_fields(plan):
    from dtfe_b200.device import DeviceDTFE
    with DeviceDTFE(0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        return d.interpolate(FIELDS, method=0)


@pytest.mark.parametrize("which,value", [("tet_v", -1), ("tet_v", "V"), ("tet_n", -2), ("tet_n", "T")])
def test_upload_out_of_range_ids(plan, which, value):
    from copy import copy
    from dtfe_b200.device import DeviceDTFE
    bad = copy(plan)
    arr = getattr(plan, which).copy()
    v = {"V": plan.n_verts, "T": plan.n_tets}.get(value, value)
    arr[plan.n_tets // 2, 1] = v
    setattr(bad, which, arr)
    want = _reference_fields(plan)
    with DeviceDTFE(0) as d:
        with pytest.raises(N.DTFEError) as e:
            d.upload(bad)
        assert e.value.code == N.ERR_ARG
        assert "outside" in str(e.value)
        # nothing usable was uploaded
        with pytest.raises(N.DTFEError) as e2:
            d.vertex_density(plan.rho_bar)
        assert e2.value.code == N.ERR_STATE
        # the handle takes the next valid upload
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        got = d.interpolate(FIELDS, method=0)
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f


def test_walk_step_limit(plan):
    from dtfe_b200.device import DeviceDTFE
    want = _reference_fields(plan)
    with DeviceDTFE(0, 0, max_walk_steps=1) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        with pytest.raises(N.DTFEError) as e:
            d.interpolate(FIELDS, method=0)
        assert e.value.code == N.ERR_WALK
        st = d.last_status
        assert st["n_walk_failures"] > 0
        assert st["n_samples_located"] == int(np.prod(plan.grid))
        # the limit back at its default: the same handle gives the full result
        d.set_max_walk_steps(0)
        got = d.interpolate(FIELDS, method=0)
        assert d.last_status["n_walk_failures"] == 0
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f


def test_walk_step_limit_averaged(plan):
    """The averaged methods report the same failure."""
    from dtfe_b200.device import DeviceDTFE
    with DeviceDTFE(0, 0) as d:
        d.load(plan)
        d.vertex_density(plan.rho_bar)
        d.set_max_walk_steps(1)
        with pytest.raises(N.DTFEError) as e:
            d.interpolate(["density"], method=3, n_samples=8)
        assert e.value.code == N.ERR_WALK
        assert d.last_status["n_walk_failures"] > 0
