"""GPU Delaunay tessellation (dtfe_gpu_tessellate) against the host
tessellator (delaunay.cpp, the stand-in for CGAL's delaunayTriangulation,
src/CGAL_triangulation/triangulation.cpp:162-195): the same tetrahedra in the
same canonical order, array for array, or a non-zero status where the
certificate meets an exact tie."""
import numpy as np
import pytest

from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _check_equal(sets):
    from dtfe_b200 import device as D
    host = P.tessellate_many(sets)
    dev = D.tessellate(sets)
    for (tv_h, _tn, _vm), (tv_d, st), pts in zip(host, dev, sets):
        assert st == 0, f"status {st} for a set of {len(pts)} points"
        assert tv_d.shape == tv_h.shape
        assert np.array_equal(tv_d, tv_h)


def test_uniform_random_sets(built):
    rng = np.random.default_rng(3)
    sets = [(rng.random((n, 3)) * 10.0).astype(np.float32) for n in (5, 40, 700, 6000)]
    _check_equal(sets)


def test_zeldovich_subboxes(built):
    """The padded sub-box point sets of a Zel'dovich plan (four sub-boxes),
    in the planner's Morton order."""
    pos, _ = S.zeldovich_lattice(24, 100.0, 1.0, seed=5)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(24, 24, 24), n_threads=4)
    sets = [plan.xyz[b.vert_offset:b.vert_offset + b.n_verts] for b in plan.boxes]
    _check_equal(sets)


def test_config0_size_subboxes(built):
    """64^3 Zel'dovich particles (rms 0.5, seed 0) split for 4 threads with
    the default padding: every sub-box tessellation equals the host's."""
    pos, _ = S.zeldovich_lattice(64, 100.0, 0.5, seed=0)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(128, 128, 128), n_threads=4)
    sets = [plan.xyz[b.vert_offset:b.vert_offset + b.n_verts] for b in plan.boxes]
    _check_equal(sets)
    assert sum(len(s) for s in sets) > 300_000


def test_clustered_set(built):
    """A dense NFW-like cluster inside a lattice: candidate blocks near the
    centre hold many points, the hull is far."""
    pos, _ = S.lattice_plus_nfw(20000, 10.0, seed=11)
    _check_equal([np.ascontiguousarray(pos, np.float32)])


def test_ties_and_bad_input_are_reported(built):
    """A cubic lattice (co-spherical corners), a non-finite coordinate, a
    three-point set and an empty set give non-zero status and no tetrahedra;
    a good set in the same call is still tessellated."""
    from dtfe_b200 import device as D
    g = np.arange(5, dtype=np.float32)
    lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(8)
    good = rng.random((300, 3)).astype(np.float32)
    nan = good.copy()
    nan[7, 1] = np.nan
    tiny = good[:3].copy()
    empty = np.zeros((0, 3), np.float32)
    out = D.tessellate([lattice, good, nan, tiny, empty])
    assert out[0][1] & 1 and len(out[0][0]) == 0
    assert out[1][1] == 0
    assert np.array_equal(out[1][0], P.tessellate_many([good])[0][0])
    assert out[2][1] & 32 and len(out[2][0]) == 0
    assert out[3][1] & 32 and len(out[3][0]) == 0
    assert out[4][1] & 32 and len(out[4][0]) == 0
    assert D.tessellate([empty])[0][1] & 32


def test_plan_with_gpu_tessellator(built):
    """make_plan(tessellator="gpu"): the same tet_v and tet_n as the host
    tessellator's plan, neighbours derived on the device; a perfect lattice
    (every set tied) falls back to the host set by set."""
    for rms in (1.0, 0.0):
        pos, _ = S.zeldovich_lattice(20, 100.0, rms, seed=6)
        w = np.ones(len(pos), np.float32)
        a = P.make_plan(pos, w, None, None, grid=(20, 20, 20), n_threads=4)
        b = P.make_plan(pos, w, None, None, grid=(20, 20, 20), n_threads=4, tessellator="gpu")
        assert np.array_equal(a.tet_v, b.tet_v)
        assert np.array_equal(a.tet_n, b.tet_n)
        assert np.array_equal(a.xyz, b.xyz)
