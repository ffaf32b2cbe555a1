"""Host Delaunay tessellator: same tetrahedra as scipy's Qhull, consistent
neighbours, positive orientation, empty circumspheres, edge cases."""
import numpy as np
import pytest
from scipy.spatial import Delaunay

from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S


def _check_structure(pts, tv, tn):
    X = pts[tv]
    det = np.einsum("ij,ij->i", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]))
    assert (det > 0).all()
    T = len(tv)
    for k in range(4):
        u = tn[:, k]
        has = u >= 0
        # the neighbour across face k holds the 3 other vertices and points back
        back = (tn[u[has]] == np.flatnonzero(has)[:, None]).any(axis=1)
        assert back.all()
        face = np.delete(tv[has], k, axis=1)
        shared = (tv[u[has]][:, :, None] == face[:, None, :]).any(axis=1).sum(axis=1)
        assert (shared == 3).all()
    assert T > 0


def _same_as_qhull(pts, tv):
    D = Delaunay(pts)
    a = set(map(tuple, np.sort(tv, 1).tolist()))
    b = set(map(tuple, np.sort(D.simplices, 1).tolist()))
    return a == b


@pytest.mark.parametrize("n,seed", [(5, 0), (50, 1), (3000, 2)])
def test_random_points_match_qhull(built, n, seed):
    pts = np.random.default_rng(seed).random((n, 3)).astype(np.float32).astype(np.float64)
    (tv, tn, vm), = P.tessellate_many([pts])
    _check_structure(pts, tv, tn)
    assert _same_as_qhull(pts, tv)
    assert (vm == np.arange(n)).all()


def test_zeldovich_matches_qhull(built):
    pos, _ = S.zeldovich_lattice(16, 100.0, 0.5, 0)
    (tv, tn, _), = P.tessellate_many([pos])
    pts = pos.astype(np.float64)
    _check_structure(pts, tv, tn)
    assert _same_as_qhull(pts, tv)


def test_empty_circumspheres(built):
    pts = np.random.default_rng(5).random((800, 3))
    (tv, tn, _), = P.tessellate_many([pts])
    X = pts[tv]
    # circumcentres
    a = X[:, 0]
    A = np.stack([X[:, 1] - a, X[:, 2] - a, X[:, 3] - a], axis=1)
    rhs = 0.5 * np.einsum("tij,tij->ti", A, A)
    c = np.linalg.solve(A, rhs[..., None])[..., 0] + a
    r2 = np.sum((X[:, 0] - c) ** 2, axis=1)
    d2 = ((pts[None, :, :] - c[:, None, :]) ** 2).sum(-1)
    assert (d2 >= r2[:, None] * (1 - 1e-9)).all()


def test_hull_faces_and_volume(built):
    pts = np.random.default_rng(7).random((400, 3))
    (tv, tn, _), = P.tessellate_many([pts])
    from scipy.spatial import ConvexHull
    X = pts[tv]
    vol = np.abs(np.einsum("ij,ij->i", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]))).sum() / 6
    assert abs(vol - ConvexHull(pts).volume) < 1e-12
    assert (tn < 0).sum() == len(ConvexHull(pts).simplices)


def test_duplicates_and_degenerate(built):
    pts = np.random.default_rng(8).random((100, 3))
    dup = np.concatenate([pts, pts[:10]])
    (tv, tn, vm), = P.tessellate_many([dup])
    assert (vm[100:] == np.arange(10)).all()
    assert tv.max() < 100
    # fewer than 4 points / all coplanar: no tetrahedra, no crash
    (tv, tn, vm), = P.tessellate_many([np.random.default_rng(0).random((3, 3))])
    assert len(tv) == 0
    flat = np.random.default_rng(1).random((50, 3))
    flat[:, 2] = 0.5
    (tv, tn, vm), = P.tessellate_many([flat])
    assert len(tv) == 0


def test_cospherical_lattice(built):
    # a perfect cubic lattice: every cube is cospherical (maximally degenerate)
    g = np.arange(6, dtype=np.float64)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    (tv, tn, _), = P.tessellate_many([pts])
    _check_structure(pts, tv, tn)
    X = pts[tv]
    vol = np.einsum("ij,ij->i", X[:, 1] - X[:, 0], np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 0])).sum() / 6
    assert abs(vol - 125.0) < 1e-9
