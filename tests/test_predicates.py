"""Exact orientation / in-sphere predicates against rational arithmetic."""
from fractions import Fraction

import numpy as np
import pytest

from dtfe_b200 import _native as N


def _det3(r):
    return (r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1])
            - r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0])
            + r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]))


def orient_q(a, b, c, d):
    A = [Fraction(x) for x in a]
    rows = [[Fraction(p[k]) - A[k] for k in range(3)] for p in (b, c, d)]
    v = _det3(rows)
    return (v > 0) - (v < 0)


def insphere_q(a, b, c, d, e):
    E = [Fraction(x) for x in e]
    rows = []
    for p in (a, b, c, d):
        r = [Fraction(p[k]) - E[k] for k in range(3)]
        rows.append(r + [r[0] * r[0] + r[1] * r[1] + r[2] * r[2]])
    # 4x4 determinant by cofactor expansion along the last column
    det = Fraction(0)
    for i in range(4):
        minor = [rows[j][:3] for j in range(4) if j != i]
        det += (-1) ** (i + 3) * rows[i][3] * _det3(minor)
    v = -det  # positive inside for positively oriented (a,b,c,d)
    return (v > 0) - (v < 0)


def _arr(p):
    return np.ascontiguousarray(p, np.float64)


def _cases(rng, n):
    out = []
    for _ in range(n):
        kind = rng.integers(0, 4)
        a, b, c = rng.random((3, 3))
        if kind == 0:
            d = rng.random(3)
        elif kind == 1:  # exactly coplanar (small integers)
            a, b, c = rng.integers(-4, 5, (3, 3)).astype(float)
            s, t = rng.integers(-3, 4, 2)
            d = a + s * (b - a) + t * (c - a)
        elif kind == 2:  # nearly coplanar
            s, t = rng.random(2)
            d = a + s * (b - a) + t * (c - a) + rng.normal(0, 1e-15, 3)
        else:  # tiny and huge magnitudes mixed
            d = rng.random(3) * 1e-9 + np.array([1e-12, 0, 0])
        out.append((a, b, c, d))
    return out


def test_orient_matches_rational(built):
    lib = N.host()
    rng = np.random.default_rng(0)
    for a, b, c, d in _cases(rng, 400):
        q = orient_q(a, b, c, d)
        pa, pb, pc, pd = map(_arr, (a, b, c, d))
        assert lib.dtfe_orient(pa.ctypes.data, pb.ctypes.data, pc.ctypes.data, pd.ctypes.data) == q
        assert lib.dtfe_orient_exact(pa.ctypes.data, pb.ctypes.data, pc.ctypes.data, pd.ctypes.data) == q


def test_insphere_matches_rational(built):
    lib = N.host()
    rng = np.random.default_rng(1)
    n_zero = 0
    for i in range(300):
        # integer points: cospherical configurations occur exactly
        P = rng.integers(-3, 4, (5, 3)).astype(float)
        if i % 3 == 0:
            P = rng.random((5, 3))
        if orient_q(*P[:4]) == 0:
            continue
        if orient_q(*P[:4]) < 0:
            P[[2, 3]] = P[[3, 2]]
        q = insphere_q(*P)
        n_zero += q == 0
        ps = [_arr(p) for p in P]
        assert lib.dtfe_insphere(*[p.ctypes.data for p in ps]) == q
        assert lib.dtfe_insphere_exact(*[p.ctypes.data for p in ps]) == q
    assert n_zero > 0  # the exact zero branch was exercised


def test_insphere_sign_convention(built):
    lib = N.host()
    P = [_arr(p) for p in ([0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1])]
    assert lib.dtfe_orient(*[p.ctypes.data for p in P]) == 1
    inside = _arr([0.25, 0.25, 0.25])
    outside = _arr([2.0, 2.0, 2.0])
    assert lib.dtfe_insphere(*[p.ctypes.data for p in P], inside.ctypes.data) == 1
    assert lib.dtfe_insphere(*[p.ctypes.data for p in P], outside.ctypes.data) == -1
