"""The Sobol generator behind averaging method 1 (dtfe_b200/csrc/sobol.h, the
Bratley-Fox construction GSL's gsl_qrng_sobol implements): known points,
exact dyadic values, the simplex filter of quasiRandomSequence
(averaged_interpolation_1.cc:32-50)."""
import numpy as np

import oracle as O


def test_first_points_two_dimensions():
    # first points of the Bratley-Fox sequence in its first two dimensions
    # (van der Corput, then x + 1), Gray-code order, origin skipped
    want = [(0.5, 0.5), (0.75, 0.25), (0.25, 0.75), (0.375, 0.375), (0.875, 0.875), (0.625, 0.125),
            (0.125, 0.625)]
    pts = _unfiltered(64)
    for i, (a, b) in enumerate(want):
        assert pts[i, 0] == a and pts[i, 1] == b, i
    # each coordinate's first 2^k - 1 points are the nonzero multiples of 2^-k
    for k in (3, 4, 5, 6):
        n = 2 ** k - 1
        for d in range(3):
            vals = np.sort(pts[:n, d] * 2 ** k)
            assert np.array_equal(vals, np.arange(1, 2 ** k)), (k, d)


def _unfiltered(n):
    """First n points of the sequence, without the simplex filter, from the
    same direction-number recurrences in Python integers."""
    m = np.zeros((3, 30), np.uint64)
    m[0, :] = 1
    m[1, 0] = 1
    for j in range(1, 30):
        m[1, j] = (m[1, j - 1] << np.uint64(1)) ^ m[1, j - 1]
    m[2, 0] = m[2, 1] = 1
    for j in range(2, 30):
        m[2, j] = (m[2, j - 1] << np.uint64(1)) ^ (m[2, j - 2] << np.uint64(2)) ^ m[2, j - 2]
    v = np.array([[int(m[d, j]) << (29 - j) for j in range(30)] for d in range(3)], dtype=object)
    num = [0, 0, 0]
    out = np.zeros((n, 3))
    for k in range(n):
        c = 0
        x = k
        while x & 1:
            c += 1
            x >>= 1
        for d in range(3):
            num[d] ^= v[d][c]
            out[k, d] = num[d] / float(1 << 30)
    return out


def test_simplex_table_matches_filter():
    pts = _unfiltered(4000)
    keep = pts[(pts.astype(np.float64).sum(1).astype(np.float32) <= 1.0)]
    tab = O.sobol_simplex(len(keep))
    assert np.array_equal(tab, keep.astype(np.float32))
    assert (tab.astype(np.float64).sum(1) <= 1.0 + 1e-7).all() and (tab >= 0).all()
