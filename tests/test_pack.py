"""Packed tessellation (dtfe_tets_pack / dtfe_tets_unpack) round trips."""
import numpy as np

from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S


def test_pack_roundtrip_plan(built):
    pos, _ = S.zeldovich_lattice(16, 100.0, 1.0, seed=2)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(16, 16, 16), n_threads=4)
    packed = P.pack_tets(plan.tet_v, plan.tet_n)
    assert packed.nbytes < 0.6 * (plan.tet_v.nbytes + plan.tet_n.nbytes)
    tv, tn = P.unpack_tets(packed, plan.n_tets)
    assert np.array_equal(tv, plan.tet_v) and np.array_equal(tn, plan.tet_n)


def test_pack_roundtrip_escapes(built):
    rng = np.random.default_rng(0)
    T = 1000
    tv = np.sort(rng.integers(0, 2_000_000_000, (T, 4)), axis=1).astype(np.int32)
    tv[::7] = tv[::7, ::-1]          # not smallest-first: escaped offsets
    tn = rng.integers(-1, T, (T, 4)).astype(np.int32)
    tn[::3, 0] = 2_000_000_000       # far neighbours
    tn[5] = -1
    packed = P.pack_tets(tv, tn)
    a, b = P.unpack_tets(packed, T)
    assert np.array_equal(a, tv) and np.array_equal(b, tn)
    e = P.pack_tets(np.zeros((0, 4), np.int32), np.zeros((0, 4), np.int32))
    a, b = P.unpack_tets(e, 0)
    assert a.shape == (0, 4)
