"""Packed tessellation (dtfe_tets_pack / dtfe_tets_unpack) round trips."""
import numpy as np
import pytest

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


def test_pack_layout_header(built):
    """The header's offsets are 16-byte aligned and in order, the format the
    device decoder checks before a packed upload."""
    pos, _ = S.zeldovich_lattice(10, 100.0, 1.0, seed=4)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(10, 10, 10), n_threads=2)
    packed = P.pack_tets(plan.tet_v, plan.tet_n)
    hd = packed[:80].view(np.int64)
    T, nb, ne = int(hd[1]), int(hd[2]), int(hd[3])
    assert hd[0] == 0x32505444 and T == plan.n_tets and nb == (T + 255) // 256
    off = [int(x) for x in hd[4:10]]
    assert all(o % 16 == 0 for o in off) and off == sorted(off)
    assert off[-1] + 4 * ne <= packed.nbytes
    flags = packed[off[3]:off[3] + T]
    boff = packed[off[2]:off[2] + 8 * (nb + 1)].view(np.int64)
    sizes = 8 + np.unpackbits(flags[:, None], axis=1).sum(1)
    per_block = np.add.reduceat(sizes, np.arange(0, T, 256))
    assert np.array_equal(np.diff(boff), per_block)


def test_pack_vertices_roundtrip(built):
    """The vertex-only form (dtfe_tets_pack_vertices): tet_v restored bit for
    bit, well under a fifth of the 32 bytes per tetrahedron of the plain
    arrays."""
    pos, _ = S.zeldovich_lattice(16, 100.0, 1.0, seed=2)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(16, 16, 16), n_threads=4)
    packed = P.pack_tet_vertices(plan.tet_v)
    assert packed.nbytes < 0.2 * (plan.tet_v.nbytes + plan.tet_n.nbytes)
    assert np.array_equal(P.unpack_tet_vertices(packed, plan.n_tets), plan.tet_v)


def test_pack_vertices_escapes_and_order(built):
    """Far jumps between consecutive tetrahedra and large offsets escape to
    32 bits; tetrahedra not in the canonical vertex order are refused."""
    rng = np.random.default_rng(1)
    T = 3000
    tv = np.empty((T, 4), np.int64)
    tv[:, 0] = rng.integers(0, 1_000_000_000, T)
    tv[:, 1] = tv[:, 0] + rng.integers(1, 100_000, T)
    lo = tv[:, 1] + rng.integers(1, 300, T)
    hi = lo + rng.integers(1, 70_000, T)
    swap = rng.random(T) < 0.5
    tv[:, 2] = np.where(swap, hi, lo)
    tv[:, 3] = np.where(swap, lo, hi)
    tv = tv.astype(np.int32)
    packed = P.pack_tet_vertices(tv)
    assert np.array_equal(P.unpack_tet_vertices(packed, T), tv)
    e = P.pack_tet_vertices(np.zeros((0, 4), np.int32))
    assert P.unpack_tet_vertices(e, 0).shape == (0, 4)
    bad = tv.copy()
    bad[7] = bad[7, ::-1]
    import pytest
    with pytest.raises(ValueError):
        P.pack_tet_vertices(bad)


def test_vertex_codes_rebuild_the_padded_vertices():
    """plan.vertex_codes: each vertex is its source particle shifted by the
    coded periodic image in float32, exactly the position the planner
    selected; images on both sides of the box occur, and an unrelated
    position is refused."""
    import numpy as np
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    pos, psi = S.zeldovich_lattice(14, 100.0, 1.0, seed=40)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(14, 14, 14), n_threads=4)
    codes, L = P.vertex_codes(plan, pos)
    src = codes & np.uint32((1 << 27) - 1)
    img = codes >> np.uint32(27)
    assert np.array_equal(src, plan.src.astype(np.uint32))
    i = np.stack([img // 9, (img // 3) % 3, img % 3], axis=1).astype(np.float32) - np.float32(1)
    rebuilt = (pos[src] - i * L).astype(np.float32)
    assert np.array_equal(rebuilt, plan.xyz)
    assert img.min() < 13 < img.max()
    bad = plan.xyz.copy()
    plan.xyz[5, 0] += np.float32(0.5)
    try:
        with pytest.raises(ValueError):
            P.vertex_codes(plan, pos)
    finally:
        plan.xyz[...] = bad


def test_vertex_codes_non_periodic():
    """Without periodic images every vertex is its particle unshifted
    (image 13), and the codes index the particle arrays directly."""
    import numpy as np
    from dtfe_b200 import plan as P
    rng = np.random.default_rng(41)
    pos = (rng.random((2000, 3)) * 100.0).astype(np.float32)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(10, 10, 10), n_threads=4,
                       periodic=False, padding=np.full(6, 3.0, np.float32), average_density_value=2e-3)
    codes, L = P.vertex_codes(plan, pos)
    assert np.all((codes >> np.uint32(27)) == 13)
    src = codes & np.uint32((1 << 27) - 1)
    assert np.array_equal(pos[src], plan.xyz)


def test_plan_rejects_unknown_tessellator():
    """make_plan's tessellator is "host" (default) or "gpu"."""
    from dtfe_b200 import plan as P
    from dtfe_b200 import synthetic as S
    pos, _ = S.zeldovich_lattice(8, 100.0, 1.0, seed=3)
    with pytest.raises(ValueError):
        P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(8, 8, 8), n_threads=2,
                    tessellator="qhull")
