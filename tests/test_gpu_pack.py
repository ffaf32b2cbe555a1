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


def test_async_double_buffered_matches_sync(gpu_built):
    """Two handles used alternately with dtfe_gpu_interpolate_async (the
    double-buffered e2e loop) give the synchronous call's fields."""
    from dtfe_b200.device import DeviceDTFE
    pos, psi = S.zeldovich_lattice(16, 100.0, 1.0, seed=13)
    vel = (50 * psi).astype(np.float32)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), vel, None, grid=(16, 16, 16), n_threads=4)
    packed = P.pack_tets(plan.tet_v, plan.tet_n)
    G = int(np.prod(plan.grid))
    nc = {"density": 1, "velocity": 3, "velocity_gradient": 9, "velocity_divergence": 1}
    with DeviceDTFE(0) as ref_dev:
        ref_dev.load(plan)
        ref_dev.vertex_density(plan.rho_bar)
        ref = ref_dev.interpolate(FIELDS, method=0)
    devs = [DeviceDTFE(0), DeviceDTFE(0)]
    outs = [{f: np.full((G, nc[f]), np.nan, np.float32) for f in FIELDS} for _ in range(2)]
    try:
        for d in devs:
            d.upload_packed(plan, packed)
            d.set_subboxes(plan)
        devs[0].chain_uploads(devs[1])
        devs[1].chain_uploads(devs[0])
        for step in range(4):
            d = devs[step % 2]
            d.synchronize()
            d.upload_packed(plan, packed)
            d.vertex_density(plan.rho_bar)
            d.interpolate_async(FIELDS, outs[step % 2], method=0)
        for d in devs:
            d.synchronize()
        for o in outs:
            for f in FIELDS:
                assert np.array_equal(o[f].reshape(ref[f].shape), ref[f]), f
        assert devs[0].read_status()["n_samples_located"] == G
    finally:
        for d in devs:
            d.chain_uploads(None)
        for d in devs:
            d.close()


def test_packed_malformed_is_reported(gpu_built):
    """A packed buffer whose block sizes no longer add up (one flag byte
    changed) or whose header is not a packed tessellation is refused: the
    host rejects a bad header at upload, the device decoder's own bounds
    checks count the bad block and the next status read raises."""
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    pos, _ = S.zeldovich_lattice(12, 100.0, 1.0, seed=14)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(12, 12, 12), n_threads=2)
    packed = P.pack_tets(plan.tet_v, plan.tet_n)
    hd = packed[:80].view(np.int64)
    with DeviceDTFE(0) as dev:
        bad = packed.copy()
        bad[:8].view(np.int64)[0] = 0x31505444     # an older magic
        with pytest.raises(N.DTFEError):
            dev.upload_packed(plan, bad)
        bad = packed.copy()
        bad[int(hd[7]) + 3] ^= 0x01               # a flag byte of block 0: its bytes no longer add up
        dev.upload_packed(plan, bad)
        dev.set_subboxes(plan)
        dev.vertex_density(plan.rho_bar)
        with pytest.raises(N.DTFEError, match="did not decode"):
            dev.interpolate(["density"], method=0)
        # a good upload clears it
        dev.upload_packed(plan, packed)
        dev.vertex_density(plan.rho_bar)
        dev.interpolate(["density"], method=0)


def _plans():
    """A periodic multi-sub-box plan, a sparse non-periodic one (many hull
    faces, sub-boxes with few or no tetrahedra) and a single box around one
    vertex of very high degree (400 points on a jittered shell around it:
    its star holds far more faces than a per-vertex table, so the fallback
    search settles them)."""
    pos, psi = S.zeldovich_lattice(18, 100.0, 1.0, seed=15)
    vel = (40 * psi).astype(np.float32)
    a = P.make_plan(pos, np.ones(len(pos), np.float32), vel, None, grid=(18, 16, 20), n_threads=8)
    rng = np.random.default_rng(16)
    p2 = (rng.random((300, 3)) * 100).astype(np.float32)
    b = P.make_plan(p2, rng.uniform(0.5, 1.5, 300).astype(np.float32), rng.standard_normal((300, 3)).astype(
        np.float32), None, grid=(12, 12, 12), n_threads=6, periodic=False, padding=np.full(6, 4.0, np.float32),
        average_density_value=3e-4)
    rng = np.random.default_rng(17)
    d = rng.standard_normal((400, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    shell = 50.0 + d * (20.0 * (1.0 + 0.05 * rng.random((400, 1))))
    p3 = np.vstack([[[50.0, 50.0, 50.0]], shell, rng.random((200, 3)) * 100.0]).astype(np.float32)
    c = P.make_plan(p3, np.ones(len(p3), np.float32), rng.standard_normal((len(p3), 3)).astype(np.float32), None,
                    grid=(10, 10, 10), n_threads=1, periodic=False, padding=np.full(6, 2.0, np.float32),
                    average_density_value=1e-3)
    return [a, b, c]


@pytest.mark.parametrize("which", [0, 1, 2])
@pytest.mark.parametrize("form", ["plain_without_neighbours", "packed_vertices"])
def test_neighbours_derived_on_device(gpu_built, which, form):
    """Only the vertices cross (tet_n = NULL, or the vertex-only packed form
    of dtfe_tets_pack_vertices): the device's tet_v and its derived tet_n
    equal the host arrays exactly (-1 on the hull), and the fields equal
    those of the full upload bit for bit."""
    from dtfe_b200.device import DeviceDTFE
    plan = _plans()[which]
    with DeviceDTFE(0) as ref_dev:
        ref_dev.load(plan)
        ref_dev.vertex_density(plan.rho_bar)
        ref = ref_dev.interpolate(FIELDS, method=0)
        ref_d = ref_dev.download_vertex_density(plan.n_verts)
    with DeviceDTFE(0) as dev:
        if form == "plain_without_neighbours":
            dev.upload(plan, neighbours=False)
        else:
            dev.upload_packed(plan, P.pack_tet_vertices(plan.tet_v))
        tv, tn = dev.download_tets(plan.n_tets)
        assert np.array_equal(tv, plan.tet_v)
        assert np.array_equal(tn, plan.tet_n)
        dev.set_subboxes(plan)
        dev.vertex_density(plan.rho_bar)
        got = dev.interpolate(FIELDS, method=0)
        assert np.array_equal(dev.download_vertex_density(plan.n_verts), ref_d)
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f]), f


def test_packed_vertices_malformed_is_reported(gpu_built):
    """A vertex-only packed buffer with a wrong header is refused at upload;
    one whose block sizes no longer add up, or whose vertices leave the
    canonical order, is counted by the decoder's checks and reported by the
    next status read; a good upload clears it."""
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    pos, _ = S.zeldovich_lattice(12, 100.0, 1.0, seed=17)
    plan = P.make_plan(pos, np.ones(len(pos), np.float32), None, None, grid=(12, 12, 12), n_threads=2)
    packed = P.pack_tet_vertices(plan.tet_v)
    hd = packed[:80].view(np.int64)
    assert hd[0] == 0x33505444
    with DeviceDTFE(0) as dev:
        bad = packed.copy()
        bad[:80].view(np.int64)[9] = packed.nbytes + 16     # data beyond the buffer
        with pytest.raises(N.DTFEError):
            dev.upload_packed(plan, bad)
        for corrupt in ("flag", "data"):
            bad = packed.copy()
            if corrupt == "flag":
                bad[int(hd[7]) + 1] ^= 0x01      # a width nibble of block 0: its bytes no longer add up
            else:
                data = int(hd[9])
                bad[data + 1] = 0                # tetrahedron 0's second-vertex offset: 0, not above the first
            dev.upload_packed(plan, bad)
            dev.set_subboxes(plan)
            dev.vertex_density(plan.rho_bar)
            with pytest.raises(N.DTFEError, match="did not decode"):
                dev.interpolate(["density"], method=0)
        dev.upload_packed(plan, packed)
        dev.set_subboxes(plan)
        dev.vertex_density(plan.rho_bar)
        dev.interpolate(["density"], method=0)


@pytest.mark.parametrize("form", ["packed", "packed_vertices"])
def test_packed_particles_upload(gpu_built, form):
    """The input particles cross once with a code per vertex
    (dtfe_gpu_upload_packed_particles): the device rebuilds the padded,
    periodic vertex set exactly (positions, weights, velocities, scalars),
    so vertex densities and fields equal those of the per-vertex upload bit
    for bit; a code outside the particles is reported by the next status
    read and a good upload clears it."""
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    pos, psi = S.zeldovich_lattice(16, 100.0, 1.0, seed=18)
    rng = np.random.default_rng(19)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (40 * psi).astype(np.float32)
    sc = rng.standard_normal((len(pos), 2)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, sc, grid=(16, 14, 18), n_threads=8)
    codes, L = P.vertex_codes(plan, pos)
    assert (codes >> 27).max() > 13 and (codes >> 27).min() < 13  # images on both sides
    parts = {"pos": pos, "weight": w, "velocity": vel, "scalar": sc, "codes": codes, "box_length": L}
    packed = P.pack_tets(plan.tet_v, plan.tet_n) if form == "packed" else P.pack_tet_vertices(plan.tet_v)
    fields = FIELDS + ["scalar", "scalar_gradient"]
    with DeviceDTFE(0, 2) as ref_dev:
        ref_dev.load(plan)
        ref_dev.vertex_density(plan.rho_bar)
        ref = ref_dev.interpolate(fields, method=0)
        ref_d = ref_dev.download_vertex_density(plan.n_verts)
    with DeviceDTFE(0, 2) as dev:
        dev.upload_packed_particles(plan, packed, parts)
        dev.set_subboxes(plan)
        dev.vertex_density(plan.rho_bar)
        got = dev.interpolate(fields, method=0)
        assert np.array_equal(dev.download_vertex_density(plan.n_verts).view(np.int32), ref_d.view(np.int32))
        for f in fields:
            assert np.array_equal(got[f], ref[f]), f
        bad = dict(parts, codes=codes.copy())
        bad["codes"][7] = np.uint32(len(pos))              # a particle that does not exist
        dev.upload_packed_particles(plan, packed, bad)
        dev.vertex_density(plan.rho_bar)
        with pytest.raises(N.DTFEError, match="did not decode"):
            dev.interpolate(["density"], method=0)
        dev.upload_packed_particles(plan, packed, parts)
        dev.vertex_density(plan.rho_bar)
        again = dev.interpolate(["density"], method=0)
        assert np.array_equal(again["density"], ref["density"])
