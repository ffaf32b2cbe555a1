"""The DTFE() drop-in (dtfe_b200/shim) called as a reference caller calls
DTFE(): the reference's own Particle_data / User_options / Quantities types,
the reference's control flow with 4 OpenMP sub-boxes.  Its Quantities must
equal, bit for bit, the device API run on the same plan (the plan builders
are themselves pinned against the reference), and the reference's contract
holds: the particle vector is cleared, an automatic average density is
written back."""
import numpy as np
import pytest

import dropin as D

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not D.available(), reason="drop-in driver not built (needs the reference headers)")]

from dtfe_b200 import plan as P  # noqa: E402
from dtfe_b200 import synthetic as S  # noqa: E402

GRID = (12, 10, 14)
ALL = ["density", "velocity", "velocity_gradient", "velocity_divergence", "velocity_shear", "velocity_vorticity"]


@pytest.fixture(scope="module")
def particles(gpu_built):
    pos, psi = S.zeldovich_lattice(14, 100.0, 0.9, seed=8)
    rng = np.random.default_rng(9)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (25 * psi).astype(np.float32)
    sc = rng.standard_normal(len(pos)).astype(np.float32)
    return pos, w, vel, sc


def test_dropin_cell_centre_and_averages(particles):
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel, sc = particles
    u, a, avg, left = D.run("DTFE", pos, w, vel, sc, GRID, u_fields=ALL + ["scalar"],
                            a_fields=["density", "velocity"], method=3, n_points=8)
    assert left == 0
    assert avg == float(P.average_density(w))
    plan = P.make_plan(pos, w, vel, sc[:, None], grid=GRID, n_threads=4)
    with DeviceDTFE(0, 1) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        ref_u = dev.interpolate(ALL + ["scalar"], method=0)
        ref_a = dev.interpolate(["density", "velocity"], method=3, n_samples=8)
    for f in ALL + ["scalar"]:
        assert np.array_equal(u[f].reshape(ref_u[f].shape), ref_u[f]), f
    for f in ("density", "velocity"):
        assert np.array_equal(a[f].reshape(ref_a[f].shape), ref_a[f]), f


def test_dropin_monte_carlo_seeded(particles):
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel, _ = particles
    _, a, _, _ = D.run("DTFE", pos, w, vel, None, GRID, average_density=1e-3, a_fields=["density", "velocity_std"],
                       method=2, n_points=8, seed=17)
    plan = P.make_plan(pos, w, vel, None, grid=GRID, n_threads=4, average_density_value=1e-3)
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        ref = dev.interpolate(["density", "velocity_std"], method=2, n_samples=8, seed=17)
    for f in ("density", "velocity_std"):
        assert np.array_equal(a[f].reshape(ref[f].shape), ref[f]), f


@pytest.mark.parametrize("kind", ["NGP", "CIC", "TSC"])
def test_dropin_deposition(particles, kind):
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel, _ = particles
    _, a, _, _ = D.run(kind, pos, w, vel, None, GRID, a_fields=["density", "velocity"])
    dp = P.make_deposit_plan(pos, w, vel, grid=GRID, n_threads=4, kind=kind)
    with DeviceDTFE(0) as dev:
        ref = dev.deposit(dp)
    assert np.array_equal(a["density"][:, 0], ref["density"])
    assert np.array_equal(a["velocity"], ref["velocity"])


def test_dropin_sph(particles):
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel, _ = particles
    _, a, _, _ = D.run("SPH", pos, w, vel, None, GRID, a_fields=["density", "velocity"], sph_neighbors=32)
    plan = P.make_plan(pos, w, vel, None, grid=GRID, n_threads=4)
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        ref = dev.sph(plan.rho_bar, n_neighbors=32, velocity=True)
    assert np.array_equal(a["density"][:, 0], ref["density"])
    assert np.array_equal(a["velocity"], ref["velocity"])


def test_dropin_method1(particles):
    """The reference's default averaging (method 1, 100 points per cell)
    through DTFE(): the device API's method 1 on the same plan, bit for bit;
    no velocity standard deviation, as the reference."""
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel, sc = particles
    _, a, _, _ = D.run("DTFE", pos, w, vel, sc, GRID, a_fields=["density", "velocity", "velocity_gradient", "scalar"],
                       method=1, n_points=100)
    plan = P.make_plan(pos, w, vel, sc[:, None], grid=GRID, n_threads=4)
    with DeviceDTFE(0, 1) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        ref = dev.interpolate(["density", "velocity", "velocity_gradient", "scalar"], method=N.METHOD_TETRAHEDRA,
                              n_samples=100)
    for f in ("density", "velocity", "velocity_gradient", "scalar"):
        assert np.array_equal(a[f].reshape(ref[f].shape), ref[f]), f


def test_dropin_user_sampling(particles):
    """DTFE() with user sampling points (the samples vector): the samples
    inside the box, in order, equal the device API's user-point interpolation
    on the reference's single-box plan."""
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel, sc = particles
    rng = np.random.default_rng(11)
    samples = rng.uniform(-10, 110, (3000, 3)).astype(np.float32)
    fields = ["density", "velocity", "velocity_gradient", "velocity_divergence", "scalar"]
    u = D.run_points(pos, w, vel, sc, GRID, samples, u_fields=fields)
    plan = P.make_plan(pos, w, vel, sc[:, None], grid=GRID, n_threads=1)
    with DeviceDTFE(0, 1) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        ref = dev.interpolate_points(fields, samples, [0, 100, 0, 100, 0, 100])
    for f in fields:
        assert len(u[f]) == len(ref[f]) < len(samples)
        assert np.array_equal(u[f].reshape(ref[f].shape), ref[f]), f


def test_dropin_redshift_cone(particles):
    """DTFE() on a redshift-cone grid (redshiftConeOn): the gridSize bins in
    (r, theta, psi), equal to the oracle's interpolateRedshiftCone on the
    reference's single-box plan, bit for bit, shells beyond the padded hull
    included."""
    import oracle as O
    pos, w, vel, sc = particles
    fields = ["density", "velocity", "velocity_gradient", "velocity_divergence", "scalar"]
    cone, origin = (2.0, 110.0, 5.0, 175.0, 200.0, 100.0), (50.0, 40.0, 60.0)
    u = D.run_cone(pos, w, vel, sc, GRID, cone, origin, u_fields=fields)
    plan = P.make_plan(pos, w, vel, sc[:, None], grid=GRID, n_threads=1)
    d32, d64, _ = O.vertex_density(plan)
    ref = O.interpolate_cone(plan, d32, d64, fields, cone, origin, GRID, mode=O.MODE_REF)
    for f in fields:
        assert np.array_equal(u[f].reshape(ref[f].shape), ref[f].astype(np.float32)), f
    assert (ref["density"] == 0).any() and (ref["density"] != 0).any()


def test_dropin_averages_at_samples_and_cones(particles):
    """DTFE() with aField at user sampling points and on a redshift cone: the
    reference's forced Monte-Carlo averages (method 2, 20 points unless
    noPointsOn), equal to the device API's dtfe_gpu_average_points /
    Monte-Carlo cone on the single-box plan with the same seed."""
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel, sc = particles
    rng = np.random.default_rng(12)
    samples = rng.uniform(-10, 110, (1500, 3)).astype(np.float32)
    delta = rng.uniform(1, 9, (1500, 3)).astype(np.float32)
    fields = ["density", "velocity", "velocity_gradient", "scalar"]
    cone, origin = (2.0, 80.0, 5.0, 175.0, 0.0, 300.0), (50.0, 40.0, 60.0)
    u, a = D.run_points(pos, w, vel, sc, GRID, samples, u_fields=["density"], a_fields=fields, delta=delta, seed=9)
    _, ac = D.run_cone(pos, w, vel, sc, GRID, cone, origin, u_fields=["density"], a_fields=fields, n_points=6,
                       seed=4)
    plan = P.make_plan(pos, w, vel, sc[:, None], grid=GRID, n_threads=1)
    with DeviceDTFE(0, 1) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        ref = dev.average_points(fields, samples, delta, [0, 100, 0, 100, 0, 100], 20, seed=9)
        refc = dev.interpolate_cone(fields, cone, origin, GRID, n_samples=6, seed=4)
    for f in fields:
        assert len(a[f]) == len(ref[f]) == len(u["density"]) < len(samples)
        assert np.array_equal(a[f].reshape(ref[f].shape), ref[f]), f
        assert np.array_equal(ac[f].reshape(refc[f].shape), refc[f]), f


PLANNING = {
    "region_fractions": dict(region=(0.2, 0.7, 0.1, 0.6, 0.3, 0.9)),
    "region_absolute": dict(region=(10.0, 60.0, 20.0, 75.0, 5.0, 55.0), region_mpc=True),
    "partition_all": dict(partition=(2, 1, 2)),
    "partition_one": dict(partition=(2, 2, 1), part_no=3),
    "padding_relative": dict(padding=(0.05, 0.06, 0.07, 0.05, 0.04, 0.08), padding_mode=1),
    "padding_absolute": dict(padding=(6.0, 5.0, 7.0, 6.0, 5.0, 8.0), padding_mode=2),
    "region_partition_one": dict(region=(0.1, 0.8, 0.2, 0.9, 0.0, 0.7), partition=(2, 2, 2), part_no=5),
}


@pytest.mark.parametrize("case", list(PLANNING))
def test_dropin_planning_options(particles, case):
    """--region, --partition (every chunk in one batched step, or one
    --partNo chunk on its own grid) and given padding lengths through
    DTFE(): the device API on the planner's plan for the same options, bit for
    bit, and the reference's own DTFE() (its src/DTFE.cpp in the harness) on
    the same call: the same grid and region, fields within 2e-6 (RMS floor)
    — its vertex densities are float sums of float volumes, the GPU's exact
    sums of FP64 volumes, a few 1e-7 apart on this input."""
    from conftest import rel_err
    from dtfe_b200.device import DeviceDTFE
    if not D.available("reference"):
        pytest.skip("the reference's DTFE() is not built")
    pos, w, vel, _ = particles
    opts = PLANNING[case]
    avg = float(w.sum()) / 1e6
    fields = ["density", "velocity", "velocity_gradient", "velocity_divergence"]
    kw = dict(average_density=avg, u_fields=fields, a_fields=["density"], method=3, n_points=8, n_threads=4, **opts)
    u, a, reg = D.run_ex("DTFE", pos, w, vel, None, GRID, which="dropin", **kw)
    ur, ar, regr = D.run_ex("DTFE", pos, w, vel, None, GRID, which="reference", **kw)
    assert np.array_equal(reg, regr)
    pk = {}
    if "region" in opts:
        r = np.asarray(opts["region"], np.float32)
        pk["region"] = r if opts.get("region_mpc") else np.float32(100.0) * r
    if "partition" in opts:
        pk["partition"] = opts["partition"]
        pk["part_no"] = opts.get("part_no", -1)
    if "padding" in opts:
        pk["padding"] = opts["padding"]
        pk["padding_absolute"] = opts.get("padding_mode", 1) == 2
    plan = P.native_plan("DTFE", pos, w, vel, None, grid=GRID, n_threads=4, average_density_value=avg, **pk)
    assert np.array_equal(plan.covered_region, reg)
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        ref_u = dev.interpolate(fields, method=0)
        ref_a = dev.interpolate(["density"], method=3, n_samples=8)
    assert len(u["density"]) == len(ur["density"]) == int(np.prod(plan.grid))
    for f in fields:
        assert np.array_equal(u[f].reshape(ref_u[f].shape), ref_u[f]), f
        assert rel_err(u[f], ur[f]) <= 2e-6, (f, rel_err(u[f], ur[f]))
    assert np.array_equal(a["density"].reshape(ref_a["density"].shape), ref_a["density"])
    assert rel_err(a["density"], ar["density"]) <= 2e-6
