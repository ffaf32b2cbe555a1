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
