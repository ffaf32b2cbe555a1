"""The planning options of DTFE() against the reference's own DTFE().

The reference's src/DTFE.cpp (DTFE(), DTFE_parallel(), the user_options.cc it
includes) is compiled in the harness (oracle/_ref/libdtfe_refmain.so, CPU) and
run through the same test driver as the drop-in.  For --region (box fractions
and absolute), --partition over every chunk, --partition with --partNo, and
given padding lengths (--padding l1..l6 in box lengths, --paddingMpc), this
project's planner (dtfe_plan_build_ex) followed by the oracle in the
reference's arithmetic (its float vertex-density sums included) must give the
same grid, the same covered region and the same fields, bit for bit.  The
harness's CGAL facade numbers a sub-box's points in the planner's order, so
the reference sees the planner's tessellation of every sub-box.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S

import dropin

pytestmark = pytest.mark.skipif(not dropin.available("reference"),
                                reason="reference tree not available (harness not built)")

FIELDS = ["density", "velocity", "velocity_gradient", "velocity_divergence"]
GRID = (12, 10, 14)
BOX = (0.0, 100.0, 0.0, 100.0, 0.0, 100.0)

CASES = {
    "plain": dict(),
    "region_fractions": dict(region=(0.2, 0.7, 0.1, 0.6, 0.3, 0.9)),
    "region_absolute": dict(region=(10.0, 60.0, 20.0, 75.0, 5.0, 55.0), region_mpc=True),
    "partition_all": dict(partition=(2, 1, 2)),
    "partition_one": dict(partition=(2, 2, 1), part_no=3),
    "padding_relative": dict(padding=(0.05, 0.06, 0.07, 0.05, 0.04, 0.08), padding_mode=1),
    "padding_absolute": dict(padding=(6.0, 5.0, 7.0, 6.0, 5.0, 8.0), padding_mode=2),
    "region_partition_one": dict(region=(0.1, 0.8, 0.2, 0.9, 0.0, 0.7), partition=(2, 2, 2), part_no=5),
}


def _inputs(n=14, seed=11):
    pos, psi = S.zeldovich_lattice(n, 100.0, 0.8, seed=seed)
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (30 * psi + rng.normal(0, 5, psi.shape)).astype(np.float32)
    return pos, w, vel


def _absolute_region(region, mpc):
    """User_options::updateEntries' conversion of box fractions, with its
    [i % 2] indexing of the box offset and length (src/user_options.cc:952-958)."""
    r = np.asarray(region, np.float32)
    if mpc:
        return r
    off = np.array([BOX[0], BOX[2], BOX[4]], np.float32)
    ln = np.array([BOX[1] - BOX[0], BOX[3] - BOX[2], BOX[5] - BOX[4]], np.float32)
    return np.array([off[i % 2] + r[i] * ln[i % 2] for i in range(6)], np.float32)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("periodic", [True, False])
def test_reference_dtfe_flow(built, case, periodic):
    opts = CASES[case]
    if not periodic and "region" not in opts and "padding" not in opts and case != "plain":
        pytest.skip("covered by the periodic run")
    pos, w, vel = _inputs()
    avg = float(w.sum()) / 1e6
    u, _, reg = dropin.run_ex("DTFE", pos, w, vel, None, GRID, box=BOX, periodic=periodic, average_density=avg,
                              u_fields=FIELDS, n_threads=4, which="reference", **opts)
    kw = {}
    if "region" in opts:
        kw["region"] = _absolute_region(opts["region"], opts.get("region_mpc", False))
    if "partition" in opts:
        kw["partition"] = opts["partition"]
        kw["part_no"] = opts.get("part_no", -1)
    if "padding" in opts:
        kw["padding"] = opts["padding"]
        kw["padding_absolute"] = opts.get("padding_mode", 1) == 2
    plan = P.native_plan("DTFE", pos, w, vel, None, grid=GRID, box=BOX, periodic=periodic, n_threads=4,
                         average_density_value=avg, **kw)
    assert np.array_equal(reg, plan.covered_region), (reg, plan.covered_region)
    G = int(np.prod(plan.grid))
    assert len(u["density"]) == G
    dref = O.vertex_density_ref(plan)
    want, _ = O.interpolate(plan, dref, dref.astype(np.float64), FIELDS, mode=O.MODE_REF)
    for f in FIELDS:
        got = u[f].reshape(want[f].shape)
        assert np.array_equal(got, want[f].astype(np.float32)), (case, f, rel_err(got, want[f]))


def test_region_outside_box_refused(built):
    """A non-periodic region outside the box is refused by the planner
    (Box::validSubBox, src/box.h:115-138, where the reference exits the
    process)."""
    pos, w, vel = _inputs()
    with pytest.raises(RuntimeError):
        P.native_plan("DTFE", pos, w, vel, None, grid=GRID, box=BOX, periodic=False, n_threads=2,
                      region=(-10.0, 50.0, 0.0, 50.0, 0.0, 50.0))
