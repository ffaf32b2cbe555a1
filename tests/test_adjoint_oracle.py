"""The FP64 adjoint oracle against central finite differences (CPU).

Pins the analytic gradients that the GPU adjoints are compared with: the
DTFE density / velocity / divergence loss (oracle_dtfe_grad), its local
finite-difference routine (oracle_dtfe_fd, checked against differences of
the full loss) and the NGP / CIC / TSC deposition loss.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from dtfe_b200 import plan as P
from dtfe_b200 import synthetic as S


def _problem(n=8, full=False, seed=3):
    pos, psi = S.zeldovich_lattice(n, 100.0, 0.5, seed=seed)
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (100.0 * psi / (100.0 / n) + rng.normal(0, 50, psi.shape)).astype(np.float32)
    plan = P.make_plan(pos, w, vel, None, grid=(n, n, n), n_threads=1, padding_particles=2.0,
                       average_density_value=float(w.sum()) / 1e6)
    d32, d64, _ = O.vertex_density(plan)
    _, loc = O.interpolate(plan, d32, d64, ["density"], mode=O.MODE_FP64, want_loc=True)
    G = int(np.prod(plan.grid))
    a = rng.standard_normal(G)
    c = rng.standard_normal((G, 3))
    b = rng.standard_normal(G)
    prob = O.AdjointProblem(plan, loc, a=a, c=c, b=b, full_value=full)
    return plan, prob, len(pos)


def _per_particle(src, g, n):
    out = np.zeros((n,) + g.shape[1:])
    np.add.at(out, src, g)
    return out


@pytest.mark.parametrize("full", [False, True])
def test_dtfe_grad_matches_full_fd(built, full):
    plan, prob, n = _problem(full=full)
    x = plan.xyz.astype(np.float64)
    w = plan.weight.astype(np.float64)
    v = plan.velocity.astype(np.float64)
    gx, gv, gw = prob.grad(x, w, v)
    px = _per_particle(plan.src, gx, n)
    pv = _per_particle(plan.src, gv, n)
    pw = _per_particle(plan.src, gw, n)
    rng = np.random.default_rng(5)
    h = 1e-6 * 100.0
    for i in rng.choice(n, 6, replace=False):
        m = plan.src == i
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[m, k] += h
            xm[m, k] -= h
            fd = (prob.loss(xp, w, v) - prob.loss(xm, w, v)) / (2 * h)
            assert abs(fd - px[i, k]) <= 1e-6 * max(1.0, abs(px[i, k])) + 1e-6 * np.abs(px).max()
            vp, vm = v.copy(), v.copy()
            vp[m, k] += 1e-3
            vm[m, k] -= 1e-3
            fdv = (prob.loss(x, w, vp) - prob.loss(x, w, vm)) / 2e-3
            assert abs(fdv - pv[i, k]) <= 1e-7 * max(1.0, np.abs(pv).max())
        wp, wm = w.copy(), w.copy()
        wp[m] += 1e-4
        wm[m] -= 1e-4
        fdw = (prob.loss(x, wp, v) - prob.loss(x, wm, v)) / 2e-4
        assert abs(fdw - pw[i]) <= 1e-7 * max(1.0, np.abs(pw).max())


def test_local_fd_matches_analytic(built):
    plan, prob, n = _problem(n=10, full=False, seed=9)
    x = plan.xyz.astype(np.float64)
    w = plan.weight.astype(np.float64)
    v = plan.velocity.astype(np.float64)
    gx, gv, gw = prob.grad(x, w, v)
    sel = np.random.default_rng(1).choice(n, 60, replace=False)
    fd = O.dtfe_fd(prob, x, w, v, sel, h_pos=1e-4)
    an = np.concatenate([_per_particle(plan.src, gx, n)[sel], _per_particle(plan.src, gv, n)[sel],
                         _per_particle(plan.src, gw, n)[sel, None]], axis=1)
    for cols in (slice(0, 3), slice(3, 6), slice(6, 7)):
        assert rel_err(fd[:, cols], an[:, cols]) < 1e-6


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_deposit_grad_matches_fd(built, kind):
    rng = np.random.default_rng(kind)
    region = np.array([10, 90, 5, 95, 0, 100], np.float32)
    grid = np.array([8, 9, 10], np.int32)
    # particles inside, on the clipped boundary layers and outside the region
    pos = rng.uniform(-5, 105, (400, 3))
    w = rng.uniform(0.5, 1.5, 400)
    a = rng.standard_normal(int(np.prod(grid)))
    L, gx, gw = O.deposit_loss_grad(kind, pos, w, region, grid, 1e-6, a)
    h = 1e-4
    fdx = np.zeros_like(gx)
    for k in range(3):
        for s in (1, -1):
            p = pos.copy()
            p[:, k] += s * h
            # per particle: the loss is a sum of independent particle terms
            for i in range(len(pos)):
                Li, _, _ = O.deposit_loss_grad(kind, p[i:i + 1], w[i:i + 1], region, grid, 1e-6, a, False)
                fdx[i, k] += s * Li / (2 * h)
    assert rel_err(fdx, gx) < 1e-5
    fdw = np.array([O.deposit_loss_grad(kind, pos[i:i + 1], np.ones(1), region, grid, 1e-6, a, False)[0]
                    for i in range(len(pos))])
    assert rel_err(fdw, gw) < 1e-9
    assert abs(L - float((w * fdw).sum())) <= 1e-9 * max(1.0, abs(L))
