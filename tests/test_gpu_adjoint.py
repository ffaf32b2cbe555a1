"""GPU adjoints against the FP64 oracle gradients and finite differences.

dtfe_gpu_adjoint_dev (density, velocity, divergence grids -> vertex
positions, velocities, weights) and dtfe_gpu_deposit_adjoint_dev (CIC / TSC
density -> particle positions, weights), directly through the C ABI and
through the torch.autograd wrappers.  Tolerance: 1e-5 relative (RMS floor)
against the oracle's analytic FP64 gradient, which is itself pinned against
central differences on the CPU; 1e-4 against the FP64 central differences
(h = 1e-6 box) evaluated here.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from dtfe_b200 import plan as P  # noqa: E402
from dtfe_b200 import synthetic as S  # noqa: E402


def _particles(n, seed, disp=0.5):
    pos, psi = S.zeldovich_lattice(n, 100.0, disp, seed=seed)
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.5, 1.5, len(pos)).astype(np.float32)
    vel = (100.0 * psi / (100.0 / n) + rng.normal(0, 50, psi.shape)).astype(np.float32)
    return pos, w, vel


def _per_particle(src, g, n):
    out = np.zeros((n,) + g.shape[1:])
    np.add.at(out, src, g)
    return out


@pytest.mark.parametrize("n,threads,full", [(12, 1, False), (16, 4, True), (16, 8, False)])
def test_adjoint_matches_oracle(gpu_built, n, threads, full):
    from dtfe_b200.device import DeviceDTFE
    pos, w, vel = _particles(n, 21 + n)
    plan = P.make_plan(pos, w, vel, None, grid=(n, n, n), n_threads=threads, padding_particles=3.0,
                       average_density_value=float(w.sum()) / 1e6)
    G = int(np.prod(plan.grid))
    V = plan.n_verts
    rng = np.random.default_rng(n)
    a, c, b = rng.standard_normal(G), rng.standard_normal((G, 3)), rng.standard_normal(G)
    cuda = torch.device("cuda", 0)
    ta, tc, tb = (torch.tensor(t, dtype=torch.float32, device=cuda) for t in (a, c, b))
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        dens = torch.empty(G, device=cuda)
        vg = torch.empty((G, 3), device=cuda)
        div = torch.empty(G, device=cuda)
        dev.interpolate_dev(["density", "velocity", "velocity_divergence"], {"density": dens, "velocity": vg,
                                                                    "velocity_divergence": div}, fix=full)
        gx = torch.empty((V, 3), device=cuda)
        gv = torch.empty((V, 3), device=cuda)
        gw = torch.empty(V, device=cuda)
        dev.adjoint_dev(gx, grad_density=ta, grad_velocity=tc, grad_divergence=tb, grad_vel=gv, grad_w=gw)
        torch.cuda.synchronize()
    d32, d64, _ = O.vertex_density(plan)
    _, loc = O.interpolate(plan, d32, d64, ["density"], mode=O.MODE_FP64, want_loc=True)
    prob = O.AdjointProblem(plan, loc, a=a, c=c, b=b, full_value=full)
    x64, w64, v64 = plan.xyz.astype(np.float64), plan.weight.astype(np.float64), plan.velocity.astype(np.float64)
    ox, ov, ow = prob.grad(x64, w64, v64)
    assert rel_err(gx.cpu().numpy(), ox) < 1e-5
    assert rel_err(gv.cpu().numpy(), ov) < 1e-5
    assert rel_err(gw.cpu().numpy(), ow) < 1e-5
    # and against FP64 central differences for 200 particles (all images moved)
    sel = rng.choice(len(pos), 200, replace=False)
    fd = O.dtfe_fd(prob, x64, w64, v64, sel, h_pos=1e-6 * 100.0)
    px = _per_particle(plan.src, gx.cpu().numpy().astype(np.float64), len(pos))[sel]
    pv = _per_particle(plan.src, gv.cpu().numpy().astype(np.float64), len(pos))[sel]
    pw = _per_particle(plan.src, gw.cpu().numpy().astype(np.float64), len(pos))[sel]
    assert rel_err(px, fd[:, :3]) < 1e-4
    assert rel_err(pv, fd[:, 3:6]) < 1e-4
    assert rel_err(pw, fd[:, 6]) < 1e-4


def test_autograd_dtfe(gpu_built):
    from dtfe_b200.autograd import DTFEGrid
    n = 16
    pos, w, vel = _particles(n, 5)
    cuda = torch.device("cuda", 0)
    avg = float(w.sum()) / 1e6
    mod = DTFEGrid(grid=(n, n, n), n_threads=2, padding_particles=3.0, average_density=avg)
    tp = torch.tensor(pos, device=cuda, requires_grad=True)
    tw = torch.tensor(w, device=cuda, requires_grad=True)
    tv = torch.tensor(vel, device=cuda, requires_grad=True)
    dens, v, div = mod(tp, tw, tv)
    rng = np.random.default_rng(2)
    a = torch.tensor(rng.standard_normal(dens.shape), dtype=torch.float32, device=cuda)
    c = torch.tensor(rng.standard_normal(v.shape), dtype=torch.float32, device=cuda)
    b = torch.tensor(rng.standard_normal(div.shape), dtype=torch.float32, device=cuda)
    loss = (a * dens).sum() + (c * v).sum() + (b * div).sum()
    loss.backward()
    plan = mod.last_plan
    d32, d64, _ = O.vertex_density(plan)
    _, loc = O.interpolate(plan, d32, d64, ["density"], mode=O.MODE_FP64, want_loc=True)
    prob = O.AdjointProblem(plan, loc, a=a.cpu().numpy().ravel(), c=c.cpu().numpy().reshape(-1, 3),
                            b=b.cpu().numpy().ravel())
    ox, ov, ow = prob.grad(plan.xyz.astype(np.float64), plan.weight.astype(np.float64),
                           plan.velocity.astype(np.float64))
    N = len(pos)
    assert rel_err(tp.grad.cpu().numpy(), _per_particle(plan.src, ox, N)) < 1e-5
    assert rel_err(tv.grad.cpu().numpy(), _per_particle(plan.src, ov, N)) < 1e-5
    assert rel_err(tw.grad.cpu().numpy(), _per_particle(plan.src, ow, N)) < 1e-5
    # forward values: the same as the plain interpolation of that plan
    o, _ = O.interpolate(plan, d32, d64, ["density"], mode=O.MODE_FP64)
    assert rel_err(dens.detach().cpu().numpy().ravel(), o["density"]) < 1e-5


def test_autograd_stale_handle_raises(gpu_built):
    from dtfe_b200.autograd import DTFEGrid
    n = 8
    pos, w, vel = _particles(n, 7)
    cuda = torch.device("cuda", 0)
    mod = DTFEGrid(grid=(n, n, n), padding_particles=3.0, average_density=float(w.sum()) / 1e6)
    tp = torch.tensor(pos, device=cuda, requires_grad=True)
    tw = torch.tensor(w, device=cuda)
    tv = torch.tensor(vel, device=cuda)
    d1, _, _ = mod(tp, tw, tv)
    d2, _, _ = mod(tp, tw, tv)
    with pytest.raises(RuntimeError):
        d1.sum().backward()
    d2.sum().backward()
    assert torch.isfinite(tp.grad).all()


def test_adjoint_needs_centre_interpolation(gpu_built):
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    n = 8
    pos, w, vel = _particles(n, 8)
    plan = P.make_plan(pos, w, vel, None, grid=(n, n, n), padding_particles=3.0)
    cuda = torch.device("cuda", 0)
    G = n ** 3
    gx = torch.empty((plan.n_verts, 3), device=cuda)
    a = torch.ones(G, device=cuda)
    with DeviceDTFE(0) as dev:
        dev.load(plan)
        dev.vertex_density(plan.rho_bar)
        with pytest.raises(N.DTFEError):
            dev.adjoint_dev(gx, grad_density=a)
        out = torch.empty(G, device=cuda)
        dev.interpolate_dev(["density"], {"density": out}, method=3, n_samples=8)
        with pytest.raises(N.DTFEError):  # an averaged interpolation is not differentiated
            dev.adjoint_dev(gx, grad_density=a)


@pytest.mark.parametrize("kind", ["NGP", "CIC", "TSC"])
def test_deposit_adjoint(gpu_built, kind):
    from dtfe_b200.autograd import DepositGrid
    n = 16
    pos, w, _ = _particles(n, 11, disp=1.0)
    grid = (12, 12, 12)
    avg = float(w.sum()) / 1e6
    cuda = torch.device("cuda", 0)
    mod = DepositGrid(kind, grid=grid, n_threads=4, average_density=avg)
    tp = torch.tensor(pos, device=cuda, requires_grad=True)
    tw = torch.tensor(w, device=cuda, requires_grad=True)
    dens = mod(tp, tw)
    a = np.random.default_rng(4).standard_normal(grid)
    (torch.tensor(a, dtype=torch.float32, device=cuda) * dens).sum().backward()
    dplan = P.make_deposit_plan(pos, w, None, grid=grid, n_threads=4, kind=kind, average_density_value=avg)
    gx = np.zeros((dplan.n, 3))
    gw = np.zeros(dplan.n)
    for b in dplan.boxes:
        o, m = b.particle_offset, b.n_particles
        dims = [b.tile_dims[i] for i in range(3)]
        org = [b.tile_origin[i] for i in range(3)]
        at = a[org[0]:org[0] + dims[0], org[1]:org[1] + dims[1], org[2]:org[2] + dims[2]].ravel()
        _, x_, w_ = O.deposit_loss_grad(dplan.kind, dplan.pos[o:o + m], dplan.weight[o:o + m],
                                        np.array(list(b.region), np.float32), np.array(dims, np.int32),
                                        dplan.rho_bar, at)
        gx[o:o + m], gw[o:o + m] = x_, w_
    N = len(pos)
    assert rel_err(tw.grad.cpu().numpy(), _per_particle(dplan.src, gw, N)) < 1e-5
    if kind == "NGP":
        assert float(tp.grad.abs().max()) == 0.0
    else:
        assert rel_err(tp.grad.cpu().numpy(), _per_particle(dplan.src, gx, N)) < 1e-5
