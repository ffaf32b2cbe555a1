"""Differentiable DTFE and CIC / TSC grids (``torch.autograd.Function``).

The reference computes fields only; these functions add the reverse pass.
Forward: the host tessellation of the given particles (frozen for the
backward), vertex densities and cell-centre density, velocity and velocity
divergence on the device.  Backward: ``dtfe_gpu_adjoint_dev`` (per-cell
Jacobians recomputed from the tessellation, not stored) returns per-vertex
gradients, which are summed over each particle's periodic images.

Held fixed: the tessellation topology, the cell -> tetrahedron assignment
and the average density (given, or computed once from the weights), so the
gradients are those of the piecewise-linear interpolant on the current
tessellation.  Both classes own one device handle; a backward must follow
its own forward before the handle runs another forward.
"""
from __future__ import annotations

import numpy as np
import torch

from . import plan as P
from .device import DeviceDTFE


def _host(t: torch.Tensor | None, shape_tail=()) -> np.ndarray | None:
    if t is None:
        return None
    return np.ascontiguousarray(t.detach().to("cpu", torch.float32).numpy())


def _grad(t, like_shape, dev) -> torch.Tensor | None:
    if t is None:
        return None
    return t.detach().to(dev, torch.float32).contiguous().reshape(like_shape)


class _Owner:
    def __init__(self, device: int):
        self.device = device
        self.cuda = torch.device("cuda", device)
        self.dev = DeviceDTFE(device)
        self.generation = 0

    def check(self, gen: int) -> None:
        if gen != self.generation:
            raise RuntimeError("this handle ran another forward after the one being differentiated; "
                               "call backward before the next forward, or use one object per graph")


class _DTFEFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, weight, velocity, mod):
        o = mod._owner
        plan = P.make_plan(_host(pos), _host(weight), _host(velocity), None, grid=mod.grid, box=mod.box,
                           periodic=mod.periodic, n_threads=mod.n_threads,
                           padding_particles=mod.padding_particles, average_density_value=mod.average_density)
        torch.cuda.current_stream(o.cuda).synchronize()
        o.dev.load(plan)
        o.dev.vertex_density(plan.rho_bar)
        G = int(np.prod(plan.grid))
        dens = torch.empty(G, dtype=torch.float32, device=o.cuda)
        vel = torch.empty((G, 3), dtype=torch.float32, device=o.cuda)
        div = torch.empty(G, dtype=torch.float32, device=o.cuda)
        o.dev.interpolate_dev(["density", "velocity", "velocity_divergence"],
                              {"density": dens, "velocity": vel, "velocity_divergence": div}, method=0, fix=mod.fix_value)
        o.generation += 1
        ctx.gen = o.generation
        ctx.mod = mod
        ctx.src = torch.from_numpy(plan.src.astype(np.int64)).to(o.cuda)
        ctx.n_verts = plan.n_verts
        ctx.n = pos.shape[0]
        ctx.in_dev = (pos.device, weight.device, velocity.device)
        mod.last_plan = plan
        g = tuple(plan.grid)
        return dens.view(g), vel.view(g + (3,)), div.view(g)

    @staticmethod
    def backward(ctx, g_dens, g_vel, g_div):
        o = ctx.mod._owner
        o.check(ctx.gen)
        torch.cuda.current_stream(o.cuda).synchronize()
        G = int(np.prod(ctx.mod.grid))
        a = _grad(g_dens, (G,), o.cuda)
        c = _grad(g_vel, (G, 3), o.cuda)
        b = _grad(g_div, (G,), o.cuda)
        V = ctx.n_verts
        gx = torch.empty((V, 3), dtype=torch.float32, device=o.cuda)
        gv = torch.empty((V, 3), dtype=torch.float32, device=o.cuda)
        gw = torch.empty(V, dtype=torch.float32, device=o.cuda)
        o.dev.adjoint_dev(gx, grad_density=a, grad_velocity=c, grad_divergence=b, grad_vel=gv, grad_w=gw)
        n = ctx.n
        gpos = torch.zeros((n, 3), dtype=torch.float32, device=o.cuda).index_add_(0, ctx.src, gx)
        gvel = torch.zeros((n, 3), dtype=torch.float32, device=o.cuda).index_add_(0, ctx.src, gv)
        gwt = torch.zeros(n, dtype=torch.float32, device=o.cuda).index_add_(0, ctx.src, gw)
        dp, dw, dv = ctx.in_dev
        return gpos.to(dp), gwt.to(dw), gvel.to(dv), None


class DTFEGrid:
    """Cell-centre DTFE density, velocity and velocity divergence on a regular
    grid, differentiable with respect to particle positions, weights and
    velocities.  ``grid``, ``box``, ``periodic``, ``n_threads`` and
    ``padding_particles`` have the meaning of the reference's options
    (gridSize, boxCoordinates, periodic, parallel sub-boxes, padding);
    ``fix_value`` evaluates the velocity value with the full offset product
    instead of the reference's z-term-only form."""

    def __init__(self, grid=(64, 64, 64), box=(0, 100, 0, 100, 0, 100), periodic: bool = True,
                 n_threads: int = 1, padding_particles: float = 5.0, average_density: float | None = None,
                 fix_value: bool = False, device: int = 0):
        self.grid = tuple(int(g) for g in grid)
        self.box = tuple(float(b) for b in box)
        self.periodic = periodic
        self.n_threads = n_threads
        self.padding_particles = padding_particles
        self.average_density = average_density
        self.fix_value = fix_value
        self._owner = _Owner(device)
        self.last_plan = None

    def __call__(self, pos: torch.Tensor, weight: torch.Tensor, velocity: torch.Tensor):
        """Returns (density (gx, gy, gz), velocity (gx, gy, gz, 3), divergence)."""
        return _DTFEFunction.apply(pos, weight, velocity, self)


class _DepositFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, weight, mod):
        o = mod._owner
        dplan = P.make_deposit_plan(_host(pos), _host(weight), None, grid=mod.grid, box=mod.box,
                                    periodic=mod.periodic, n_threads=mod.n_threads, kind=mod.kind,
                                    average_density_value=mod.average_density)
        torch.cuda.current_stream(o.cuda).synchronize()
        G = int(np.prod(dplan.grid))
        dens = torch.empty(G, dtype=torch.float32, device=o.cuda)
        o.dev.deposit_dev(dplan, dens)
        o.generation += 1
        ctx.gen = o.generation
        ctx.mod = mod
        ctx.src = torch.from_numpy(dplan.src).to(o.cuda)
        ctx.copies = dplan.n
        ctx.n = pos.shape[0]
        ctx.in_dev = (pos.device, weight.device)
        return dens.view(dplan.grid)

    @staticmethod
    def backward(ctx, g_dens):
        o = ctx.mod._owner
        o.check(ctx.gen)
        torch.cuda.current_stream(o.cuda).synchronize()
        G = int(np.prod(ctx.mod.grid))
        a = _grad(g_dens, (G,), o.cuda)
        m = ctx.copies
        gx = torch.empty((m, 3), dtype=torch.float32, device=o.cuda)
        gw = torch.empty(m, dtype=torch.float32, device=o.cuda)
        o.dev.deposit_adjoint_dev(a, gx, gw)
        n = ctx.n
        gpos = torch.zeros((n, 3), dtype=torch.float32, device=o.cuda).index_add_(0, ctx.src, gx)
        gwt = torch.zeros(n, dtype=torch.float32, device=o.cuda).index_add_(0, ctx.src, gw)
        dp, dw = ctx.in_dev
        return gpos.to(dp), gwt.to(dw), None


class DepositGrid:
    """NGP / CIC / TSC density on a regular grid (the reference's
    *_interpolation_regular_grid normalisation), differentiable with respect
    to particle positions and weights (NGP: zero position gradient)."""

    def __init__(self, kind: str = "CIC", grid=(64, 64, 64), box=(0, 100, 0, 100, 0, 100), periodic: bool = True,
                 n_threads: int = 1, average_density: float | None = None, device: int = 0):
        if kind not in P.DEPOSIT_KINDS:
            raise ValueError(f"unknown deposition kind {kind!r}")
        self.kind = kind
        self.grid = tuple(int(g) for g in grid)
        self.box = tuple(float(b) for b in box)
        self.periodic = periodic
        self.n_threads = n_threads
        self.average_density = average_density
        self._owner = _Owner(device)

    def __call__(self, pos: torch.Tensor, weight: torch.Tensor) -> torch.Tensor:
        return _DepositFunction.apply(pos, weight, self)
