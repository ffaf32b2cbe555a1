"""Seeded synthetic particle sets for the benchmark and test workloads.

The reference is benchmarked on N-body snapshots that are not part of this
project; these generators produce inputs with the same shapes, sizes and
statistics:

* ``zeldovich_lattice(n, L, rms, seed)`` — an n^3 cell-centred lattice in a
  periodic box of side L displaced by psi = -grad(phi), phi a Gaussian random
  field with P(k) ~ k^-2 smoothed by a Gaussian of 2 lattice spacings and
  scaled so that rms|psi| = rms * spacing.
* ``workload(name)`` — the five named workloads:
    ``zeldovich64_density``   64^3 particles, rms 0.5, density to a 128^3 grid
    ``zeldovich256_full``     256^3 particles, rms 1.0, velocity 100 km/s per unit
                              displacement + N(0, 50 km/s), one scalar, 256^3 grid
    ``zeldovich128_adjoint``  128^3 particles, rms 0.5, weights U[0.5, 1.5], 128^3 grid
    ``subboxes64_nfw``        64 periodic sub-boxes, log-normal counts in
                              [1e4, 1e6] (median 1e5), lattice + NFW cluster, 64^3 grids
    ``zeldovich512_scalars``  512^3 particles as the 256^3 set, 2 scalars N(0,1)
  Positions are float32 in [0, L).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BOX = 100.0  # Mpc/h


@dataclass
class Particles:
    pos: np.ndarray                 # (N, 3) float32
    weight: np.ndarray              # (N,) float32
    velocity: np.ndarray | None = None   # (N, 3) float32
    scalar: np.ndarray | None = None     # (N, S) float32
    box: tuple = (0.0, BOX, 0.0, BOX, 0.0, BOX)
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def zeldovich_displacement(n: int, L: float, rms: float, seed: int) -> np.ndarray:
    """Displacement field psi (n^3, 3) float64, rms|psi| = rms * L/n."""
    rng = np.random.default_rng(seed)
    dx = L / n
    noise = rng.standard_normal((n, n, n))
    nk = np.fft.rfftn(noise)
    k1 = 2 * np.pi * np.fft.fftfreq(n, d=dx)
    kz = 2 * np.pi * np.fft.rfftfreq(n, d=dx)
    kx, ky, kzz = np.meshgrid(k1, k1, kz, indexing="ij")
    k2 = kx * kx + ky * ky + kzz * kzz
    sigma = 2.0 * dx
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(k2 > 0, 1.0 / np.sqrt(k2), 0.0) * np.exp(-0.5 * k2 * sigma * sigma)
    phik = nk * amp
    psi = np.empty((n, n, n, 3))
    for a, ka in enumerate((kx, ky, kzz)):
        psi[..., a] = np.fft.irfftn(-1j * ka * phik, s=(n, n, n), axes=(0, 1, 2))
    psi = psi.reshape(-1, 3)
    cur = np.sqrt(np.mean(np.sum(psi * psi, axis=1)))
    return psi * (rms * dx / cur)


def zeldovich_lattice(n: int, L: float = BOX, rms: float = 0.5, seed: int = 0):
    """Returns (positions float32 (n^3,3) wrapped into [0,L), psi float64)."""
    dx = L / n
    g = (np.arange(n) + 0.5) * dx
    q = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    psi = zeldovich_displacement(n, L, rms, seed)
    x = np.mod(q + psi, L)
    pos = x.astype(np.float32)
    pos[pos >= np.float32(L)] = np.float32(0.0)
    return pos, psi


def nfw_radii(n: int, rs: float, c: float, rng) -> np.ndarray:
    """Radii drawn from an NFW profile truncated at c*rs (inverse CDF)."""
    x = np.linspace(0.0, c, 20001)
    m = np.log1p(x) - x / (1.0 + x)
    u = rng.random(n) * m[-1]
    return np.interp(u, m, x) * rs


def lattice_plus_nfw(nk: int, side: float, seed: int):
    """One periodic sub-box of about nk particles: a Zel'dovich lattice (rms
    0.5 spacing) holding 80% of them and an NFW-like cluster (r_s = 0.05 side,
    truncated at 10 r_s, random centre) holding 20%.  Velocities: 100 km/s per
    unit lattice displacement + N(0, 50 km/s) on the lattice, N(0, 300 km/s)
    per component in the cluster.  Returns (pos, vel) float32."""
    rng = np.random.default_rng(seed)
    n_cl = int(round(0.2 * nk))
    n_lat = max(2, int(round((nk - n_cl) ** (1.0 / 3.0))))
    lat, psi = zeldovich_lattice(n_lat, side, 0.5, seed + 1)
    v_lat = 100.0 * psi / (side / n_lat) + rng.normal(0.0, 50.0, psi.shape)
    r = nfw_radii(n_cl, 0.05 * side, 10.0, rng)
    d = rng.standard_normal((n_cl, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    centre = rng.random(3) * side
    cl = np.mod(centre + d * r[:, None], side).astype(np.float32)
    cl[cl >= np.float32(side)] = np.float32(0.0)
    v_cl = rng.normal(0.0, 300.0, (n_cl, 3))
    return (np.concatenate([lat, cl]).astype(np.float32),
            np.concatenate([v_lat, v_cl]).astype(np.float32))


def subbox_set(counts, side: float, seed0: int = 1000) -> list:
    """Periodic sub-boxes [0, side)^3 with the given particle counts."""
    boxes = []
    for i, nk in enumerate(counts):
        pos, vel = lattice_plus_nfw(int(nk), side, seed=seed0 + i)
        boxes.append(Particles(pos, np.ones(len(pos), np.float32), vel, box=(0.0, side, 0.0, side, 0.0, side)))
    return boxes


def workload(name: str) -> dict:
    """Builds a named workload: particles plus grid/interpolation settings."""
    if name == "zeldovich64_density":
        pos, _ = zeldovich_lattice(64, BOX, 0.5, seed=0)
        p = Particles(pos, np.ones(len(pos), np.float32))
        return dict(particles=p, grid=(128, 128, 128), fields=("density",), name=name)
    if name in ("zeldovich256_full", "zeldovich512_scalars"):
        n = 256 if name == "zeldovich256_full" else 512
        pos, psi = zeldovich_lattice(n, BOX, 1.0, seed=1)
        rng = np.random.default_rng(2)
        vel = (100.0 * psi / (BOX / n) + rng.normal(0.0, 50.0, psi.shape)).astype(np.float32)
        S = 1 if n == 256 else 2
        srng = np.random.default_rng(9 if n == 256 else 8)
        sc = srng.standard_normal((len(pos), S)).astype(np.float32)
        p = Particles(pos, np.ones(len(pos), np.float32), vel, sc)
        return dict(particles=p, grid=(n, n, n), name=name,
                    fields=("density", "velocity", "velocity_gradient", "velocity_divergence",
                            "velocity_shear", "velocity_vorticity"))
    if name == "zeldovich128_adjoint":
        pos, psi = zeldovich_lattice(128, BOX, 0.5, seed=0)
        w = np.random.default_rng(4).uniform(0.5, 1.5, len(pos)).astype(np.float32)
        vel = (100.0 * psi / (BOX / 128)).astype(np.float32)
        p = Particles(pos, w, vel)
        return dict(particles=p, grid=(128, 128, 128), fields=("density", "velocity_divergence"), name=name)
    if name == "subboxes64_nfw":
        rng = np.random.default_rng(7)
        counts = np.clip(np.exp(rng.normal(np.log(1e5), 1.0, 64)), 1e4, 1e6).astype(np.int64)
        boxes = subbox_set(counts, BOX / 4.0)
        return dict(subboxes=boxes, grid=(64, 64, 64), fields=("density", "velocity"),
                    padding_fraction=0.1, name=name)
    raise KeyError(name)
