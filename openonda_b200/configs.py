"""Seeded synthetic particle fields for the five benchmark workloads.

The reference ships no benchmark inputs, so every workload is generated here from a
seed.  All generators return float64 numpy arrays in the reference's layout:
``positions (N,3)``, ``strengths (N,3)``, ``radii (N,)``, ``viscosities (N,)``.

Rings follow the reference's own convention (``vortex_ring_vpm``,
OpenONDA/utilities/vpm_flow_models.py:87-159): the ring lies in the y-z plane with
its axis along x, the core has the Gaussian profile
``omega(d) = Gamma / (pi sigma^2) exp(-d^2 / sigma^2)`` (vpm_flow_models.py:136) and
each particle carries ``alpha = omega * vol`` along the azimuthal direction
``(0, -sin(theta), cos(theta))`` (vpm_flow_models.py:141-142).

Torus lattice: ``n_azimuthal`` planes at equal angles; in each plane
``n_section`` points fill the disc of radius ``3 sigma`` on a sunflower (Vogel)
spiral, so every point owns the same cross-section area ``pi (3 sigma)^2 / n_section``.
The particle volume is that area times the local arc length ``(R + d_radial) dtheta``.
The lattice spacing is ``h = mean(vol)^(1/3)`` and particle cores are ``1.2 h``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GOLDEN_ANGLE = np.pi * (3.0 - np.sqrt(5.0))


@dataclass
class ParticleField:
    positions: np.ndarray
    strengths: np.ndarray
    radii: np.ndarray
    viscosities: np.ndarray
    description: str = ""

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])


def torus_lattice(ring_radius: float, core_sigma: float, n_azimuthal: int, n_section: int,
                  centre=(0.0, 0.0, 0.0), theta0: float = 0.0, radial_offset=None,
                  extent: float = 3.0):
    """Return (positions, volumes, theta, d_axial, d_radial) of a torus lattice.

    ``radial_offset(theta)``, when given, displaces the core centreline radially.
    """
    a = extent * core_sigma
    m = np.arange(n_section, dtype=np.float64)
    rho = a * np.sqrt((m + 0.5) / n_section)
    phi = m * GOLDEN_ANGLE
    d_axial = rho * np.cos(phi)  # along the ring axis (x)
    d_radial = rho * np.sin(phi)  # in the ring plane, away from the axis
    theta = theta0 + 2.0 * np.pi * np.arange(n_azimuthal, dtype=np.float64) / n_azimuthal
    dtheta = 2.0 * np.pi / n_azimuthal
    area = np.pi * a * a / n_section

    th = np.repeat(theta, n_section)
    da = np.tile(d_axial, n_azimuthal)
    dr = np.tile(d_radial, n_azimuthal)
    rc = np.full_like(th, ring_radius)
    if radial_offset is not None:
        rc = rc + radial_offset(th)
    r_plane = rc + dr
    pos = np.empty((th.size, 3), dtype=np.float64)
    pos[:, 0] = centre[0] + da
    pos[:, 1] = centre[1] + r_plane * np.cos(th)
    pos[:, 2] = centre[2] + r_plane * np.sin(th)
    vol = area * r_plane * dtheta
    return pos, vol, th, da, dr


def gaussian_ring_strengths(theta, d_axial, d_radial, vol, gamma, core_sigma):
    d2 = d_axial * d_axial + d_radial * d_radial
    omega = gamma / (np.pi * core_sigma * core_sigma) * np.exp(-d2 / (core_sigma * core_sigma))
    a = np.zeros((theta.size, 3), dtype=np.float64)
    a[:, 1] = -omega * np.sin(theta) * vol
    a[:, 2] = omega * np.cos(theta) * vol
    return a


def vortex_ring(n_azimuthal=64, n_section=128, ring_radius=1.0, gamma=1.0, core_sigma=0.1,
                nu=1e-4, centre=(0.0, 0.0, 0.0), radial_offset=None, core_factor=1.2,
                theta0: float = 0.0) -> ParticleField:
    pos, vol, th, da, dr = torus_lattice(ring_radius, core_sigma, n_azimuthal, n_section,
                                         centre=centre, theta0=theta0,
                                         radial_offset=radial_offset)
    alpha = gaussian_ring_strengths(th, da, dr, vol, gamma, core_sigma)
    h = float(np.mean(vol)) ** (1.0 / 3.0)
    radii = np.full(pos.shape[0], core_factor * h)
    visc = np.full(pos.shape[0], nu)
    return ParticleField(pos, alpha, radii, visc,
                         f"ring R={ring_radius} Gamma={gamma} sigma={core_sigma} "
                         f"{n_azimuthal}x{n_section} core={core_factor}h")


def ring_8192() -> ParticleField:
    """Thick ring R=1, Gamma=1, sigma=0.1 on a 64 x 128 torus lattice (N=8192), nu=1e-4."""
    return vortex_ring(64, 128, 1.0, 1.0, 0.1, nu=1e-4)


def leapfrog_rings(n_azimuthal=256, n_section=256, separation=0.4, core_sigma=0.08,
                   nu=1e-4) -> ParticleField:
    """Two coaxial rings R=1, Gamma=1, sigma=0.08, offset by ``separation`` along x."""
    a = vortex_ring(n_azimuthal, n_section, 1.0, 1.0, core_sigma, nu=nu,
                    centre=(-0.5 * separation, 0.0, 0.0))
    b = vortex_ring(n_azimuthal, n_section, 1.0, 1.0, core_sigma, nu=nu,
                    centre=(0.5 * separation, 0.0, 0.0))
    return ParticleField(np.concatenate([a.positions, b.positions]),
                         np.concatenate([a.strengths, b.strengths]),
                         np.concatenate([a.radii, b.radii]),
                         np.concatenate([a.viscosities, b.viscosities]),
                         f"leapfrog 2x({a.description}) sep={separation}")


def random_cloud(n: int, seed: int = 0, nu: float = 1e-4) -> ParticleField:
    """Uniform positions in [-1,1]^3, alpha ~ N(0, 1e-3) per component, sigma ~ U(0.02, 0.05)."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1.0, 1.0, size=(n, 3))
    alpha = rng.normal(0.0, 1e-3, size=(n, 3))
    radii = rng.uniform(0.02, 0.05, size=n)
    visc = np.full(n, nu)
    return ParticleField(pos, alpha, radii, visc, f"random cloud N={n} seed={seed}")


def perturbed_ring(n_azimuthal=256, n_section=256, amplitude=0.02, modes=range(2, 9),
                   seed: int = 0, core_sigma=0.1, nu=1e-4) -> ParticleField:
    """Ring R=1, sigma=0.1 whose centreline radius carries modes 2-8 with seeded phases.

    The total amplitude is split evenly: each mode has amplitude ``amplitude/len(modes)``.
    """
    rng = np.random.default_rng(seed)
    modes = list(modes)
    phases = rng.uniform(0.0, 2.0 * np.pi, size=len(modes))
    amp = amplitude / len(modes)

    def offset(th):
        return sum(amp * np.cos(k * th + p) for k, p in zip(modes, phases))

    f = vortex_ring(n_azimuthal, n_section, 1.0, 1.0, core_sigma, nu=nu, radial_offset=offset)
    f.description += f" radial modes {modes[0]}-{modes[-1]} amp={amplitude} seed={seed}"
    return f


def les_ring(n_azimuthal=1024, n_section=1024, core_sigma=0.05, noise=0.01, seed: int = 0,
             nu=1e-5) -> ParticleField:
    """Ring R=1, Gamma=1, sigma=0.05 with seeded azimuthal-mode noise of amplitude 0.01."""
    rng = np.random.default_rng(seed)
    modes = np.arange(1, 33)
    phases = rng.uniform(0.0, 2.0 * np.pi, size=modes.size)
    weights = rng.normal(size=modes.size)
    weights *= noise / np.sqrt(np.sum(weights * weights))

    def offset(th):
        return sum(w * np.cos(k * th + p) for k, w, p in zip(modes, weights, phases))

    f = vortex_ring(n_azimuthal, n_section, 1.0, 1.0, core_sigma, nu=nu, radial_offset=offset)
    f.description += f" azimuthal noise amp={noise} seed={seed}"
    return f
