"""Analytical vorticity fields on particles, computed on the GPU.

Same functions, arguments and return values as OpenONDA/utilities/vpm_flow_models.py
(``lamb_oseen_vpm`` :14-83, ``vortex_ring_vpm`` :87-163): numpy inputs give numpy outputs,
CUDA tensors give CUDA tensors.  The per-particle work and the circulation rescaling of the
ring run in the library kernels (``vpm_ic_lamb_oseen``, ``vpm_ic_vortex_ring``).
``isotropic_turbulence_vpm`` (:167-271) runs its FFT synthesis on the GPU (cuFFT through
torch.fft) with the same random phases (numpy's MT19937 stream for seed 0, drawn on the
host from a private generator instead of re-seeding the global one).
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _lib
from ._dev import cuda_device, stream, to_device

epsilon = 1e-9


def gaussian(r, omega_0, a):
    """vpm_flow_models.py:5-6."""
    return omega_0 * np.exp(-(r ** 2) / a ** 2)


def _prepare(particle_positions, volumes):
    tensor_in = isinstance(particle_positions, torch.Tensor)
    dev = cuda_device(particle_positions.device if tensor_in and
                      particle_positions.device.type == "cuda" else None)
    x = to_device(particle_positions, dev, (3,), "particle_positions")
    v = to_device(volumes, dev, (), "volumes").reshape(-1)
    if v.shape[0] != x.shape[0]:
        raise ValueError("volumes must have one entry per particle")
    return tensor_in, dev, x, v


def _outputs(n, dev):
    return (torch.zeros((n, 3), dtype=torch.float64, device=dev),
            torch.empty((n, 3), dtype=torch.float64, device=dev),
            torch.empty(n, dtype=torch.float64, device=dev),
            torch.empty(n, dtype=torch.float64, device=dev))


def _finish(tensor_in, out):
    return out if tensor_in else tuple(t.cpu().numpy() for t in out)


def lamb_oseen_vpm(particle_positions, volumes, particle_radius: float,
                   particle_viscosity: float, vortex_center, vortex_strength: float,
                   core_radius: float, epsilon_W: float = 0.0, phase_W: float = 0.0,
                   N_W: float = 12):
    """Lamb-Oseen vortex along z with a sinusoidal displacement of its axis.
    Returns (velocities (zero), strengths, radii, viscosities)."""
    tensor_in, dev, x, v = _prepare(particle_positions, volumes)
    n = x.shape[0]
    out = _outputs(n, dev)
    c = np.asarray(vortex_center, dtype=np.float64).reshape(3)
    _lib.check(_lib.load().vpm_ic_lamb_oseen(
        x.data_ptr(), v.data_ptr(), n, float(particle_radius), float(particle_viscosity),
        float(c[0]), float(c[1]), float(c[2]), float(vortex_strength), float(core_radius),
        float(epsilon_W), float(phase_W), float(N_W), out[1].data_ptr(), out[2].data_ptr(),
        out[3].data_ptr(), stream(dev)))
    return _finish(tensor_in, out)


def vortex_ring_vpm(particle_positions, volumes, particle_radius: float,
                    particle_viscosity: float, ring_center, ring_radius: float,
                    ring_strength: float, ring_thickness: float, epsilon_W: float = 0.0,
                    phase_W: float = 0.0, N_W: float = 12):
    """Gaussian-core vortex ring in the y-z plane with an azimuthal core displacement,
    strengths rescaled so that sum|alpha| = 2 pi R Gamma.
    Returns (velocities (zero), strengths, radii, viscosities).  Raises ZeroDivisionError
    when the field carries no circulation (as the reference does)."""
    tensor_in, dev, x, v = _prepare(particle_positions, volumes)
    n = x.shape[0]
    out = _outputs(n, dev)
    c = np.asarray(ring_center, dtype=np.float64).reshape(3)
    lib = _lib.load()
    ws = torch.empty(max(int(lib.vpm_ic_workspace_bytes(n)), 256), dtype=torch.uint8,
                     device=dev)
    _lib.check(lib.vpm_ic_vortex_ring(
        x.data_ptr(), v.data_ptr(), n, float(particle_radius), float(particle_viscosity),
        float(c[0]), float(c[1]), float(c[2]), float(ring_radius), float(ring_strength),
        float(ring_thickness), float(epsilon_W), float(phase_W), float(N_W),
        out[1].data_ptr(), out[2].data_ptr(), out[3].data_ptr(), ws.data_ptr(), ws.numel(),
        stream(dev)))
    if n and not bool(torch.isfinite(out[1]).all()):
        raise ZeroDivisionError("vortex_ring_vpm: the particles carry no circulation")
    return _finish(tensor_in, out)


def isotropic_turbulence_vpm(box_size: float, particle_distance: float, particle_radius: float,
                             device=None):
    """Particles on a cubic lattice carrying a synthetic isotropic velocity field with a
    k^-5/3 spectrum and a Gaussian cut-off at k_max/3 (vpm_flow_models.py:167-271).
    Returns (positions, velocities, strengths, radii): numpy arrays, or CUDA tensors when
    ``device`` names a CUDA device.

    Kept as in the reference: the three velocity components share one set of random phases
    before the divergence-free projection, and each vorticity component keeps only the first
    of its two central differences (the reference's second term is a separate statement
    whose value is discarded, :250-262), so omega = (du_z/dy, du_x/dz, du_y/dx)."""
    dev = cuda_device(device)
    axis = np.arange(-box_size / 2, box_size / 2, step=particle_distance)
    n = len(axis)
    L = box_size
    k_diss = (np.pi * n / L) / 3
    ax = torch.from_numpy(axis).to(dev)
    xx, yy, zz = torch.meshgrid(ax, ax, ax, indexing="ij")
    positions = torch.stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)], dim=1)
    k = torch.from_numpy(np.fft.fftfreq(n, L / n) * 2 * np.pi).to(dev)
    KX, KY, KZ = torch.meshgrid(k, k, k, indexing="ij")
    K = torch.sqrt(KX * KX + KY * KY + KZ * KZ)
    E = K ** (-5 / 3) * torch.exp(-((K / k_diss) ** 2))
    E[K == 0] = 0
    phases = torch.exp((2j * np.pi) * torch.from_numpy(np.random.RandomState(0).rand(n, n, n))
                       .to(dev))
    amp = torch.sqrt(E)
    ux, uy, uz = amp * phases, amp * phases, amp * phases
    Kd = K + 1e-10
    dot = (KX * ux + KY * uy + KZ * uz) / Kd
    ux = ux - dot * KX / Kd
    uy = uy - dot * KY / Kd
    uz = uz - dot * KZ / Kd
    u = [torch.fft.ifftn(c).real for c in (ux, uy, uz)]
    velocities = torch.stack([c.reshape(-1) for c in u], dim=1)
    h2 = 2 * particle_distance
    w0 = (torch.roll(u[2], -1, dims=1) - torch.roll(u[2], 1, dims=1)) / h2
    w1 = (torch.roll(u[0], -1, dims=2) - torch.roll(u[0], 1, dims=2)) / h2
    w2 = (torch.roll(u[1], -1, dims=0) - torch.roll(u[1], 1, dims=0)) / h2
    strengths = (torch.stack([w0.reshape(-1), w1.reshape(-1), w2.reshape(-1)], dim=1)
                 * (4 / 3) * particle_distance ** 3)
    radii = torch.full((n ** 3,), float(particle_radius), dtype=torch.float64, device=dev)
    out = (positions.contiguous(), velocities.contiguous(), strengths.contiguous(), radii)
    return out if device is not None else tuple(t.cpu().numpy() for t in out)
