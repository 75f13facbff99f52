"""CPU restatement of the reference's initial-condition and lattice generators (TEST
INFRASTRUCTURE: only tests/ import this module; it is the checker, never the product).

Restates, in numpy with the reference's operation order:

* ``vortex_ring_vpm``  -- OpenONDA/utilities/vpm_flow_models.py:87-163
* ``lamb_oseen_vpm``   -- OpenONDA/utilities/vpm_flow_models.py:14-83
* ``get_rectangular_point_distribuition``    -- OpenONDA/utilities/vpm_solver_helper.py:21-68
* ``get_2D_rectangular_point_distribuition`` -- vpm_solver_helper.py:71-117
* ``get_hexagonal_point_distribution``       -- vpm_solver_helper.py:120-161
* ``get_cylindrical_point_distribuition``    -- vpm_solver_helper.py:164-253
* ``isotropic_turbulence_vpm`` -- OpenONDA/utilities/vpm_flow_models.py:167-271

Pinned by tests/test_ic_oracle.py against tests/golden/ic.npz, which holds the reference
functions' own outputs (tests/golden/make_golden.py, job ``ic``).  The reference compiles the
ring, Lamb-Oseen and cylinder generators with numba ``fastmath`` (reassociation, contraction,
its own transcendental functions), so agreement is to a few ulp, not bitwise.
"""
from __future__ import annotations

import math

import numpy as np


def _linspace(start, stop, num):
    # numpy / numba: start + i * step, last element = stop
    return np.linspace(start, stop, num=num)


def _arange(start, stop, step):
    # numba's arange (the hexagonal generator is @njit): ceil((stop - start)/step) items,
    # start + i * step
    n = max(int(math.ceil((stop - start) / step)), 0)
    return start + np.arange(n, dtype=np.float64) * step


def vortex_ring_vpm(particle_positions, volumes, particle_radius, particle_viscosity,
                    ring_center, ring_radius, ring_strength, ring_thickness, epsilon_W=0.0,
                    phase_W=0.0, N_W=12):
    """vpm_flow_models.py:87-163."""
    c = np.asarray(ring_center, dtype=np.float64)
    X = particle_positions[:, 0] - c[0]
    Y = particle_positions[:, 1] - c[1]
    Z = particle_positions[:, 2] - c[2]
    theta = np.arctan2(Z, Y)
    Y = Y - epsilon_W * np.cos(phase_W + N_W * theta)
    Z = Z - epsilon_W * np.sin(phase_W + N_W * theta)
    r_yz = np.sqrt(Y * Y + Z * Z)
    d = np.abs(r_yz - ring_radius)
    th2 = ring_thickness * ring_thickness
    mag = (ring_strength / (np.pi * th2)) * np.exp(-(d * d) / th2)
    decay = np.exp(-(X * X) / th2)
    a = np.empty_like(particle_positions, dtype=np.float64)
    a[:, 0] = np.zeros_like(X) * volumes
    a[:, 1] = (-mag * np.sin(theta)) * decay * volumes
    a[:, 2] = (mag * np.cos(theta)) * decay * volumes
    total = np.sum(np.sqrt(np.sum(a * a, axis=1)))
    a *= np.abs(2 * np.pi * ring_radius * ring_strength / total)
    n = len(particle_positions)
    return (np.zeros_like(a), a, np.full(n, particle_radius, dtype=np.float64),
            np.full(n, particle_viscosity, dtype=np.float64))


def lamb_oseen_vpm(particle_positions, volumes, particle_radius, particle_viscosity,
                   vortex_center, vortex_strength, core_radius, epsilon_W=0.0, phase_W=0.0,
                   N_W=12):
    """vpm_flow_models.py:14-83."""
    c = np.asarray(vortex_center, dtype=np.float64)
    z = particle_positions[:, 2]
    px = c[0] + epsilon_W * np.sin(phase_W + N_W * z)
    py = c[1] + epsilon_W * np.cos(phase_W + N_W * z)
    x = particle_positions[:, 0] - px
    y = particle_positions[:, 1] - py
    r = np.sqrt(x * x + y * y)
    rc2 = core_radius * core_radius
    a = np.zeros_like(particle_positions, dtype=np.float64)
    a[:, 2] = (vortex_strength / (np.pi * rc2)) * np.exp(-(r * r) / rc2) * volumes
    n = len(particle_positions)
    return (np.zeros_like(a), a, np.full(n, particle_radius, dtype=np.float64),
            np.full(n, particle_viscosity, dtype=np.float64))


def _odd(k):
    return k + 1 if k % 2 == 0 else k


def get_rectangular_point_distribuition(box_limits, spacing):
    """vpm_solver_helper.py:21-68."""
    b = np.asarray(box_limits, dtype=np.float64)
    nums = [_odd(int(np.ceil((b[2 * k + 1] - b[2 * k]) / spacing)) + 1) for k in range(3)]
    axes = [_linspace(b[2 * k], b[2 * k + 1], nums[k]) for k in range(3)]
    xx, yy, zz = np.meshgrid(*axes, indexing="ij")
    pts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    vol = (b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]) / len(pts)
    return pts, np.full(len(pts), vol)


def get_2D_rectangular_point_distribuition(box_limits, spacing):
    """vpm_solver_helper.py:71-117."""
    b = np.asarray(box_limits, dtype=np.float64)
    nums = [_odd(int(np.ceil((b[2 * k + 1] - b[2 * k]) / spacing)) + 1) for k in range(2)]
    xx, yy = np.meshgrid(_linspace(b[0], b[1], nums[0]), _linspace(b[2], b[3], nums[1]),
                         indexing="ij")
    pts = np.stack([xx.ravel(), yy.ravel(), np.zeros(xx.size)], axis=1)
    vol = (b[1] - b[0]) * (b[3] - b[2]) / len(pts)
    return pts, np.full(len(pts), vol)


def get_hexagonal_point_distribution(box_limits, spacing):
    """vpm_solver_helper.py:120-161."""
    x0, x1, y0, y1, z0, z1 = (float(v) for v in box_limits)
    sy = spacing * np.sqrt(3) / 2
    xs = _arange(x0, x1 + spacing, spacing)
    ys = _arange(y0, y1 + sy, sy)
    zs = _arange(z0, z1 + spacing, spacing)
    off = np.where(np.arange(len(ys)) % 2 == 1, spacing / 2, 0.0)
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    xx = xx + off[None, :, None]
    pts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    return pts, np.full(len(pts), spacing ** 3 * np.sqrt(3) / 2)


def get_cylindrical_point_distribuition(particle_distance, radius=1.0, height=2.0,
                                        center=np.array([0, 0, 0]), axis="x"):
    """vpm_solver_helper.py:164-253."""
    if axis not in ("x", "y", "z"):
        raise ValueError("Invalid axis. Choose from 'x', 'y', or 'z'.")
    c = np.asarray(center, dtype=np.float64)
    nr = int(radius / particle_distance)
    nh = int(height / particle_distance)
    nth = int(np.pi * radius / particle_distance)
    dtheta = 2 * np.pi / nth
    dz = height / nh
    dr = radius / nr
    r = _linspace(dr, radius, nr)
    z = _linspace(-height / 2, height / 2, nh + 1)
    th = _linspace(0, 2 * np.pi, nth)[:-1]
    R, Zg, T = np.meshgrid(r, z, th, indexing="ij")
    R, Zg, T = R.ravel(), Zg.ravel(), T.ravel()
    a, b = R * np.cos(T), R * np.sin(T)
    order = {"x": (Zg, a, b), "y": (a, Zg, b), "z": (a, b, Zg)}[axis]
    body = np.stack([order[0] + c[0], order[1] + c[1], order[2] + c[2]], axis=1)
    vol = (R * dtheta) * dr * dz
    zero = np.zeros_like(z)
    ax = {"x": (z, zero, zero), "y": (zero, z, zero), "z": (zero, zero, z)}[axis]
    axis_pts = np.stack([ax[0] + c[0], ax[1] + c[1], ax[2] + c[2]], axis=1)
    axis_vol = np.full(len(z), np.pi * (radius ** 2) * dz / len(z))
    return np.concatenate([body, axis_pts]), np.concatenate([vol, axis_vol])


def isotropic_turbulence_vpm(box_size, particle_distance, particle_radius):
    """vpm_flow_models.py:167-271 (numpy FFTs; phases from numpy's MT19937 stream for seed 0;
    each vorticity component keeps only the first central difference, as the reference's
    second term is a discarded statement)."""
    x = np.arange(-box_size / 2, box_size / 2, step=particle_distance)
    n, L = len(x), box_size
    xx, yy, zz = np.meshgrid(x, x, x, indexing="ij")
    pts = np.vstack([xx.ravel(), yy.ravel(), zz.ravel()]).T
    k_diss = (np.pi * n / L) / 3
    k = np.fft.fftfreq(n, L / n) * 2 * np.pi
    KX, KY, KZ = np.meshgrid(k, k, k, indexing="ij")
    K = np.sqrt(KX * KX + KY * KY + KZ * KZ)
    with np.errstate(divide="ignore"):
        E = K ** (-5 / 3) * np.exp(-((K / k_diss) ** 2))
    E[K == 0] = 0
    ph = np.exp(2j * np.pi * np.random.RandomState(0).rand(n, n, n))
    ux, uy, uz = np.sqrt(E) * ph, np.sqrt(E) * ph, np.sqrt(E) * ph
    Kd = K + 1e-10
    dot = (KX * ux + KY * uy + KZ * uz) / Kd
    ux, uy, uz = ux - dot * KX / Kd, uy - dot * KY / Kd, uz - dot * KZ / Kd
    u = [np.real(np.fft.ifftn(c)) for c in (ux, uy, uz)]
    vel = np.stack([c.reshape(-1) for c in u], axis=1)
    h2 = 2 * particle_distance
    w = np.stack([((np.roll(u[2], -1, axis=1) - np.roll(u[2], 1, axis=1)) / h2).reshape(-1),
                  ((np.roll(u[0], -1, axis=2) - np.roll(u[0], 1, axis=2)) / h2).reshape(-1),
                  ((np.roll(u[1], -1, axis=0) - np.roll(u[1], 1, axis=0)) / h2).reshape(-1)],
                 axis=1)
    return pts, vel, w * (4 / 3) * particle_distance ** 3, np.full(len(pts), particle_radius)
