"""Dense FP64 torch restatement of the VPM right-hand side (TEST INFRASTRUCTURE).

A direct O(N^2)-memory transcription of the GPU-semantics kernels of
OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py -- self-induced velocity (:133-191),
stretching (:375-445), PSE (:478-530) and kinetic energy (:563-642) -- written with the
reference's own formulas (powers of rho^2 + 1) so that torch.autograd provides the FP64
reference gradient for the hand-written adjoint kernels.  The forward values are pinned to
the oracle (tests/test_dense_reference.py).  Small N only (a few hundred particles).
"""
from __future__ import annotations

import math

import torch

ONE_OVER_FOUR_PI = 1.0 / (4.0 * math.pi)


def _pairs(x, sigma):
    r = x[:, None, :] - x[None, :, :]  # r_ij = x_i - x_j
    r2 = (r * r).sum(-1)
    s = 0.5 * (sigma[:, None] + sigma[None, :])
    n = x.shape[0]
    off = ~torch.eye(n, dtype=torch.bool, device=x.device)
    return r, r2, s, off


def velocity(x, a, sigma):
    r, r2, s, off = _pairs(x, sigma)
    rho2 = r2 / (s * s)
    q = (rho2 + 2.5) / ((rho2 + 1.0) ** 2.5 * s * s * s)
    q = torch.where(off, q, torch.zeros_like(q))
    c = torch.cross(r, a[None, :, :].expand_as(r), dim=-1)
    return -ONE_OVER_FOUR_PI * (q[..., None] * c).sum(1)


def stretching(x, a, sigma):
    r, r2, s, off = _pairs(x, sigma)
    s2 = s * s
    p1 = r2 / s2 + 1.0
    f1 = (p1 + 1.5) / (s2 * s * p1 ** 2.5)
    f2 = 3.0 * (p1 + 2.5) / (s2 * s * s2 * p1 ** 3.5)
    f1 = torch.where(off, f1, torch.zeros_like(f1))
    f2 = torch.where(off, f2, torch.zeros_like(f2))
    ai = a[:, None, :].expand_as(r)
    aj = a[None, :, :].expand_as(r)
    c1 = torch.cross(ai, aj, dim=-1)
    c2 = torch.cross(r, aj, dim=-1)
    d3 = (ai * c2).sum(-1)
    return ONE_OVER_FOUR_PI * (f1[..., None] * c1 + (f2 * d3)[..., None] * r).sum(1)


def pse(x, a, sigma, nu):
    r, r2, s, off = _pairs(x, sigma)
    s2 = s * s
    s3 = s2 * s
    p1 = r2 / s2 + 1.0
    f3 = 105.0 * nu[:, None] / (s2 * s3 * p1 ** 4.5)
    f3 = torch.where(off, f3, torch.zeros_like(f3))
    d = a[None, :, :] - a[:, None, :]
    return ONE_OVER_FOUR_PI * ((f3 * s3)[..., None] * d).sum(1)


def kinetic_energy(x, a, sigma):
    r, r2, s, off = _pairs(x, sigma)
    # safe norm on the diagonal (masked out below)
    rn = torch.sqrt(torch.where(off, r2, torch.ones_like(r2)))
    u = r / rn[..., None]
    rho = rn / s
    p1 = rho * rho + 1.0
    t1 = 2.0 * rho / p1 ** 0.5
    t2 = rho ** 3 / p1 ** 1.5
    ai = a[:, None, :]
    aj = a[None, :, :]
    q1 = (ai * aj).sum(-1)
    q2 = (u * ai).sum(-1)
    q3 = (u * aj).sum(-1)
    e = (t1 * q1 + t2 * (q2 * q3 - q1)) / rn
    e = torch.where(off, e, torch.zeros_like(e))
    return e.sum() / (16.0 * math.pi)


def rhs(x, a, sigma, nu=None):
    rate = stretching(x, a, sigma)
    if nu is not None:
        rate = rate + pse(x, a, sigma, nu)
    return velocity(x, a, sigma), rate


def rk4_trajectory(x, a, sigma, nu, dt, steps):
    for _ in range(steps):
        k1x, k1a = rhs(x, a, sigma, nu)
        k2x, k2a = rhs(x + (dt / 2) * k1x, a + (dt / 2) * k1a, sigma, nu)
        k3x, k3a = rhs(x + (dt / 2) * k2x, a + (dt / 2) * k2a, sigma, nu)
        k4x, k4a = rhs(x + dt * k3x, a + dt * k3a, sigma, nu)
        x = x + (dt / 6) * (k1x + 2 * k2x + 2 * k3x + k4x)
        a = a + (dt / 6) * (k1a + 2 * k2a + 2 * k3a + k4a)
    return x, a
