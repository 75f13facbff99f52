"""Differentiation form: autograd through the B200 pair sums with hand-written adjoints.

The reference has no adjoint.  This module makes trajectories of the coupled VPM ODE

    dx/dt = u(x, alpha, sigma),   dalpha/dt = S(x, alpha, sigma) [+ P(x, alpha, sigma, nu)]

(u, S, P: the self-induced velocity, stretching and PSE sums of ParticlesPhysicsCuda.py)
differentiable with respect to initial positions, strengths, core sizes and viscosities:

* :class:`RHS` -- forward: the fused velocity + stretching sweep (+ the PSE sweep); backward:
  one ``vpm_rhs_vjp`` sweep (symmetric gather over all pairs, no atomics).
* :class:`KineticEnergy` -- forward: the FP64-summed kinetic energy sweep; backward:
  ``vpm_kinetic_energy_grad``.
* :func:`trajectory` -- classical RK4 on (x, alpha) with segment checkpointing: only the
  state at every ``checkpoint_every``-th step is kept, and each segment's forward is
  recomputed during the backward pass.

All tensors are CUDA float64; ``precision`` selects the FP64 or FP32-compensated kernels.
"""
from __future__ import annotations

import torch
from torch.utils.checkpoint import checkpoint

from . import _lib, kernels

_F64 = torch.float64


def rhs_vjp(x, a, sigma, nu, grad_u, grad_rate, precision="fp64"):
    """(dL/dx, dL/dalpha, dL/dsigma, dL/dnu) for cotangents of (u, S [+ P]).

    ``nu=None`` differentiates (u, S) without PSE; dL/dnu is then None."""
    x, a, s, n, dev = kernels._self_inputs(x, a, sigma)
    gu = kernels._check_vec("grad_u", grad_u, n)
    gr = kernels._check_vec("grad_rate", grad_rate, n)
    v = None if nu is None else kernels._check_scalar("nu", nu, n)
    op = "rhs_vjp" if v is None else "rhs_vjp_pse"
    gx = torch.empty((n, 3), dtype=_F64, device=dev)
    ga = torch.empty((n, 3), dtype=_F64, device=dev)
    gs = torch.empty((n,), dtype=_F64, device=dev)
    gnu = None if v is None else torch.empty((n,), dtype=_F64, device=dev)
    ws, _ = kernels._workspace(op, precision, n, n, dev)
    _lib.check(_lib.load().vpm_rhs_vjp(
        x.data_ptr(), a.data_ptr(), s.data_ptr(), kernels._ptr(v), n, gu.data_ptr(),
        gr.data_ptr(), gx.data_ptr(), ga.data_ptr(), gs.data_ptr(), kernels._ptr(gnu),
        _lib.precision_code(precision), ws.data_ptr(), ws.numel(), kernels._stream(dev)))
    return gx, ga, gs, gnu


def kinetic_energy_grad(x, a, sigma, precision="fp64"):
    """(dE/dx, dE/dalpha, dE/dsigma) of the total kinetic energy."""
    x, a, s, n, dev = kernels._self_inputs(x, a, sigma)
    gx = torch.empty((n, 3), dtype=_F64, device=dev)
    ga = torch.empty((n, 3), dtype=_F64, device=dev)
    gs = torch.empty((n,), dtype=_F64, device=dev)
    ws, _ = kernels._workspace("kinetic_energy_grad", precision, n, n, dev)
    _lib.check(_lib.load().vpm_kinetic_energy_grad(
        x.data_ptr(), a.data_ptr(), s.data_ptr(), n, gx.data_ptr(), ga.data_ptr(),
        gs.data_ptr(), _lib.precision_code(precision), ws.data_ptr(), ws.numel(),
        kernels._stream(dev)))
    return gx, ga, gs


class RHS(torch.autograd.Function):
    """(u, S [+ P]) with a hand-written vector-Jacobian product."""

    @staticmethod
    def forward(ctx, x, a, sigma, nu, precision, with_pse, uniform_core=False):
        u, rate = kernels.velocity_and_strength_gradients(x, a, sigma, precision=precision,
                                                          uniform_core=uniform_core)
        if with_pse:
            rate = rate + kernels.strength_gradients_pse(x, a, sigma, nu, precision=precision,
                                                         uniform_core=uniform_core)
        ctx.save_for_backward(x, a, sigma, nu if with_pse else None)
        ctx.precision, ctx.with_pse = precision, with_pse
        return u, rate

    @staticmethod
    def backward(ctx, grad_u, grad_rate):
        x, a, sigma, nu = ctx.saved_tensors
        if grad_u is None:
            grad_u = torch.zeros_like(x)
        if grad_rate is None:
            grad_rate = torch.zeros_like(a)
        gx, ga, gs, gnu = rhs_vjp(x, a, sigma, nu if ctx.with_pse else None,
                                  grad_u.contiguous(), grad_rate.contiguous(), ctx.precision)
        return gx, ga, gs, gnu, None, None, None


class KineticEnergy(torch.autograd.Function):
    """Total kinetic energy (FP64 sum) with a hand-written gradient."""

    @staticmethod
    def forward(ctx, x, a, sigma, precision):
        ctx.save_for_backward(x, a, sigma)
        ctx.precision = precision
        return kernels.total_kinetic_energy(x, a, sigma, precision=precision)

    @staticmethod
    def backward(ctx, grad_e):
        x, a, sigma = ctx.saved_tensors
        gx, ga, gs = kinetic_energy_grad(x, a, sigma, ctx.precision)
        return gx * grad_e, ga * grad_e, gs * grad_e, None


def rhs(x, a, sigma, nu=None, precision="fp64", uniform_core=False):
    """Differentiable (u, dalpha/dt); PSE is included when ``nu`` is given.  With
    ``uniform_core`` (all cores equal) the forward sums take the uniform-core form."""
    with_pse = nu is not None
    return RHS.apply(x, a, sigma, nu if with_pse else torch.zeros_like(sigma), precision,
                     with_pse, bool(uniform_core))


def kinetic_energy(x, a, sigma, precision="fp64"):
    return KineticEnergy.apply(x, a, sigma, precision)


def rk4_step(x, a, sigma, nu, dt, precision="fp64", uniform_core=False):
    """One classical RK4 step of (x, alpha) with frozen sigma and nu."""
    uc = uniform_core
    k1x, k1a = rhs(x, a, sigma, nu, precision, uc)
    k2x, k2a = rhs(x + (dt / 2) * k1x, a + (dt / 2) * k1a, sigma, nu, precision, uc)
    k3x, k3a = rhs(x + (dt / 2) * k2x, a + (dt / 2) * k2a, sigma, nu, precision, uc)
    k4x, k4a = rhs(x + dt * k3x, a + dt * k3a, sigma, nu, precision, uc)
    x1 = x + (dt / 6) * (k1x + 2 * k2x + 2 * k3x + k4x)
    a1 = a + (dt / 6) * (k1a + 2 * k2a + 2 * k3a + k4a)
    return x1, a1


def trajectory(x0, a0, sigma, nu=None, dt=0.01, steps=10, precision="fp64",
               checkpoint_every=10):
    """Integrate ``steps`` RK4 steps; differentiable w.r.t. x0, a0, sigma (and nu).

    With autograd active, every segment of ``checkpoint_every`` steps is recomputed in the
    backward pass (only segment-start states are stored); ``checkpoint_every`` 0 or None
    keeps every intermediate state instead.  sigma is frozen along the trajectory, so equal
    cores (checked once) select the uniform-core forward sums."""
    if checkpoint_every is not None and checkpoint_every < 0:
        raise ValueError(f"checkpoint_every must be >= 0 or None, got {checkpoint_every}")
    if steps < 0:
        raise ValueError(f"steps must be >= 0, got {steps}")
    x, a = x0, a0
    with torch.no_grad():
        uc = sigma.numel() > 0 and bool((sigma == sigma.reshape(-1)[0]).all())

    def segment(xs, as_, sig, visc, n_steps):
        for _ in range(n_steps):
            xs, as_ = rk4_step(xs, as_, sig, visc, dt, precision, uc)
        return xs, as_

    done = 0
    while done < steps:
        k = min(checkpoint_every or steps, steps - done)
        if torch.is_grad_enabled() and checkpoint_every and (x.requires_grad or a.requires_grad
                                                             or sigma.requires_grad):
            x, a = checkpoint(segment, x, a, sigma, nu, k, use_reentrant=False)
        else:
            x, a = segment(x, a, sigma, nu, k)
        done += k
    return x, a
