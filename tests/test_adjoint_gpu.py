"""Differentiation form on the GPU: hand-written adjoint kernels against FP64 torch.autograd
on the dense restatement (oracle/vpm_dense.py, pinned to the oracle), FP32-compensated
adjoint against the FP64 adjoint, and trajectory gradients (RK4 with segment checkpointing)
against autograd and central finite differences.  The reference has no adjoint, so parity
here is anchored on the pinned forward, not on a reference gradient."""
import numpy as np
import pytest
import torch

from oracle import vpm_dense
from conftest import normwise

pytestmark = pytest.mark.gpu


def _field(n, seed, scale=6.0):
    from openonda_b200 import configs

    f = configs.random_cloud(n, seed=seed)
    f.radii *= scale
    rng = np.random.default_rng(seed + 100)
    return f.positions, f.strengths, f.radii, rng.uniform(1e-4, 3e-4, n)


def _cuda(*arrs):
    return [torch.from_numpy(np.array(z)).cuda() for z in arrs]


@pytest.mark.parametrize("pse", [False, True])
@pytest.mark.parametrize("n", [97, 300])
def test_rhs_vjp_kernel_vs_dense_autograd(n, pse):
    from openonda_b200 import autodiff

    x, a, s, nu = _field(n, 11)
    rng = np.random.default_rng(5)
    gu, gs = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    t = lambda z: torch.from_numpy(np.array(z)).requires_grad_()
    tx, ta, ts, tn = t(x), t(a), t(s), t(nu)
    u, rate = vpm_dense.rhs(tx, ta, ts, tn if pse else None)
    L = (u * torch.from_numpy(gu)).sum() + (rate * torch.from_numpy(gs)).sum()
    ref = torch.autograd.grad(L, (tx, ta, ts, tn) if pse else (tx, ta, ts))
    cx, ca, cs, cn, cgu, cgs = _cuda(x, a, s, nu, gu, gs)
    gx, ga, gsig, gnu = autodiff.rhs_vjp(cx, ca, cs, cn if pse else None, cgu, cgs, "fp64")
    assert normwise(gx.cpu().numpy(), ref[0].numpy()) <= 1e-11
    assert normwise(ga.cpu().numpy(), ref[1].numpy()) <= 1e-11
    assert normwise(gsig.cpu().numpy(), ref[2].numpy()) <= 1e-11
    if pse:
        assert normwise(gnu.cpu().numpy(), ref[3].numpy()) <= 1e-11


def test_kinetic_energy_grad_kernel_vs_dense_autograd():
    from openonda_b200 import autodiff

    x, a, s, _ = _field(200, 12)
    t = lambda z: torch.from_numpy(np.array(z)).requires_grad_()
    tx, ta, ts = t(x), t(a), t(s)
    ref = torch.autograd.grad(vpm_dense.kinetic_energy(tx, ta, ts), (tx, ta, ts))
    gx, ga, gs = autodiff.kinetic_energy_grad(*_cuda(x, a, s), precision="fp64")
    assert normwise(gx.cpu().numpy(), ref[0].numpy()) <= 1e-11
    assert normwise(ga.cpu().numpy(), ref[1].numpy()) <= 1e-11
    assert normwise(gs.cpu().numpy(), ref[2].numpy()) <= 1e-11


@pytest.mark.parametrize("pse", [False, True])
def test_fp32c_adjoint_vs_fp64_adjoint(pse):
    from openonda_b200 import autodiff, configs

    f = configs.perturbed_ring(64, 64)  # N = 4096
    rng = np.random.default_rng(3)
    n = f.n
    gu, gs = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    r32 = lambda z: np.asarray(z, np.float32).astype(np.float64)
    cx, ca, cs, cn, cgu, cgs = _cuda(r32(f.positions), r32(f.strengths), r32(f.radii),
                                     r32(f.viscosities), gu, gs)
    nu = cn if pse else None
    g64 = autodiff.rhs_vjp(cx, ca, cs, nu, cgu, cgs, "fp64")
    g32 = autodiff.rhs_vjp(cx, ca, cs, nu, cgu, cgs, "fp32c")
    for k in range(3):
        e = normwise(g32[k].cpu().numpy(), g64[k].cpu().numpy())
        print(f"fp32c adjoint output {k}: {e:.2e}")
        assert e <= 1e-5


def test_trajectory_gradient_vs_dense_autograd():
    from openonda_b200 import autodiff

    x, a, s, nu = _field(128, 21, scale=8.0)
    dt, steps = 0.01, 5
    t = lambda z: torch.from_numpy(np.array(z)).requires_grad_()
    tx, ta, ts = t(x), t(a), t(s)
    xT, aT = vpm_dense.rk4_trajectory(tx, ta, ts, None, dt, steps)
    ref = torch.autograd.grad(vpm_dense.kinetic_energy(xT, aT, ts), (tx, ta, ts))
    cx, ca, cs = [z.requires_grad_() for z in _cuda(x, a, s)]
    xT, aT = autodiff.trajectory(cx, ca, cs, None, dt, steps, "fp64", checkpoint_every=2)
    e = autodiff.kinetic_energy(xT, aT, cs, "fp64")
    g = torch.autograd.grad(e, (cx, ca, cs))
    for k in range(3):
        assert normwise(g[k].cpu().numpy(), ref[k].numpy()) <= 1e-10, k


@pytest.mark.parametrize("every", [0, None])
def test_trajectory_without_checkpointing_matches_checkpointed(every):
    """checkpoint_every 0 or None keeps every state (no recompute) and gives the same
    gradient as segment checkpointing."""
    from openonda_b200 import autodiff

    x, a, s, _ = _field(256, 22, scale=8.0)
    dt, steps = 0.01, 3
    grads = []
    for ck in (every, 2):
        cx, ca, cs = [z.requires_grad_() for z in _cuda(x, a, s)]
        xT, aT = autodiff.trajectory(cx, ca, cs, None, dt, steps, "fp64", checkpoint_every=ck)
        e = autodiff.kinetic_energy(xT, aT, cs, "fp64")
        grads.append(torch.autograd.grad(e, (cx, ca, cs)))
    for u, v in zip(*grads):
        assert torch.equal(u, v)


def test_trajectory_gradient_vs_central_differences():
    from openonda_b200 import autodiff, configs

    f = configs.perturbed_ring(16, 24)  # N = 384
    x, a, s = _cuda(f.positions, f.strengths, f.radii)
    nu = _cuda(f.viscosities)[0]
    dt, steps = 0.01, 6

    def loss(xx, aa, ss):
        xT, aT = autodiff.trajectory(xx, aa, ss, nu, dt, steps, "fp64", checkpoint_every=3)
        return autodiff.kinetic_energy(xT, aT, ss, "fp64")

    xg, ag, sg = [z.clone().requires_grad_() for z in (x, a, s)]
    g = torch.autograd.grad(loss(xg, ag, sg), (xg, ag, sg))
    rng = np.random.default_rng(9)
    h = 1e-6
    with torch.no_grad():
        for which, base in enumerate((x, a, s)):
            for _ in range(4):
                idx = tuple(int(rng.integers(0, d)) for d in base.shape)
                scale = float(base.abs().max()) if which == 1 else 1.0
                step = h * scale
                bp, bm = base.clone(), base.clone()
                bp[idx] += step
                bm[idx] -= step
                args_p = [x, a, s]
                args_m = [x, a, s]
                args_p[which], args_m[which] = bp, bm
                fd = (float(loss(*args_p)) - float(loss(*args_m))) / (2 * step)
                ad = float(g[which][idx])
                assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)) + 1e-9 * float(
                    g[which].abs().max()), (which, idx, fd, ad)


def test_adjoint_is_deterministic():
    from openonda_b200 import autodiff

    x, a, s, nu = _cuda(*_field(5000, 4))
    gu, gs = torch.randn_like(x), torch.randn_like(a)
    for prec in ("fp64", "fp32c"):
        g1 = autodiff.rhs_vjp(x, a, s, nu, gu, gs, prec)
        g2 = autodiff.rhs_vjp(x, a, s, nu, gu, gs, prec)
        for u, v in zip(g1, g2):
            assert torch.equal(u, v)
