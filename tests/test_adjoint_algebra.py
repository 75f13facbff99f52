"""CPU check of the adjoint algebra: a numpy transcription of the per-pair formulas used by
the sweep kernels (csrc/vpm_adjoint.cuh: OpRhsVjp, OpKeGrad and their finalize passes) must
reproduce torch.autograd on the dense FP64 restatement of the reference kernels."""
import math

import numpy as np
import pytest
import torch

from oracle import vpm_dense
from conftest import normwise

C = 1.0 / (4.0 * math.pi)


def _field(n, seed):
    from openonda_b200 import configs

    f = configs.random_cloud(n, seed=seed)
    f.radii *= 6
    rng = np.random.default_rng(seed + 100)
    return (f.positions, f.strengths, f.radii, rng.uniform(1e-4, 3e-4, n),
            rng.normal(size=(n, 3)), rng.normal(size=(n, 3)))


def vjp_transcription(x, a, sig, nu, gu, gs, pse):
    """The kernel's symmetric gather, vectorised over all pairs (k: rows, l: columns)."""
    n = len(x)
    up, sp = -C * gu, C * gs          # pre-scaled cotangents
    nup = 105.0 * nu if pse else np.zeros(n)
    r = x[:, None, :] - x[None, :, :]
    s = 0.5 * (sig[:, None] + sig[None, :])
    s2 = s * s
    xx = (r * r).sum(-1) + s2
    y = 1.0 / np.sqrt(xx)
    np.fill_diagonal(y, 0.0)
    y2 = y * y
    y5 = y2 * y2 * y
    y7 = y5 * y2
    y9 = y7 * y2
    s3 = s2 * s
    t1 = xx + 1.5 * s2
    g = t1 * y5
    t2 = t1 + s2
    f = 3.0 * t2 * y7
    gs_ = -7.5 * s3 * y7
    f2r = -15.0 * (t2 + s2) * y9
    fs = -52.5 * s3 * y9
    al = np.broadcast_to(a[None, :, :], r.shape)
    ak = np.broadcast_to(a[:, None, :], r.shape)
    cl = np.cross(r, al)
    ck = np.cross(r, ak)
    w = np.cross(al, ak)
    ds = sp[:, None, :] - sp[None, :, :]
    eT = (up[:, None, :] * cl).sum(-1)
    eS = (up[None, :, :] * ck).sum(-1)
    E = (eT - eS) - (ds * w).sum(-1)
    d = (r * w).sum(-1)
    dp = (ds * r).sum(-1)
    D = d * dp
    cr = f2r * D - f * E
    sd = gs_ * E + fs * D
    gx = (cr[..., None] * r + (f * dp)[..., None] * w + (f * d)[..., None] * ds).sum(1)
    Ga = (g[..., None] * al).sum(1)
    Gu = (g[..., None] * up[None, :, :]).sum(1)
    nvec = np.cross(r, np.broadcast_to(up[None, :, :], r.shape)) - np.cross(
        al, np.broadcast_to(sp[None, :, :], r.shape))
    ga = (g[..., None] * nvec + (f * dp)[..., None] * cl).sum(1)
    gnu = None
    if pse:
        z = s * y
        k = z ** 7 * y2
        k2r = -9.0 * k * y2
        ks = z ** 6 * y ** 5 * (7.0 * (xx - s2) - 2.0 * s2)
        dd = al - ak
        qT = (sp[:, None, :] * dd).sum(-1)
        qS = (sp[None, :, :] * dd).sum(-1)
        Q = nup[:, None] * qT - nup[None, :] * qS
        cr2 = k2r * Q
        gx = gx + (cr2[..., None] * r).sum(1)
        sd = sd + ks * Q
        gnu = 105.0 * (k * qT).sum(1)
        ga = ga + ((k * nup[None, :])[..., None] * sp[None, :, :]).sum(1) \
            - k.sum(1)[:, None] * nup[:, None] * sp
    gx = gx + np.cross(Ga, up) - np.cross(a, Gu)
    ga = ga + np.cross(Ga, sp)
    gsig = 0.5 * sd.sum(1)
    return gx, ga, gsig, gnu


def kegrad_transcription(x, a, sig):
    r = x[:, None, :] - x[None, :, :]
    s = 0.5 * (sig[:, None] + sig[None, :])
    s2 = s * s
    xx = (r * r).sum(-1) + s2
    y = 1.0 / np.sqrt(xx)
    np.fill_diagonal(y, 0.0)
    y3 = y ** 3
    y5 = y ** 5
    w = y + s2 * y3
    al = np.broadcast_to(a[None, :, :], r.shape)
    ak = np.broadcast_to(a[:, None, :], r.shape)
    p1 = (ak * al).sum(-1)
    rl = (r * al).sum(-1)
    rk = (r * ak).sum(-1)
    rr = rk * rl
    q = y3 * rl
    ga = (w[..., None] * al + q[..., None] * r).sum(1)
    h2r = -(p1 * (3 * s2 * y5 + y3) + 3 * y5 * rr)
    gx = (h2r[..., None] * r + q[..., None] * ak + (y3 * rk)[..., None] * al).sum(1)
    hs = s * (p1 * (y3 - 3 * s2 * y5) - 3 * y5 * rr)
    c = 2.0 / (16.0 * math.pi)
    return c * gx, c * ga, 0.5 * c * hs.sum(1)


@pytest.mark.parametrize("pse", [False, True])
def test_rhs_vjp_algebra_matches_autograd(pse):
    x, a, s, nu, gu, gs = _field(90, 7)
    t = lambda z: torch.from_numpy(np.array(z)).requires_grad_()
    tx, ta, ts, tn = t(x), t(a), t(s), t(nu)
    u, rate = vpm_dense.rhs(tx, ta, ts, tn if pse else None)
    L = (u * torch.from_numpy(gu)).sum() + (rate * torch.from_numpy(gs)).sum()
    grads = torch.autograd.grad(L, (tx, ta, ts, tn) if pse else (tx, ta, ts))
    gx, ga, gsig, gnu = vjp_transcription(x, a, s, nu, gu, gs, pse)
    assert normwise(gx, grads[0].numpy()) <= 1e-11
    assert normwise(ga, grads[1].numpy()) <= 1e-11
    assert normwise(gsig, grads[2].numpy()) <= 1e-11
    if pse:
        assert normwise(gnu, grads[3].numpy()) <= 1e-11


def test_kinetic_energy_gradient_algebra_matches_autograd():
    x, a, s, _, _, _ = _field(90, 8)
    t = lambda z: torch.from_numpy(np.array(z)).requires_grad_()
    tx, ta, ts = t(x), t(a), t(s)
    grads = torch.autograd.grad(vpm_dense.kinetic_energy(tx, ta, ts), (tx, ta, ts))
    gx, ga, gsig = kegrad_transcription(x, a, s)
    assert normwise(gx, grads[0].numpy()) <= 1e-11
    assert normwise(ga, grads[1].numpy()) <= 1e-11
    assert normwise(gsig, grads[2].numpy()) <= 1e-11
