"""Pin the dense FP64 torch restatement (the autograd reference for the adjoint kernels) to
the oracle, on CPU."""
import numpy as np
import torch

import oracle
from oracle import vpm_dense
from conftest import normwise


def _field(n=120, seed=3):
    from openonda_b200 import configs

    f = configs.random_cloud(n, seed=seed)
    f.radii *= 6
    f.viscosities = np.random.default_rng(seed).uniform(1e-4, 3e-4, n)
    return f


def test_dense_forward_matches_oracle():
    f = _field()
    t = lambda z: torch.from_numpy(z)
    x, a, s, v = t(f.positions), t(f.strengths), t(f.radii), t(f.viscosities)
    assert normwise(vpm_dense.velocity(x, a, s).numpy(),
                    oracle.gpu.get_selfinduced_velocity(f.positions, f.strengths, f.radii)) <= 1e-13
    assert normwise(vpm_dense.stretching(x, a, s).numpy(),
                    oracle.gpu.get_strength_gradients(f.positions, f.strengths, f.radii)) <= 1e-13
    assert normwise(vpm_dense.pse(x, a, s, v).numpy(),
                    oracle.gpu.get_strength_gradients_PSE(f.positions, f.strengths, f.radii,
                                                          f.viscosities)) <= 1e-13
    ke = float(vpm_dense.kinetic_energy(x, a, s))
    ref = oracle.gpu.get_total_kinetic_energy(f.positions, f.strengths, f.radii)
    assert abs(ke - ref) <= 1e-12 * abs(ref)


def test_dense_gradient_is_finite_and_consistent():
    f = _field(40, 5)
    x = torch.from_numpy(f.positions).requires_grad_()
    a = torch.from_numpy(f.strengths).requires_grad_()
    s = torch.from_numpy(f.radii).requires_grad_()
    e = vpm_dense.kinetic_energy(x, a, s)
    gx, ga, gs = torch.autograd.grad(e, (x, a, s))
    # central difference on one coordinate of each input
    h = 1e-6
    for t, g in ((x, gx), (a, ga), (s, gs)):
        idx = (3,) + ((1,) if t.dim() == 2 else ())
        with torch.no_grad():
            t0 = t[idx].item()
            t[idx] = t0 + h
            ep = float(vpm_dense.kinetic_energy(x, a, s))
            t[idx] = t0 - h
            em = float(vpm_dense.kinetic_energy(x, a, s))
            t[idx] = t0
        fd = (ep - em) / (2 * h)
        assert abs(fd - g[idx].item()) <= 1e-6 * max(abs(fd), 1e-12)
