"""FP64 numpy restatement of the least-squares dynamic LES coefficient (TEST INFRASTRUCTURE,
not product code).

The reference has no least-squares procedure: it only rescales Cnu by the ratio of the
enstrophy to its smoothed reference (OpenONDA/solvers/VPM/vpmModule.py:887-909).  This is the
checker of the library's own procedure (vpm_les_lsq_weights / vpm_les_lsq_update and
ParticleSystem(les_coefficient="least_squares")), so its parity is unpinned: it pins the
implementation to the written-down mathematics, not to a reference.

Germano identity for the sub-filter kinetic energy k(D) = C^2 D^2 |w_D|^2 between the particle
filter (core sigma) and a test filter of core 2 sigma, least squares over all particles:

    L_i = (hat(|u|^2)_i - |hat u_i|^2) / 2
    M_i = (2 sigma_i)^2 |hat w_i|^2 - hat(sigma^2 |w|^2)_i
    Cnu = clip(sqrt(sum L M / sum M M), 1e-9, 0.0761)   (unchanged if either sum <= 0)

u and w are the particle velocity and vorticity (reference GPU semantics); hat u is the
Biot-Savart velocity with cores 2 sigma, hat w the vorticity filter sum with cores 2 sigma, and
hat f_i = sum_j zeta_{2 sigma_j}(x_i - x_j) f_j v_j with the particle volume v_j = |a_j|/|w_j|.
The pair sums come from the pinned C oracle (``oracle.gpu``); the rest is plain numpy.
"""
from __future__ import annotations

import numpy as np

EPS = 1e-9
CNU_MAX = 0.0761


def lsq_sums(physics, x, a, sigma, u=None, w=None):
    """(sum L M, sum M M) of the procedure; ``physics`` exposes the reference function names
    (``oracle.gpu``)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    a = np.ascontiguousarray(a, dtype=np.float64)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64)
    if u is None:
        u = physics.get_selfinduced_velocity(x, a, sigma)
    if w is None:
        w = physics.get_vorticity_field_at(x, x, a, sigma)
    s2 = 2.0 * sigma
    uh = physics.get_selfinduced_velocity(x, a, s2)
    wh = physics.get_vorticity_field_at(x, x, a, s2)
    wn2 = np.sum(w * w, axis=1)
    vol = np.where(wn2 > 0.0, np.sqrt(np.sum(a * a, axis=1)) / np.sqrt(np.where(wn2 > 0, wn2, 1)),
                   0.0)
    f = np.zeros_like(a)
    f[:, 0] = np.sum(u * u, axis=1) * vol
    f[:, 1] = sigma * sigma * wn2 * vol
    fh = physics.get_vorticity_field_at(x, x, f, s2)
    L = 0.5 * (fh[:, 0] - np.sum(uh * uh, axis=1))
    M = (2.0 * sigma) ** 2 * np.sum(wh * wh, axis=1) - fh[:, 1]
    return float(np.sum(L * M)), float(np.sum(M * M))


def lsq_coefficient(physics, x, a, sigma, cnu_old, u=None, w=None):
    """The updated Cnu."""
    lm, mm = lsq_sums(physics, x, a, sigma, u, w)
    if mm > 0.0 and lm > 0.0:
        return max(EPS, min(np.sqrt(lm / mm), CNU_MAX))
    return cnu_old
