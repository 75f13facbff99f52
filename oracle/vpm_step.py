"""Step-level oracle: numpy restatement of ``vpmModule.ParticleSystem``'s time step
(TEST INFRASTRUCTURE, not product code).

It reproduces the reference's sequencing exactly, including its quirks, so that the
device-resident ``ParticleSystem`` can be checked step by step:

* ``update_velocities`` (vpmModule.py:699-710): one self-induced velocity sweep.
* ``update_strengths`` (vpmModule.py:713-884): LES filter update first (vorticity sweep,
  enstrophy sweep, Cnu and nu_t, :731-737); stretching with Euler/BDF2/BDF3/BDF4 by
  ``time_step`` (:749-780) and history update (:783-787); PSE with the same BDF ladder on
  the post-stretching strengths (:797-841) -- the BDF history is therefore rewritten twice
  per step; or core spreading ``sigma <- sqrt(sigma^2 + 5.34 nu_eff dt)`` (:851-860).
* ``update_state`` (vpmModule.py:522-560): RK position update where stage 1 reuses the
  velocities of ``update_velocities`` (computed with the OLD strengths) and later stages
  use the NEW strengths (:583-692); the "RK3" is the reference's midpoint variant
  (:617-651).
* ``_update_LES_filter_constant`` (:887-909) and ``_update_LES_particles_viscosity``
  (:916-962), with epsilon = 1e-9 (vpmModule.py:22).

``physics`` is any object exposing the reference function names (the oracle's ``gpu`` or
``cpu`` module).  The relaxation branch (:867-883) raises in the reference (it divides an
(N,3) array by an (N,) array); here it normalises row-wise, the evident intent.
"""
from __future__ import annotations

import numpy as np

EPS_MODULE = 1e-9


class StepOracle:
    def __init__(self, physics, positions, strengths, radii, viscosities, *,
                 time_step_size=0.01, time_integration_method="RK4", flow_model="DNS",
                 viscous_scheme="PSE", relax_strength_solution=False, time_step=0):
        self.physics = physics
        self.x = np.array(positions, dtype=np.float64)
        self.a = np.array(strengths, dtype=np.float64)
        self.s = np.array(radii, dtype=np.float64)
        self.nu = np.array(viscosities, dtype=np.float64)
        self.nut = np.zeros_like(self.nu)
        self.u = np.zeros_like(self.x)
        self.dt = float(time_step_size)
        self.method = time_integration_method
        self.flow_model = flow_model
        self.viscous_scheme = viscous_scheme
        self.relax = relax_strength_solution
        self.time_step = int(time_step)
        self.flow_time = 0.0
        self.Cnu = 0.02958
        self.enstrophy_ref = None
        self.prev1 = None
        self.prev2 = None
        self.prev3 = None

    # -- update_velocities ------------------------------------------------------------
    def update_velocities(self):
        self.u = self.physics.get_selfinduced_velocity(self.x, self.a, self.s)

    # -- BDF ladder shared by stretching and PSE (vpmModule.py:751-787, :801-841) ------
    def _bdf(self, strengths, rate):
        dt, k = self.dt, self.time_step
        if k == 0:
            new = strengths + dt * rate
        elif k == 1:
            new = (4 * strengths - self.prev1) / 3 + (2 / 3) * dt * rate
        elif k == 2:
            new = (18 * strengths - 9 * self.prev1 + 2 * self.prev2) / 11 + (6 / 11) * dt * rate
        else:
            new = ((48 * strengths - 36 * self.prev1 + 16 * self.prev2 - 3 * self.prev3) / 25
                   + (12 / 25) * dt * rate)
        if k >= 3:
            self.prev3 = self.prev2.copy()
        if k >= 2:
            self.prev2 = self.prev1.copy()
        self.prev1 = new.copy()
        return new

    # -- update_strengths -------------------------------------------------------------
    def update_strengths(self):
        if self.flow_model == "Potential":
            return
        x, a, s = self.x, self.a.copy(), self.s
        if self.flow_model == "LES":
            w = self.physics.get_vorticity_field_at(x, x, a, s)
            ens = self.physics.get_total_enstrophy(x, a, s)
            self._update_les_constant(ens)
            self._update_les_viscosity(w, s)
        if self.prev1 is None:
            self.prev1 = np.zeros_like(a)
            self.prev2 = np.zeros_like(a)
            self.prev3 = np.zeros_like(a)
        if self.flow_model in ("LES", "DNS"):
            rate = self.physics.get_strength_gradients(x, a, s)
            a = self._bdf(a, rate)
            self.a = a.copy()
        if self.viscous_scheme == "PSE":
            nu_eff = self.nu + self.nut
            rate = self.physics.get_strength_gradients_PSE(x, a, s, nu_eff)
            a = self._bdf(a, rate)
            self.a = a.copy()
        elif self.viscous_scheme == "CoreSpreading":
            nu_eff = self.nu + self.nut
            self.s = np.sqrt(s ** 2 + 5.34 * nu_eff * self.dt)
        if self.relax:
            alpha = 0.95
            w = self.physics.get_vorticity_field_at(self.x, self.x, self.a, self.s)
            wn = np.sqrt(np.sum(w * w, axis=1))
            an = np.sqrt(np.sum(self.a * self.a, axis=1))
            self.a = self.a * alpha + (1 - alpha) * (w / wn[:, None]) * an[:, None]

    def _update_les_constant(self, enstrophy):
        rms = np.sqrt(enstrophy)
        if self.enstrophy_ref is None:
            self.enstrophy_ref = rms
        self.enstrophy_ref = 0.1 * rms + 0.9 * self.enstrophy_ref
        self.Cnu *= rms / (self.enstrophy_ref + EPS_MODULE)
        self.Cnu = max(EPS_MODULE, min(self.Cnu, 0.0761))

    def _update_les_viscosity(self, w, radii):
        beta0 = np.pi / 4
        wm = np.sqrt(np.sum(w * w, axis=1))
        wu = w / wm[:, None]
        wa = np.mean(w, axis=0)
        wau = wa / np.sqrt(np.sum(wa * wa))
        beta = np.arccos(np.clip(wu @ wau, -1.0, 1.0))
        psi = np.where((beta0 <= beta) & (beta <= np.pi - beta0), 1.0, 0.0)
        nut = psi * (self.Cnu * radii) ** 2 * wm
        if np.max(nut) > EPS_MODULE:
            self.nut = nut

    # -- update_state -----------------------------------------------------------------
    def update_state(self):
        x, u, dt = self.x, self.u, self.dt
        vel = self.physics.get_selfinduced_velocity
        a, s = self.a, self.s
        if self.method == "Euler":
            xn = x + u * dt
        elif self.method == "RK2":
            k2 = vel(x + u * (dt * 0.5), a, s)
            xn = x + k2 * dt
        elif self.method == "RK3":
            k2 = vel(x + u * (dt / 2), a, s)
            k3 = vel(x + (dt / 2) * k2, a, s)
            xn = x + dt * k3
        elif self.method == "RK4":
            k2 = vel(x + (dt / 2) * u, a, s)
            k3 = vel(x + (dt / 2) * k2, a, s)
            k4 = vel(x + dt * k3, a, s)
            xn = x + (dt / 6) * (u + 2 * k2 + 2 * k3 + k4)
        else:
            raise ValueError(self.method)
        self.flow_time += dt
        self.time_step += 1
        self.x = xn

    def step(self):
        self.update_velocities()
        self.update_strengths()
        self.update_state()
