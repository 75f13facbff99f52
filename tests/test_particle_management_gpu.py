"""Device-resident ParticleSystem beyond the time step: O(N) diagnostics and particle-field
control against the reference ParticleSystem's own outputs (tests/golden/manage.npz), probe
fields against the oracle, exact checkpoint/resume, and subdivision as the reference's
source describes it (vpmModule.py:1040-1094; the reference method itself calls a missing
getter, :1065)."""
import os

import numpy as np
import pytest

import oracle
from conftest import golden, normwise

pytestmark = pytest.mark.gpu


def _system(tmp_path, g=None, **cfg):
    from openonda_b200.vpm.vpmModule import ParticleSystem

    ps = ParticleSystem(monitor_variables=[], backup_frequency=10 ** 9,
                        backup_filename=str(tmp_path / "b"), **cfg)
    if g is not None:
        x = g["field/positions"]
        ps.add_particle_field(x, np.zeros_like(x), g["field/strengths"], g["field/radii"],
                              g["field/viscosities"])
    return ps


def test_diagnostics_vs_reference(tmp_path):
    g = golden("manage.npz")
    ps = _system(tmp_path, g)
    assert normwise(ps.get_total_linear_impulse(), g["diag/linear_impulse"]) <= 1e-13
    assert normwise(ps.get_total_angular_impulse(), g["diag/angular_impulse"]) <= 1e-13
    assert normwise(ps.get_total_strength(), g["diag/total_strength"]) <= 1e-13
    ref = float(g["diag/total_strength_magnitude"])
    assert abs(ps.get_total_strength_magnitude() - ref) <= 1e-13 * ref


@pytest.mark.parametrize("case", ["relative_conserve", "absolute"])
def test_remove_weak_particles_vs_reference(tmp_path, case):
    g = golden("manage.npz")
    ps = _system(tmp_path, g)
    mode = "relative" if case.startswith("relative") else "absolute"
    ps.remove_weak_particles(mode, float(g[f"{case}/threshold"]),
                             conserve_total_circulation=(case == "relative_conserve"))
    assert len(ps) == g[f"{case}/positions"].shape[0]
    assert np.array_equal(ps.get_particle_positions(), g[f"{case}/positions"])
    assert np.array_equal(ps.get_particle_radii(), g[f"{case}/radii"])
    assert normwise(ps.get_particle_strengths(), g[f"{case}/strengths"]) <= 1e-15


def test_subdivide_strong_particles(tmp_path):
    g = golden("manage.npz")
    ps = _system(tmp_path, g)
    x, a, s = g["field/positions"], g["field/strengths"], g["field/radii"]
    mags = np.linalg.norm(a, axis=1)
    from openonda_b200.vpm.vpmModule import get_highest_nonzero_indices

    idx = get_highest_nonzero_indices(mags, top_percentage=5)
    ps.subdivide_strong_particles(top_percentage=5)
    keep = np.setdiff1d(np.arange(len(x)), idx)
    n_new = 2 * len(idx)
    assert len(ps) == len(x) - len(idx) + n_new
    xs, as_ = ps.get_particle_positions(), ps.get_particle_strengths()
    # survivors keep their order and come first; the halves are appended after them
    assert np.array_equal(xs[:len(keep)], x[keep])
    dx = (s[idx] * a[idx].T / mags[idx]).T * 0.25
    expect_x = np.stack([x[idx] + dx, x[idx] - dx], axis=1).reshape(-1, 3)
    assert normwise(xs[len(keep):], expect_x) <= 1e-15
    assert normwise(as_[len(keep):], np.repeat(a[idx] / 2, 2, axis=0)) <= 1e-15
    # the total strength vector is conserved
    assert normwise(ps.get_total_strength(), a.sum(axis=0)) <= 1e-13


def test_probe_fields_through_the_system(tmp_path):
    g = golden("manage.npz")
    ps = _system(tmp_path, g)
    x, a, s = g["field/positions"], g["field/strengths"], g["field/radii"]
    grid = np.stack(np.meshgrid(*(np.linspace(-0.8, 0.8, 7),) * 3, indexing="ij"),
                    axis=-1).reshape(-1, 3)
    assert normwise(ps.get_induced_velocity_at(grid),
                    oracle.gpu.get_induced_velocity_at(grid, x, a, s)) <= 1e-12
    assert normwise(ps.get_vorticity_field_at(grid),
                    oracle.gpu.get_vorticity_field_at(grid, x, a, s)) <= 1e-12
    assert normwise(ps.get_particle_vorticities(),
                    oracle.gpu.get_vorticity_field_at(x, x, a, s)) <= 1e-12


@pytest.mark.parametrize("use_graph", [False, True])
def test_checkpoint_resume_is_exact(tmp_path, use_graph):
    """save_checkpoint after 5 steps, 4 more steps; a new system loaded from the checkpoint
    and stepped 4 times must hold the same state bit for bit (BDF history, LES state and
    clock are part of the checkpoint)."""
    from openonda_b200 import configs

    f = configs.random_cloud(600, seed=5, nu=1e-3)
    f.strengths[:, 2] += 2e-3
    f.radii *= 4
    cfg = dict(flow_model="LES", viscous_scheme="PSE", time_integration_method="RK4",
               time_step_size=0.005)
    os.makedirs(tmp_path / "a", exist_ok=True)
    os.makedirs(tmp_path / "b", exist_ok=True)
    a = _system(tmp_path / "a", **cfg)
    a.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                         f.viscosities)
    a.advance(5, use_graph=use_graph)
    ck = str(tmp_path / "ck.npz")
    a.save_checkpoint(ck)
    a.advance(4, use_graph=use_graph)
    # built with another step size: the checkpoint's step size must take over
    b = _system(tmp_path / "b", **dict(cfg, time_step_size=0.02))
    b.load_checkpoint(ck)
    assert b.time_step == 5 and b.time_step_size == 0.005
    b.advance(4, use_graph=use_graph)
    for get in ("get_particle_positions", "get_particle_strengths", "get_particle_radii",
                "get_particle_velocities", "get_particle_viscosities_t"):
        assert np.array_equal(getattr(a, get)(), getattr(b, get)()), get
    assert a.Cnu == b.Cnu and a.time_step == b.time_step and a.flow_time == b.flow_time
