"""Device-resident ParticleSystem: step-level parity against the reference's own trajectories
(vpmModule.ParticleSystem with the Numba-CUDA module under the simulator, golden
steps_gpu.npz; the 8192-particle ring step, golden step_ring8192.npz) and against the pinned
step oracle (oracle/vpm_step.py with oracle.gpu kernels) for the other flow models."""
import os

import numpy as np
import pytest

import oracle
from conftest import golden, normwise
from oracle.vpm_step import StepOracle

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _system(tmp_path, **cfg):
    from openonda_b200.vpm.vpmModule import ParticleSystem

    return ParticleSystem(monitor_variables=[], backup_frequency=10 ** 9,
                          backup_filename=str(tmp_path / "b"), **cfg)


def _run(ps, n):
    out = []
    for _ in range(n):
        ps.update_velocities()
        ps.update_strengths()
        ps.update_state()
        out.append(dict(x=ps.get_particle_positions(), a=ps.get_particle_strengths(),
                        s=ps.get_particle_radii(), u=ps.get_particle_velocities(),
                        nut=ps.get_particle_viscosities_t(), cnu=ps.Cnu))
    return out


def _load(ps, g, name):
    n = g[f"{name}/init_positions"].shape[0]
    ps.add_particle_field(g[f"{name}/init_positions"], np.zeros((n, 3)),
                          g[f"{name}/init_strengths"], g[f"{name}/init_radii"],
                          g[f"{name}/init_viscosities"])


STEP_GPU = {
    "dns_pse_rk4": dict(flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
                        time_step_size=0.01, n=5),
    "les_cs_rk4": dict(flow_model="LES", viscous_scheme="CoreSpreading",
                       time_integration_method="RK4", time_step_size=0.01, n=3),
    "les_pse_rk2": dict(flow_model="LES", viscous_scheme="PSE", time_integration_method="RK2",
                        time_step_size=0.01, n=4),
}


@pytest.mark.parametrize("name", sorted(STEP_GPU))
def test_trajectory_vs_reference_numba_cuda(tmp_path, name):
    g = golden("steps_gpu.npz")
    cfg = dict(STEP_GPU[name])
    n = cfg.pop("n")
    ps = _system(tmp_path, **cfg)
    _load(ps, g, name)
    for k, st in enumerate(_run(ps, n)):
        for key, ref in (("x", "positions"), ("a", "strengths"), ("s", "radii"),
                         ("u", "velocities")):
            assert normwise(st[key], g[f"{name}/{ref}"][k]) <= TOL, (name, k, key)
        assert normwise(st["nut"], g[f"{name}/viscosities_t"][k]) <= 1e-10, (name, k)
        assert abs(st["cnu"] - g[f"{name}/Cnu"][k]) <= 1e-12 * abs(st["cnu"])


def test_ring8192_one_rk4_step_vs_reference_sequencing(tmp_path):
    g = golden("step_ring8192.npz")
    ps = _system(tmp_path, flow_model="DNS", viscous_scheme="PSE",
                 time_integration_method="RK4", time_step_size=0.01)
    _load(ps, g, "step")
    st = _run(ps, 1)[0]
    for key, ref in (("x", "positions"), ("a", "strengths"), ("s", "radii"), ("u", "velocities")):
        assert normwise(st[key], g[f"step/{ref}"][0]) <= TOL, key


ORACLE_CASES = {
    "dns_cs_rk3": dict(flow_model="DNS", viscous_scheme="CoreSpreading",
                       time_integration_method="RK3", time_step_size=0.01, n=4, field="ring"),
    "pseudo2d_pse_euler": dict(flow_model="pseudo2D", viscous_scheme="PSE",
                               time_integration_method="Euler", time_step_size=0.01, n=3,
                               field="ring"),
    "potential_rk2": dict(flow_model="Potential", viscous_scheme=None,
                          time_integration_method="RK2", time_step_size=0.02, n=2,
                          field="ring"),
    "les_pse_rk4_relax": dict(flow_model="LES", viscous_scheme="PSE",
                              time_integration_method="RK4", time_step_size=0.005, n=5,
                              field="cloud", relax_strength_solution=True),
}


def _field(kind):
    from openonda_b200 import configs

    if kind == "ring":
        return configs.vortex_ring(16, 40, 1.0, 1.0, 0.1, nu=1e-3)  # N = 640
    if kind == "ring1600":  # three tiles or more for every both-sides sweep
        return configs.vortex_ring(16, 100, 1.0, 1.0, 0.1, nu=1e-3)
    f = configs.random_cloud(1700 if kind == "cloud1700" else 700, seed=41, nu=1e-3)
    f.strengths[:, 2] += 2e-3
    f.radii *= 4.0
    return f


@pytest.mark.parametrize("name", sorted(ORACLE_CASES))
def test_trajectory_vs_step_oracle(tmp_path, name):
    cfg = dict(ORACLE_CASES[name])
    n, kind = cfg.pop("n"), cfg.pop("field")
    f = _field(kind)
    so = StepOracle(oracle.gpu, f.positions, f.strengths, f.radii, f.viscosities, **cfg)
    ps = _system(tmp_path, **cfg)
    ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                          f.viscosities)
    got = _run(ps, n)
    for k in range(n):
        so.step()
        assert normwise(got[k]["x"], so.x) <= 1e-11, (name, k, "x")
        assert normwise(got[k]["a"], so.a) <= 1e-11, (name, k, "a")
        assert normwise(got[k]["s"], so.s) <= 1e-11, (name, k, "s")
        assert normwise(got[k]["u"], so.u) <= 1e-11, (name, k, "u")
        assert abs(got[k]["cnu"] - so.Cnu) <= 1e-11 * abs(so.Cnu)


def test_fp32c_trajectory_tracks_fp64(tmp_path):
    from openonda_b200 import configs

    f = configs.ring_8192()
    runs = {}
    for prec in ("fp64", "fp32c"):
        ps = _system(tmp_path, flow_model="DNS", viscous_scheme="PSE",
                     time_integration_method="RK4", time_step_size=0.01, precision=prec)
        ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                              f.viscosities)
        runs[prec] = _run(ps, 3)
    for k in range(3):
        assert normwise(runs["fp32c"][k]["u"], runs["fp64"][k]["u"]) <= 2e-5
        assert normwise(runs["fp32c"][k]["x"], runs["fp64"][k]["x"]) <= 1e-7


def test_checkpoint_resume_is_exact(tmp_path):
    from openonda_b200 import configs

    f = configs.vortex_ring(8, 32, 1.0, 1.0, 0.1, nu=1e-3)
    kw = dict(flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
              time_step_size=0.01)
    a = _system(tmp_path, **kw)
    a.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                         f.viscosities)
    _run(a, 2)
    ck = str(tmp_path / "ck.npz")
    a.save_checkpoint(ck)
    ra = _run(a, 3)
    b = _system(tmp_path, **kw)
    b.load_checkpoint(ck)
    rb = _run(b, 3)
    for k in range(3):
        for key in ("x", "a", "s"):
            assert np.array_equal(ra[k][key], rb[k][key]), (k, key)


def test_backup_files_written(tmp_path):
    from openonda_b200 import configs
    from openonda_b200.vpm.vpmModule import ParticleSystem

    f = configs.vortex_ring(4, 8, 1.0, 1.0, 0.1)
    ps = ParticleSystem(monitor_variables=["Circulation", "Kinetic energy", "Linear impulse",
                                           "Angular impulse", "Enstrophy", "Helicity"],
                        backup_frequency=2, backup_filename=str(tmp_path / "ring"),
                        flow_model="DNS", viscous_scheme="PSE", time_step_size=0.01)
    ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                          f.viscosities)
    _run(ps, 3)
    assert os.path.exists(tmp_path / "ring_0000000.npz")
    assert os.path.exists(tmp_path / "ring_0000002.npz")


def test_diagnostics_match_numpy(tmp_path):
    from openonda_b200 import configs

    f = configs.random_cloud(3000, seed=4)
    ps = _system(tmp_path)
    ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                          f.viscosities)
    x, a = f.positions, f.strengths
    np.testing.assert_allclose(ps.get_total_linear_impulse(),
                               0.5 * np.sum(np.cross(x, a), axis=0), rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(ps.get_total_angular_impulse(),
                               (1 / 3) * np.sum(np.cross(x, np.cross(x, a)), axis=0),
                               rtol=1e-12, atol=1e-18)
    assert ps.get_total_strength_magnitude() == pytest.approx(
        np.sum(np.linalg.norm(a, axis=1)), rel=1e-13)
    np.testing.assert_allclose(ps.get_total_strength(), a.sum(axis=0), rtol=1e-12, atol=1e-18)
    assert ps.get_total_kinetic_energy() == pytest.approx(
        oracle.gpu.get_total_kinetic_energy(x, a, f.radii), rel=1e-12)
    assert ps.get_total_enstrophy() == pytest.approx(
        oracle.gpu.get_total_enstrophy(x, a, f.radii), rel=1e-12)


def test_particle_management(tmp_path):
    from openonda_b200 import configs

    f = configs.vortex_ring(8, 16, 1.0, 1.0, 0.1)
    ps = _system(tmp_path)
    ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                          f.viscosities, group_id=3)
    n0 = len(ps)
    mags = np.linalg.norm(f.strengths, axis=1)
    before = mags.sum()
    ps.remove_weak_particles("relative", 0.5, conserve_total_circulation=True)
    keep = ~(mags / mags.max() < 0.5)
    assert len(ps) == int(keep.sum()) < n0
    assert ps.get_total_strength_magnitude() == pytest.approx(before, rel=1e-12)
    assert np.all(ps.get_particle_group_id() == 3)
    m = len(ps)
    ps.subdivide_strong_particles(top_percentage=10)
    top = max(int(10 * m / 100), 1)
    assert len(ps) == m + top
    p = ps[0]
    assert p.position.shape == (3,) and p.radius > 0
    ps.remove_particles([0, 1, 1])
    assert len(ps) == m + top - 2
    ps.remove_all_particles()
    assert len(ps) == 0


GRAPH_CASES = {
    "dns_pse_rk4": dict(flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
                        time_step_size=0.005),
    "les_pse_rk4": dict(flow_model="LES", viscous_scheme="PSE", time_integration_method="RK4",
                        time_step_size=0.005),
    "les_cs_rk2_relax": dict(flow_model="LES", viscous_scheme="CoreSpreading",
                             time_integration_method="RK2", time_step_size=0.005,
                             relax_strength_solution=True),
    "potential_rk3": dict(flow_model="Potential", viscous_scheme=None,
                          time_integration_method="RK3", time_step_size=0.01),
    "dns_cs_euler_fp32c": dict(flow_model="DNS", viscous_scheme="CoreSpreading",
                               time_integration_method="Euler", time_step_size=0.005,
                               precision="fp32c"),
}


GRAPH_CASES["ring_dns_pse_rk4_uniform_core"] = dict(
    flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
    time_step_size=0.005, field="ring")
GRAPH_CASES["ring_dns_cs_rk2_uniform_core"] = dict(
    flow_model="DNS", viscous_scheme="CoreSpreading", time_integration_method="RK2",
    time_step_size=0.005, field="ring")
# FP32c self sums on the both-sides schedule (forced on below its size threshold)
GRAPH_CASES["les_pse_rk4_fp32c_both_sides"] = dict(
    flow_model="LES", viscous_scheme="PSE", time_integration_method="RK4",
    time_step_size=0.005, precision="fp32c", field="cloud1700", both_sides=True)
GRAPH_CASES["ring_dns_pse_rk4_fp32c_both_sides"] = dict(
    flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
    time_step_size=0.005, precision="fp32c", field="ring1600", both_sides=True)


@pytest.mark.parametrize("name", sorted(GRAPH_CASES))
def test_advance_with_cuda_graph_equals_eager_loop(tmp_path, name):
    """advance() replays one captured step from time step 3 on; it must reproduce the
    reference loop (update_velocities, update_strengths, update_state) bit for bit,
    including the steps where a backup is due and after a change that forces a recapture.
    The FP32c cases run with the both-sides schedule forced on (its zeroing, diagonal and
    diagonal-pair launches inside the captured graph); the others with it off."""
    from openonda_b200 import kernels

    cfg = dict(GRAPH_CASES[name])
    f = _field(cfg.pop("field", "cloud"))
    both_sides = cfg.pop("both_sides", False)
    prev = kernels.set_symmetric_min_n(0 if both_sides else 1 << 40)
    try:
        if both_sides:
            for op in ("selfinduced_velocity", "velocity_and_strength_gradients",
                       "strength_gradients_pse", "les_step_sums"):
                assert kernels.sweep_launches(op, "fp32c", f.n, f.n) > 2, op
        _advance_vs_eager(tmp_path, name, cfg, f)
    finally:
        kernels.set_symmetric_min_n(prev)


def _advance_vs_eager(tmp_path, name, cfg, f):
    import torch

    from openonda_b200.vpm.vpmModule import ParticleSystem

    def make(sub):
        ps = ParticleSystem(monitor_variables=[], backup_frequency=4,
                            backup_filename=str(tmp_path / sub / "b"), **cfg)
        ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                              f.viscosities)
        return ps

    os.makedirs(tmp_path / "e", exist_ok=True)
    os.makedirs(tmp_path / "g", exist_ok=True)
    eager, graph = make("e"), make("g")
    # ring fields have one core (uniform-core sweeps, kept through core spreading)
    assert graph._uc == bool(np.all(f.radii == f.radii[0]))
    _run(eager, 9)
    graph.advance(9)
    assert graph._uc == eager._uc
    assert graph._graph is not None  # steps 3..8 replayed
    eager.update_dt(0.004)  # settings change: the next graph step captures again
    graph.update_dt(0.004)
    _run(eager, 3)
    graph.advance(3)
    for get in ("get_particle_positions", "get_particle_strengths", "get_particle_radii",
                "get_particle_velocities", "get_particle_viscosities_t"):
        a, b = getattr(eager, get)(), getattr(graph, get)()
        assert np.array_equal(a, b), (name, get, float(np.max(np.abs(a - b))))
    assert eager.time_step == graph.time_step == 12
    assert eager.flow_time == graph.flow_time
    assert eager.Cnu == graph.Cnu
    from openonda_b200 import kernels

    assert kernels.device_errors() == 0  # no false uniform-core claim
    torch.cuda.synchronize()
