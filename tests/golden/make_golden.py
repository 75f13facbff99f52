"""Generate the golden vectors that pin the oracle to the reference.

Run in a container that holds the reference checkout (default path below, or
``--reference DIR``):

    python tests/golden/make_golden.py

It executes the reference's own code and writes ``tests/golden/*.npz``:

* ``gpu_kernels.npz``  -- ``OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py`` run under the
  Numba CUDA simulator (``NUMBA_ENABLE_CUDASIM=1``, in a child process) on small seeded
  inputs.  The three scalar kernels are launched directly with a zeroed accumulator (the
  reference wrapper never clears it, ParticlesPhysicsCuda.py:545,655,764) and then divided
  the way the wrappers divide (:556, :668, :777).
* ``cpu_kernels.npz``  -- ``ParticlesPhysics.py`` (the Numba-CPU module) on seeded inputs.
* ``ring8192.npz``     -- the 8192-particle ring lattice: CPU-module outputs for the
  functions whose CPU and GPU semantics coincide (probe velocity, stretching) plus the
  CPU-semantics self velocity and PSE.
* ``steps_cpu.npz``    -- ``vpmModule.ParticleSystem`` (processing_unit='CPU') trajectories.
* ``steps_gpu.npz``    -- ``vpmModule.ParticleSystem`` with the Numba-CUDA module under the
  simulator (GPU semantics), small N.
* ``ic.npz``           -- ``OpenONDA/utilities/vpm_flow_models.py`` (vortex_ring_vpm,
  lamb_oseen_vpm, isotropic_turbulence_vpm) and ``vpm_solver_helper.py`` (rectangular, 2-D rectangular, hexagonal and
  cylindrical lattices) on the seeded cases of ``ic_cases()``.
* ``manage.npz``       -- the reference ParticleSystem's O(N) diagnostics, remove_weak_particles
  (relative with circulation conservation, absolute) and get_highest_nonzero_indices.
* ``step_ring8192.npz`` -- one DNS+PSE+RK4 step of the 8192-particle ring through the
  reference ``ParticleSystem`` sequencing with the GPU-semantics oracle kernels injected as
  its physics module (the simulator is too slow at this size).

Nothing else in the repository reads the reference; the tests read only these files.
"""
from __future__ import annotations

import argparse
import contextlib
import importlib
import importlib.util
import io
import os
import subprocess
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from openonda_b200 import configs  # noqa: E402

DEFAULT_REF = "/root/reference"


def vpm_dir(ref):
    return os.path.join(ref, "OpenONDA", "solvers", "VPM")


def load_by_path(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------------------------------
# Inputs
# ------------------------------------------------------------------------------------
def kernel_cases():
    """Small seeded inputs shared by the GPU- and CPU-semantics kernel fixtures."""
    cases = {}
    f = configs.random_cloud(64, seed=11)
    cases["cloud64"] = f
    f = configs.random_cloud(200, seed=12)
    f.viscosities = np.random.default_rng(5).uniform(1e-4, 3e-4, size=200)
    cases["cloud200"] = f
    cases["ring128"] = configs.vortex_ring(8, 16, 1.0, 1.0, 0.1, nu=2e-4)
    f = configs.random_cloud(24, seed=13)
    f.positions[17] = f.positions[5]  # two distinct particles at one point
    cases["coincident24"] = f
    cases["single1"] = configs.random_cloud(1, seed=14)
    cases["cloud33"] = configs.random_cloud(33, seed=15)
    return cases


def probe_targets(field, seed):
    rng = np.random.default_rng(seed)
    t = rng.uniform(-1.1, 1.1, size=(37, 3))
    t[0] = field.positions[0]  # exactly on a source: r^2 = 0 is skipped
    t[1] = field.positions[-1] + 1e-5  # r^2 = 3e-10 < 1e-8 is skipped
    return t


# ------------------------------------------------------------------------------------
# GPU semantics under the simulator (child process)
# ------------------------------------------------------------------------------------
def _gpu_child(ref, out_path):
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    from numba import cuda

    g = load_by_path("ref_particles_physics_cuda", os.path.join(vpm_dir(ref),
                                                                 "ParticlesPhysicsCuda.py"))

    def scalar(kernel, x, a, s, post):
        acc = cuda.to_device(np.zeros(1))
        bpg = (len(x) + g.threads_per_block - 1) // g.threads_per_block
        kernel[bpg, g.threads_per_block](cuda.to_device(x), cuda.to_device(a),
                                         cuda.to_device(s), acc)
        return acc.copy_to_host()[0] / post

    out = {}
    for name, f in kernel_cases().items():
        x, a, s, v = f.positions, f.strengths, f.radii, f.viscosities
        t = probe_targets(f, 99)
        out[f"{name}/positions"] = x
        out[f"{name}/strengths"] = a
        out[f"{name}/radii"] = s
        out[f"{name}/viscosities"] = v
        out[f"{name}/targets"] = t
        out[f"{name}/induced_velocity_at"] = g.get_induced_velocity_at(t, x, a, s)
        out[f"{name}/selfinduced_velocity"] = g.get_selfinduced_velocity(x, a, s)
        out[f"{name}/vorticity_field_at"] = g.get_vorticity_field_at(x, x, a, s)
        out[f"{name}/strength_gradients"] = g.get_strength_gradients(x, a, s)
        out[f"{name}/strength_gradients_PSE"] = g.get_strength_gradients_PSE(x, a, s, v)
        with np.errstate(all="ignore"):
            out[f"{name}/total_kinetic_energy"] = scalar(g.get_total_kinetic_energy_kernel,
                                                         x, a, s, 1.0)
        out[f"{name}/total_helicity"] = scalar(g.get_total_helicity_kernel, x, a, s, 4 * np.pi)
        out[f"{name}/total_enstrophy"] = scalar(g.get_total_enstrophy_kernel_simple, x, a, s,
                                                4 * np.pi)
    np.savez_compressed(out_path, **out)


def make_gpu_kernels(ref):
    out = os.path.join(HERE, "gpu_kernels.npz")
    env = dict(os.environ, NUMBA_ENABLE_CUDASIM="1")
    subprocess.run([sys.executable, __file__, "--reference", ref, "--child", "gpu_kernels",
                    "--out", out], check=True, env=env)


# ------------------------------------------------------------------------------------
# CPU semantics
# ------------------------------------------------------------------------------------
def make_cpu_kernels(ref):
    c = load_by_path("ref_particles_physics", os.path.join(vpm_dir(ref), "ParticlesPhysics.py"))
    out = {}
    cases = kernel_cases()
    cases["ring2048"] = configs.vortex_ring(32, 64, 1.0, 1.0, 0.1, nu=1e-4)
    for name, f in cases.items():
        x, a, s, v = f.positions, f.strengths, f.radii, f.viscosities
        t = probe_targets(f, 98)
        out[f"{name}/positions"] = x
        out[f"{name}/strengths"] = a
        out[f"{name}/radii"] = s
        out[f"{name}/viscosities"] = v
        out[f"{name}/targets"] = t
        out[f"{name}/induced_velocity_at"] = c.get_induced_velocity_at(t, x, a, s)
        out[f"{name}/selfinduced_velocity"] = c.get_selfinduced_velocity(x, a, s)
        out[f"{name}/vorticity_field_at"] = c.get_vorticity_field_at(t, x, a, s)
        out[f"{name}/strength_gradients"] = c.get_strength_gradients(x, a, s)
        out[f"{name}/strength_gradients_PSE"] = c.get_strength_gradients_PSE(x, a, s, v)
        with np.errstate(all="ignore"):
            out[f"{name}/total_kinetic_energy"] = c.get_total_kinetic_energy(x, a, s)
        out[f"{name}/total_helicity"] = c.get_total_helicity(x, a, s)
        out[f"{name}/total_enstrophy"] = c.get_total_enstrophy(x, a, s)
    np.savez_compressed(os.path.join(HERE, "cpu_kernels.npz"), **out)


def make_ring8192(ref):
    c = load_by_path("ref_particles_physics", os.path.join(vpm_dir(ref), "ParticlesPhysics.py"))
    f = configs.ring_8192()
    x, a, s, v = f.positions, f.strengths, f.radii, f.viscosities
    t = x[::16].copy()
    out = dict(positions=x, strengths=a, radii=s, viscosities=v, targets=t)
    out["induced_velocity_at"] = c.get_induced_velocity_at(t, x, a, s)
    out["strength_gradients"] = c.get_strength_gradients(x, a, s)
    out["cpu_selfinduced_velocity"] = c.get_selfinduced_velocity(x, a, s)
    out["cpu_strength_gradients_PSE"] = c.get_strength_gradients_PSE(x, a, s, v)
    np.savez_compressed(os.path.join(HERE, "ring8192.npz"), **out)


# ------------------------------------------------------------------------------------
# Step-level trajectories through the reference ParticleSystem
# ------------------------------------------------------------------------------------
class _FakePolyData:
    def __init__(self, points):
        self.points = points
        self.point_data = {}

    def save(self, filename):
        pass


def import_vpm_module(ref):
    """Import the reference vpmModule without its FVM package and without pyvista."""
    for name, path in [("OpenONDA", os.path.join(ref, "OpenONDA")),
                       ("OpenONDA.solvers", os.path.join(ref, "OpenONDA", "solvers")),
                       ("OpenONDA.solvers.VPM", vpm_dir(ref))]:
        if name not in sys.modules:
            m = types.ModuleType(name)
            m.__path__ = [path]
            sys.modules[name] = m
    sys.modules.setdefault("pyvista", types.SimpleNamespace(PolyData=_FakePolyData))
    return importlib.import_module("OpenONDA.solvers.VPM.vpmModule")


def run_reference_steps(vpm, field, n_steps, physics=None, **kwargs):
    """Run the reference time loop and return the state after every step."""
    with contextlib.redirect_stdout(io.StringIO()):
        ps = vpm.ParticleSystem(monitor_variables=[], backup_frequency=10 ** 9, **kwargs)
        if physics is not None:
            ps.physics = physics
        n = field.n
        ps.add_particle_field(field.positions.copy(), np.zeros((n, 3)), field.strengths.copy(),
                              field.radii.copy(), field.viscosities.copy())
        rec = {k: [] for k in ("positions", "strengths", "radii", "velocities",
                               "viscosities_t", "Cnu")}
        for _ in range(n_steps):
            ps.update_velocities()
            ps.update_strengths()
            ps.update_state()
            rec["positions"].append(ps.get_particle_positions())
            rec["strengths"].append(ps.get_particle_strengths())
            rec["radii"].append(ps.get_particle_radii())
            rec["velocities"].append(ps.get_particle_velocities())
            rec["viscosities_t"].append(ps.get_particle_viscosities_t())
            rec["Cnu"].append(ps.Cnu)
    return {k: np.asarray(v) for k, v in rec.items()}


# relax_strength_solution=True is not exercised: the reference raises ValueError there
# (vpmModule.py:879 divides an (N,3) array by an (N,) array).
STEP_CASES_CPU = {
    "dns_pse_rk4": dict(flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
                        time_step_size=0.01, steps=5),
    "les_cs_rk2": dict(flow_model="LES", viscous_scheme="CoreSpreading",
                       time_integration_method="RK2", time_step_size=0.01, steps=4),
    "pseudo2d_cs_rk3": dict(flow_model="pseudo2D", viscous_scheme="CoreSpreading",
                            time_integration_method="RK3", time_step_size=0.01, steps=3),
    "potential_euler": dict(flow_model="Potential", viscous_scheme=None,
                            time_integration_method="Euler", time_step_size=0.01, steps=2),
    "les_pse_rk4": dict(flow_model="LES", viscous_scheme="PSE", time_integration_method="RK4",
                        time_step_size=0.005, steps=5),
}


def step_field_small():
    return configs.vortex_ring(16, 32, 1.0, 1.0, 0.1, nu=1e-3)


def step_field_les(n, seed):
    """LES cases need a field whose mean vorticity is well above rounding: on a closed ring
    the mean is ~0, and the reference's angle test (vpmModule.py:939-948) would then be
    decided by rounding noise."""
    f = configs.random_cloud(n, seed=seed, nu=1e-3)
    f.strengths[:, 2] += 2e-3  # a mean vorticity along z
    f.radii *= 4.0  # overlapping cores
    return f


def make_steps_cpu(ref):
    vpm = import_vpm_module(ref)
    out = {}
    for name, cfg in STEP_CASES_CPU.items():
        cfg = dict(cfg)
        steps = cfg.pop("steps")
        f = step_field_les(512, 31) if cfg["flow_model"] == "LES" else step_field_small()
        for k in ("positions", "strengths", "radii", "viscosities"):
            out[f"{name}/init_{k}"] = getattr(f, k)
        rec = run_reference_steps(vpm, f, steps, processing_unit="CPU", **cfg)
        for k, v in rec.items():
            out[f"{name}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "steps_cpu.npz"), **out)


STEP_CASES_GPU = {
    "dns_pse_rk4": dict(flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
                        time_step_size=0.01, steps=5),
    "les_cs_rk4": dict(flow_model="LES", viscous_scheme="CoreSpreading",
                       time_integration_method="RK4", time_step_size=0.01, steps=3),
    "les_pse_rk2": dict(flow_model="LES", viscous_scheme="PSE", time_integration_method="RK2",
                        time_step_size=0.01, steps=4),
}


def step_field_tiny():
    return configs.vortex_ring(8, 8, 1.0, 1.0, 0.1, nu=1e-3)


def _steps_gpu_child(ref, out_path):
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    from numba import cuda

    vpm = import_vpm_module(ref)
    g = importlib.import_module("OpenONDA.solvers.VPM.ParticlesPhysicsCuda")

    def enstrophy_zeroed(x, a, s):
        acc = cuda.to_device(np.zeros(1))
        bpg = (len(x) + g.threads_per_block - 1) // g.threads_per_block
        g.get_total_enstrophy_kernel_simple[bpg, g.threads_per_block](
            cuda.to_device(x), cuda.to_device(a), cuda.to_device(s), acc)
        return acc.copy_to_host()[0] / (4 * np.pi)

    physics = types.SimpleNamespace(**{k: getattr(g, k) for k in dir(g) if k.startswith("get_")})
    physics.get_total_enstrophy = enstrophy_zeroed
    out = {}
    for name, cfg in STEP_CASES_GPU.items():
        cfg = dict(cfg)
        steps = cfg.pop("steps")
        f = step_field_les(64, 32) if cfg["flow_model"] == "LES" else step_field_tiny()
        for k in ("positions", "strengths", "radii", "viscosities"):
            out[f"{name}/init_{k}"] = getattr(f, k)
        # processing_unit only selects the module (vpmModule.py:141-154); the simulator lacks
        # cuda.CudaSupportError (vpmModule.py:107), so select CPU and inject the CUDA module.
        rec = run_reference_steps(vpm, f, steps, physics=physics, processing_unit="CPU", **cfg)
        for k, v in rec.items():
            out[f"{name}/{k}"] = v
    np.savez_compressed(out_path, **out)


def make_steps_gpu(ref):
    out = os.path.join(HERE, "steps_gpu.npz")
    env = dict(os.environ, NUMBA_ENABLE_CUDASIM="1")
    subprocess.run([sys.executable, __file__, "--reference", ref, "--child", "steps_gpu",
                    "--out", out], check=True, env=env)


def make_step_ring8192(ref):
    import oracle

    vpm = import_vpm_module(ref)
    physics = types.SimpleNamespace(
        get_selfinduced_velocity=oracle.gpu.get_selfinduced_velocity,
        get_induced_velocity_at=oracle.gpu.get_induced_velocity_at,
        get_vorticity_field_at=oracle.gpu.get_vorticity_field_at,
        get_strength_gradients=oracle.gpu.get_strength_gradients,
        get_strength_gradients_PSE=oracle.gpu.get_strength_gradients_PSE,
        get_total_kinetic_energy=oracle.gpu.get_total_kinetic_energy,
        get_total_helicity=oracle.gpu.get_total_helicity,
        get_total_enstrophy=oracle.gpu.get_total_enstrophy,
    )
    f = configs.ring_8192()
    rec = run_reference_steps(vpm, f, 1, physics=physics, processing_unit="CPU",
                              flow_model="DNS", viscous_scheme="PSE",
                              time_integration_method="RK4", time_step_size=0.01)
    out = {f"step/init_{k}": getattr(f, k)
           for k in ("positions", "strengths", "radii", "viscosities")}
    for k, v in rec.items():
        out[f"step/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "step_ring8192.npz"), **out)


def ic_cases():
    """Seeded inputs for the initial-condition and lattice generators (shared with tests)."""
    rng = np.random.default_rng(77)
    ring_pts = rng.uniform(-1.3, 1.3, size=(3000, 3))
    ring_pts[:, 0] *= 0.3
    return {
        "ring": dict(positions=ring_pts, volumes=rng.uniform(1e-4, 2e-4, 3000),
                     args=(0.05, 1e-4, np.array([0.1, -0.05, 0.02]), 1.0, 1.0, 0.1, 0.02,
                           0.3, 5.0)),
        "ring_plain": dict(positions=ring_pts[:1000], volumes=np.full(1000, 1.5e-4),
                           args=(0.04, 2e-5, np.zeros(3), 0.8, 2.0, 0.15)),
        "lamb": dict(positions=rng.uniform(-0.5, 0.5, size=(2000, 3)),
                     volumes=rng.uniform(1e-4, 2e-4, 2000),
                     args=(0.05, 1e-4, np.array([0.02, -0.01, 0.0]), 1.5, 0.12, 0.01, 0.7,
                           12.0)),
        "rect3": dict(box=np.array([-1.0, 1.0, -0.5, 0.5, -0.3, 0.3]), spacing=0.1),
        "rect3b": dict(box=np.array([-0.7, 0.9, -0.25, 0.55, 0.0, 0.4]), spacing=0.037),
        "rect2": dict(box=np.array([-1.0, 1.0, -0.6, 0.4, 0.0, 0.0]), spacing=0.03),
        "hex": dict(box=np.array([-0.5, 0.5, -0.4, 0.4, -0.2, 0.2]), spacing=0.05),
        "cyl_x": dict(d=0.05, radius=1.0, height=2.0, center=np.zeros(3), axis="x"),
        "cyl_y": dict(d=0.07, radius=0.6, height=1.3, center=np.array([0.1, 0.2, -0.3]),
                      axis="y"),
        "cyl_z": dict(d=0.09, radius=0.5, height=0.8, center=np.array([-1.0, 0.0, 2.0]),
                      axis="z"),
        "turb8": dict(box=1.0, d=0.125, radius=0.2),
        "turb16": dict(box=2.0, d=0.125, radius=0.15),
    }


def make_ic(ref):
    util = os.path.join(ref, "OpenONDA", "utilities")
    fm = load_by_path("ref_vpm_flow_models", os.path.join(util, "vpm_flow_models.py"))
    sh = load_by_path("ref_vpm_solver_helper", os.path.join(util, "vpm_solver_helper.py"))
    out = {}
    for name, c in ic_cases().items():
        if name.startswith("ring") or name == "lamb":
            fn = fm.vortex_ring_vpm if name.startswith("ring") else fm.lamb_oseen_vpm
            vel, a, s, nu = fn(c["positions"], c["volumes"], *c["args"])
            out[f"{name}/positions"] = c["positions"]
            out[f"{name}/volumes"] = c["volumes"]
            for k, v in (("velocities", vel), ("strengths", a), ("radii", s),
                         ("viscosities", nu)):
                out[f"{name}/{k}"] = v
        elif name.startswith("rect"):
            fn = (sh.get_rectangular_point_distribuition if name != "rect2"
                  else sh.get_2D_rectangular_point_distribuition)
            out[f"{name}/points"], out[f"{name}/volumes"] = fn(c["box"], c["spacing"])
        elif name.startswith("turb"):
            state = np.random.get_state()  # the reference re-seeds numpy's global generator
            res = fm.isotropic_turbulence_vpm(c["box"], c["d"], c["radius"])
            np.random.set_state(state)
            for k, v in zip(("positions", "velocities", "strengths", "radii"), res):
                out[f"{name}/{k}"] = v
        elif name == "hex":
            out[f"{name}/points"], out[f"{name}/volumes"] = sh.get_hexagonal_point_distribution(
                c["box"], c["spacing"])
        else:
            out[f"{name}/points"], out[f"{name}/volumes"] = \
                sh.get_cylindrical_point_distribuition(c["d"], c["radius"], c["height"],
                                                        c["center"], c["axis"])
    np.savez_compressed(os.path.join(HERE, "ic.npz"), **out)


def manage_field():
    f = configs.random_cloud(400, seed=31, nu=1e-3)
    f.strengths *= np.random.default_rng(32).uniform(0.1, 3.0, size=(400, 1))
    return f


def make_manage(ref):
    """Particle-field control and O(N) diagnostics of the reference ParticleSystem
    (vpmModule.py:264-284, :970-1037, :1124-1166) on a seeded cloud."""
    vpm = import_vpm_module(ref)
    f = manage_field()
    mags = np.linalg.norm(f.strengths, axis=1)
    out = {"field/positions": f.positions, "field/strengths": f.strengths,
           "field/radii": f.radii, "field/viscosities": f.viscosities}

    def fresh():
        ps = vpm.ParticleSystem(monitor_variables=[], backup_frequency=10 ** 9,
                                processing_unit="CPU")
        ps.add_particle_field(f.positions.copy(), np.zeros_like(f.positions),
                              f.strengths.copy(), f.radii.copy(), f.viscosities.copy())
        return ps

    with contextlib.redirect_stdout(io.StringIO()):
        ps = fresh()
        out["diag/linear_impulse"] = ps.get_total_linear_impulse()
        out["diag/angular_impulse"] = ps.get_total_angular_impulse()
        out["diag/total_strength"] = ps.get_total_strength()
        out["diag/total_strength_magnitude"] = np.array(ps.get_total_strength_magnitude())
        cases = {"relative_conserve": ("relative", 0.4, True),
                 "absolute": ("absolute", float(np.median(mags)), False)}
        for name, (mode, thr, conserve) in cases.items():
            ps = fresh()
            ps.remove_weak_particles(mode, thr, conserve_total_circulation=conserve)
            out[f"{name}/positions"] = ps.get_particle_positions()
            out[f"{name}/strengths"] = ps.get_particle_strengths()
            out[f"{name}/radii"] = ps.get_particle_radii()
            out[f"{name}/threshold"] = np.array(thr)
    out["highest/top10"] = vpm.get_highest_nonzero_indices(mags, top_percentage=10)
    out["highest/above"] = vpm.get_highest_nonzero_indices(
        mags, strength_threshold=float(np.percentile(mags, 80)))
    out["highest/mags"] = mags
    np.savez_compressed(os.path.join(HERE, "manage.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REF)
    ap.add_argument("--child", default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--only", default=None, help="comma-separated subset to regenerate")
    args = ap.parse_args()
    if args.child == "gpu_kernels":
        _gpu_child(args.reference, args.out)
        return
    if args.child == "steps_gpu":
        _steps_gpu_child(args.reference, args.out)
        return
    jobs = {
        "gpu_kernels": make_gpu_kernels,
        "cpu_kernels": make_cpu_kernels,
        "ring8192": make_ring8192,
        "steps_cpu": make_steps_cpu,
        "steps_gpu": make_steps_gpu,
        "step_ring8192": make_step_ring8192,
        "ic": make_ic,
        "manage": make_manage,
    }
    only = set(args.only.split(",")) if args.only else set(jobs)
    for name, fn in jobs.items():
        if name in only:
            print(f"[make_golden] {name}", flush=True)
            fn(args.reference)


if __name__ == "__main__":
    main()
