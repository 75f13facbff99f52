"""Least-squares dynamic LES coefficient (ParticleSystem(les_coefficient="least_squares"),
vpm_les_lsq_weights / vpm_les_lsq_update): the device sums against the FP64 numpy restatement
(oracle/vpm_les_lsq.py, parity unpinned: the reference has no such procedure), FP32-compensated
against FP64, and the CUDA-graph step against the eager loop."""
import os

import numpy as np
import pytest
import torch

import oracle
from oracle import vpm_les_lsq

pytestmark = pytest.mark.gpu


def _system(tmp_path, precision="fp64", **cfg):
    from openonda_b200.vpm.vpmModule import ParticleSystem

    base = dict(flow_model="LES", viscous_scheme="PSE", time_integration_method="RK4",
                time_step_size=0.005, les_coefficient="least_squares")
    base.update(cfg)
    return ParticleSystem(monitor_variables=[], backup_frequency=10 ** 9,
                          backup_filename=str(tmp_path / "b"), precision=precision, **base)


def _fields():
    from openonda_b200 import configs

    ring = configs.les_ring(32, 64)
    cloud = configs.random_cloud(1500, seed=9, nu=1e-4)
    cloud.radii *= 4
    cloud.strengths[:, 2] += 2e-3  # a mean vorticity, as in a jet or a wake
    return {"ring": ring, "cloud": cloud}


@pytest.mark.parametrize("name", ["ring", "cloud"])
def test_lsq_sums_vs_oracle(tmp_path, name):
    f = _fields()[name]
    ps = _system(tmp_path)
    ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                          f.viscosities)
    sums = ps._les_least_squares(ps._vorticity()).cpu().numpy()
    lm, mm = vpm_les_lsq.lsq_sums(oracle.gpu, f.positions, f.strengths, f.radii)
    print(f"{name}: device {sums[0]:.12e} {sums[1]:.12e} oracle {lm:.12e} {mm:.12e}")
    assert abs(sums[0] - lm) <= 1e-10 * abs(lm)
    assert abs(sums[1] - mm) <= 1e-10 * abs(mm)
    want = vpm_les_lsq.lsq_coefficient(oracle.gpu, f.positions, f.strengths, f.radii, 0.02958)
    assert abs(ps.Cnu - want) <= 1e-12 * want


def test_lsq_fp32c_vs_fp64(tmp_path):
    f = _fields()["ring"]
    r32 = lambda z: np.asarray(z, np.float32).astype(np.float64)
    out = {}
    for prec in ("fp64", "fp32c"):
        ps = _system(tmp_path, prec)
        ps.add_particle_field(r32(f.positions), np.zeros_like(f.positions), r32(f.strengths),
                              r32(f.radii), r32(f.viscosities))
        out[prec] = ps._les_least_squares(ps._vorticity()).cpu().numpy()
    rel = np.abs(out["fp32c"] - out["fp64"]) / np.abs(out["fp64"])
    print(f"fp32c vs fp64 sums: {rel}")
    assert np.all(rel <= 1e-5)


def test_lsq_step_graph_equals_eager_and_stays_in_range(tmp_path):
    f = _fields()["cloud"]
    runs = {}
    for mode in ("eager", "graph"):
        os.makedirs(tmp_path / mode, exist_ok=True)
        ps = _system(tmp_path / mode)
        ps.add_particle_field(f.positions, np.zeros_like(f.positions), f.strengths, f.radii,
                              f.viscosities)
        ps.advance(6, use_graph=(mode == "graph"))
        runs[mode] = (ps.get_particle_positions(), ps.get_particle_strengths(),
                      ps.get_particle_viscosities_t(), ps.Cnu)
    for a, b in zip(runs["eager"][:3], runs["graph"][:3]):
        assert np.array_equal(a, b)
    assert runs["eager"][3] == runs["graph"][3]
    assert 1e-9 <= runs["eager"][3] <= 0.0761
    from openonda_b200 import kernels

    assert kernels.device_errors() == 0


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32c", 1e-6)])
def test_test_filter_sweep_equals_two_vorticity_sums(precision, tol):
    """vpm_les_test_filter (one sweep, 80-byte records) against two vpm_vorticity_field_at
    sweeps with the same cores and strengths."""
    from openonda_b200 import configs, kernels

    f = configs.random_cloud(3000, seed=13)
    f.radii *= 4
    rng = np.random.default_rng(13)
    fields = np.zeros((f.n, 3))
    fields[:, :2] = rng.uniform(0.0, 1e-3, size=(f.n, 2))
    r = (lambda z: np.asarray(z, np.float32).astype(np.float64)) if precision != "fp64" \
        else np.asarray
    x, a, s, fl = (torch.from_numpy(np.ascontiguousarray(r(z))).cuda()
                   for z in (f.positions, f.strengths, 2.0 * f.radii, fields))
    wh, fh = kernels.les_test_filter(x, a, s, fl, precision=precision)
    wref = kernels.vorticity_field_at(x, x, a, s, precision="fp64")
    fref = kernels.vorticity_field_at(x, x, fl, s, precision="fp64")
    ew = float((wh - wref).abs().max() / wref.abs().max())
    ef = float((fh[:, :2] - fref[:, :2]).abs().max() / fref[:, :2].abs().max())
    print(f"{precision}: test vorticity {ew:.2e}, filtered fields {ef:.2e}")
    assert ew <= tol and ef <= tol
    assert float(fh[:, 2].abs().max()) == 0.0
    assert kernels.device_errors() == 0

