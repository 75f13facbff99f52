"""Initial conditions and lattices on the GPU (openonda_b200.utilities) against the
reference's own outputs (tests/golden/ic.npz) and, at sizes beyond the fixtures, against
the pinned oracle (oracle/vpm_ic.py)."""
import numpy as np
import pytest
import torch

from oracle import vpm_ic
from conftest import golden, ic_cases, normwise

pytestmark = pytest.mark.gpu

CASES = ic_cases()
TOL = 1e-14  # CUDA's double transcendental functions vs numba fastmath: a few ulp
TURB_TOL = 1e-12  # cuFFT vs numpy's FFT on a 16^3 grid


def _device(name, c, **kw):
    from openonda_b200.utilities import vpm_flow_models as fm
    from openonda_b200.utilities import vpm_solver_helper as sh

    if name.startswith("turb"):
        return fm.isotropic_turbulence_vpm(c["box"], c["d"], c["radius"], **kw)
    if name.startswith("ring"):
        return fm.vortex_ring_vpm(c["positions"], c["volumes"], *c["args"])
    if name == "lamb":
        return fm.lamb_oseen_vpm(c["positions"], c["volumes"], *c["args"])
    if name == "rect2":
        return sh.get_2D_rectangular_point_distribuition(c["box"], c["spacing"], **kw)
    if name.startswith("rect"):
        return sh.get_rectangular_point_distribuition(c["box"], c["spacing"], **kw)
    if name == "hex":
        return sh.get_hexagonal_point_distribution(c["box"], c["spacing"], **kw)
    return sh.get_cylindrical_point_distribuition(c["d"], c["radius"], c["height"],
                                                  c["center"], c["axis"], **kw)


@pytest.mark.parametrize("name", sorted(CASES))
def test_ic_device_vs_reference(name):
    g = golden("ic.npz")
    out = _device(name, CASES[name])
    if name.startswith("ring") or name == "lamb":
        keys = ("velocities", "strengths", "radii", "viscosities")
    elif name.startswith("turb"):
        keys = ("positions", "velocities", "strengths", "radii")
    else:
        keys = ("points", "volumes")
    for k, v in zip(keys, out):
        assert isinstance(v, np.ndarray)
        ref = g[f"{name}/{k}"]
        assert v.shape == ref.shape, (k, v.shape)
        tol = TURB_TOL if name.startswith("turb") else TOL
        assert normwise(v, ref) <= tol, (k, normwise(v, ref))
    if name.startswith(("rect", "hex")):  # plain IEEE arithmetic: bit-exact
        assert np.array_equal(out[0], g[f"{name}/points"])


def test_lattices_return_device_tensors():
    p, v = _device("rect3b", CASES["rect3b"], device="cuda")
    assert p.is_cuda and v.is_cuda and p.dtype == torch.float64
    g = golden("ic.npz")
    assert np.array_equal(p.cpu().numpy(), g["rect3b/points"])


def test_vortex_ring_million_particles_vs_oracle():
    from openonda_b200.utilities import vpm_flow_models as fm
    from openonda_b200.utilities import vpm_solver_helper as sh

    box = [-0.4, 0.4, -1.4, 1.4, -1.4, 1.4]
    pts, vols = sh.get_rectangular_point_distribuition(box, 0.018, device="cuda")
    assert pts.shape[0] > 1_000_000
    out = fm.vortex_ring_vpm(pts, vols, 0.03, 1e-5, np.zeros(3), 1.0, 1.0, 0.05, 0.01, 0.0, 7)
    assert all(t.is_cuda for t in out)
    ref = vpm_ic.vortex_ring_vpm(pts.cpu().numpy(), vols.cpu().numpy(), 0.03, 1e-5,
                                 np.zeros(3), 1.0, 1.0, 0.05, 0.01, 0.0, 7)
    assert normwise(out[1].cpu().numpy(), ref[1]) <= 1e-13
    total = out[1].norm(dim=1).sum().item()
    assert abs(total - 2 * np.pi) <= 1e-11 * 2 * np.pi


def test_ic_errors():
    from openonda_b200 import _lib
    from openonda_b200.utilities import vpm_flow_models as fm
    from openonda_b200.utilities import vpm_solver_helper as sh

    far = np.full((10, 3), 100.0)
    with pytest.raises(ZeroDivisionError):
        fm.vortex_ring_vpm(far, np.ones(10), 0.1, 0.0, np.zeros(3), 1.0, 1.0, 0.01)
    with pytest.raises(ValueError):
        sh.get_cylindrical_point_distribuition(0.1, axis="w")
    with pytest.raises(_lib.VPMError):
        sh.get_rectangular_point_distribuition([0, 1, 0, 1, 0, 1], -0.1)
    with pytest.raises(_lib.VPMError):
        sh.get_cylindrical_point_distribuition(5.0, radius=1.0)
    e = fm.lamb_oseen_vpm(np.zeros((0, 3)), np.zeros(0), 0.1, 0.0, np.zeros(3), 1.0, 0.1)
    assert e[1].shape == (0, 3)
