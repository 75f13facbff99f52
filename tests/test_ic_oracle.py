"""Pin the initial-condition / lattice oracle (oracle/vpm_ic.py) to the reference's own
generators: tests/golden/ic.npz holds the outputs of OpenONDA/utilities/vpm_flow_models.py
and vpm_solver_helper.py on the seeded cases of make_golden.ic_cases()."""
import numpy as np
import pytest

from oracle import vpm_ic
from conftest import golden, ic_cases, normwise

CASES = ic_cases()
# numba fastmath in the reference (ring, Lamb-Oseen, cylinder): a few ulp
TOL = 1e-14


def _oracle(name, c):
    if name.startswith("turb"):
        return vpm_ic.isotropic_turbulence_vpm(c["box"], c["d"], c["radius"])
    if name.startswith("ring"):
        return vpm_ic.vortex_ring_vpm(c["positions"], c["volumes"], *c["args"])
    if name == "lamb":
        return vpm_ic.lamb_oseen_vpm(c["positions"], c["volumes"], *c["args"])
    if name == "rect2":
        return vpm_ic.get_2D_rectangular_point_distribuition(c["box"], c["spacing"])
    if name.startswith("rect"):
        return vpm_ic.get_rectangular_point_distribuition(c["box"], c["spacing"])
    if name == "hex":
        return vpm_ic.get_hexagonal_point_distribution(c["box"], c["spacing"])
    return vpm_ic.get_cylindrical_point_distribuition(c["d"], c["radius"], c["height"],
                                                      c["center"], c["axis"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_ic_oracle_vs_reference(name):
    g = golden("ic.npz")
    out = _oracle(name, CASES[name])
    if name.startswith("ring") or name == "lamb":
        keys = ("velocities", "strengths", "radii", "viscosities")
    elif name.startswith("turb"):
        keys = ("positions", "velocities", "strengths", "radii")
    else:
        keys = ("points", "volumes")
    for k, v in zip(keys, out):
        ref = g[f"{name}/{k}"]
        assert v.shape == ref.shape, (k, v.shape, ref.shape)
        e = normwise(v, ref)
        assert e <= TOL, (k, e)


def test_lattice_edge_cases():
    # a box thinner than the spacing still has 1 (odd) point along that axis... plus one:
    # ceil(0/h) + 1 = 1 point, odd
    p, v = vpm_ic.get_rectangular_point_distribuition([0, 1, 0, 1, 0.5, 0.5], 0.25)
    assert p.shape == (5 * 5 * 1, 3) and np.all(p[:, 2] == 0.5) and np.all(v == 0.0)
    with pytest.raises(ValueError):
        vpm_ic.get_cylindrical_point_distribuition(0.1, axis="w")


def test_library_lattice_sizes_match_reference():
    """The lattice sizes are host arithmetic in the library (no device needed): compare the
    size queries with the reference's own point counts."""
    import ctypes

    from openonda_b200 import _lib

    lib = _lib.load()
    g = golden("ic.npz")
    cnt = ctypes.c_int64(-1)
    for name, c in CASES.items():
        if name.startswith("rect") or name == "hex":
            b = np.ascontiguousarray(c["box"], dtype=np.float64)
            if name == "hex":
                rc = lib.vpm_lattice_hexagonal(b.ctypes.data, c["spacing"], None, None, 0,
                                               ctypes.byref(cnt), None)
            else:
                rc = lib.vpm_lattice_rectangular(b.ctypes.data, c["spacing"],
                                                 2 if name == "rect2" else 3, None, None, 0,
                                                 ctypes.byref(cnt), None)
        elif name.startswith("cyl"):
            ctr = np.ascontiguousarray(c["center"], dtype=np.float64)
            rc = lib.vpm_lattice_cylindrical(c["d"], c["radius"], c["height"], ctr.ctypes.data,
                                             "xyz".index(c["axis"]), None, None, 0,
                                             ctypes.byref(cnt), None)
        else:
            continue
        assert rc == 0, lib.vpm_last_error()
        assert cnt.value == len(g[f"{name}/points"]), name
    bad = np.array([0.0, 1.0, 0.0, 1.0, 0.0, 1.0])
    assert lib.vpm_lattice_rectangular(bad.ctypes.data, 0.0, 3, None, None, 0,
                                       ctypes.byref(cnt), None) == _lib.VPM_ERR_ARG
    assert lib.vpm_lattice_cylindrical(0.1, 1.0, 1.0, bad.ctypes.data, 3, None, None, 0,
                                       ctypes.byref(cnt), None) == _lib.VPM_ERR_ARG
