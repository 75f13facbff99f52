"""CPU oracle for the VPM pair sums (TEST INFRASTRUCTURE, not product code).

The oracle is a plain-C FP64 restatement of OpenONDA's two physics modules
(``OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py`` and ``ParticlesPhysics.py``),
compiled by :mod:`oracle.build` into ``oracle/_build/``.  Only the test suite,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline leg and its reference
arm) use it, always as the checker or the timed CPU baseline -- never as a stand-in
for the CUDA library.

Two builds of the same source exist:

* ``libvpm_oracle.so``      -O2, strict IEEE arithmetic: the parity oracle.
* ``libvpm_oracle_fast.so`` -O3 -ffast-math: the timed CPU baseline, mirroring the
  reference's ``@njit(parallel=True, fastmath=True)`` CPU module.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every function here against
golden vectors produced by running the reference's own modules
(``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_LIBS: dict[str, ctypes.CDLL] = {}

_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.c_int64

_SIGS = {
    "oracle_gpu_induced_velocity_at": ([_D, _I64, _D, _D, _D, _I64, _D], None),
    "oracle_gpu_selfinduced_velocity": ([_D, _D, _D, _I64, _D], None),
    "oracle_gpu_vorticity_field_at": ([_D, _I64, _D, _D, _D, _I64, _D], None),
    "oracle_gpu_strength_gradients": ([_D, _D, _D, _I64, _D], None),
    "oracle_gpu_strength_gradients_pse": ([_D, _D, _D, _D, _I64, _D], None),
    "oracle_gpu_total_kinetic_energy": ([_D, _D, _D, _I64], ctypes.c_double),
    "oracle_gpu_total_helicity": ([_D, _D, _D, _I64, ctypes.c_int], ctypes.c_double),
    "oracle_gpu_total_enstrophy": ([_D, _D, _D, _I64, ctypes.c_int], ctypes.c_double),
    "oracle_cpu_induced_velocity_at": ([_D, _I64, _D, _D, _D, _I64, _D], None),
    "oracle_cpu_selfinduced_velocity": ([_D, _D, _D, _I64, _D], None),
    "oracle_cpu_vorticity_field_at": ([_D, _I64, _D, _D, _D, _I64, _D], None),
    "oracle_cpu_strength_gradients": ([_D, _D, _D, _I64, _D], None),
    "oracle_cpu_strength_gradients_pse": ([_D, _D, _D, _D, _I64, _D], None),
    "oracle_cpu_total_kinetic_energy": ([_D, _D, _D, _I64], ctypes.c_double),
    "oracle_cpu_total_helicity": ([_D, _D, _D, _I64], ctypes.c_double),
    "oracle_cpu_total_enstrophy": ([_D, _D, _D, _I64], ctypes.c_double),
    "oracle_gpu_selfinduced_velocity_range": ([_D, _D, _D, _I64, _I64, _I64, _D], None),
    "oracle_gpu_strength_gradients_range": ([_D, _D, _D, _I64, _I64, _I64, _D], None),
    "oracle_cpu_selfinduced_velocity_range": ([_D, _D, _D, _I64, _I64, _I64, _D], None),
    "oracle_cpu_strength_gradients_range": ([_D, _D, _D, _I64, _I64, _I64, _D], None),
    "oracle_num_threads": ([], ctypes.c_int),
    "oracle_set_num_threads": ([ctypes.c_int], None),
}


def lib(fast: bool = False) -> ctypes.CDLL:
    """Load (building on first use if needed) the oracle shared library."""
    name = "libvpm_oracle_fast.so" if fast else "libvpm_oracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_BUILD, name)
    if not os.path.exists(path):
        from . import build as _build

        _build.build()
    cdll = ctypes.CDLL(path)
    for fname, (args, res) in _SIGS.items():
        fn = getattr(cdll, fname)
        fn.argtypes = args
        fn.restype = res
    _LIBS[name] = cdll
    return cdll


def _f64(a, cols=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if cols is not None and (a.ndim != 2 or a.shape[1] != cols):
        raise ValueError(f"expected an (n, {cols}) array, got shape {a.shape}")
    return a


def _p(a):
    return a.ctypes.data_as(_D)


class _Module:
    """Functions with the reference's names and argument order, for one semantics."""

    def __init__(self, prefix: str, fast: bool):
        self._prefix = prefix
        self._fast = fast

    def _fn(self, name):
        return getattr(lib(self._fast), f"oracle_{self._prefix}_{name}")

    def get_induced_velocity_at(self, targets, positions, strengths, radii):
        t, x, a, s = _f64(targets, 3), _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        out = np.zeros_like(t)
        self._fn("induced_velocity_at")(_p(t), len(t), _p(x), _p(a), _p(s), len(x), _p(out))
        return out

    def get_selfinduced_velocity(self, positions, strengths, radii):
        x, a, s = _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        out = np.zeros_like(x)
        self._fn("selfinduced_velocity")(_p(x), _p(a), _p(s), len(x), _p(out))
        return out

    def get_vorticity_field_at(self, targets, positions, strengths, radii):
        t, x, a, s = _f64(targets, 3), _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        out = np.zeros_like(t)
        self._fn("vorticity_field_at")(_p(t), len(t), _p(x), _p(a), _p(s), len(x), _p(out))
        return out

    def get_strength_gradients(self, positions, strengths, radii):
        x, a, s = _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        out = np.zeros_like(x)
        self._fn("strength_gradients")(_p(x), _p(a), _p(s), len(x), _p(out))
        return out

    def selfinduced_velocity_range(self, positions, strengths, radii, t0, t1):
        """Self-induced velocity of targets [t0, t1) against all particles."""
        x, a, s = _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        out = np.zeros((t1 - t0, 3))
        self._fn("selfinduced_velocity_range")(_p(x), _p(a), _p(s), len(x), t0, t1, _p(out))
        return out

    def strength_gradients_range(self, positions, strengths, radii, t0, t1):
        """Stretching of targets [t0, t1) against all particles."""
        x, a, s = _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        out = np.zeros((t1 - t0, 3))
        self._fn("strength_gradients_range")(_p(x), _p(a), _p(s), len(x), t0, t1, _p(out))
        return out

    def get_strength_gradients_PSE(self, positions, strengths, radii, viscosities):
        x, a, s, v = _f64(positions, 3), _f64(strengths, 3), _f64(radii), _f64(viscosities)
        out = np.zeros_like(x)
        self._fn("strength_gradients_pse")(_p(x), _p(a), _p(s), _p(v), len(x), _p(out))
        return out

    def get_total_kinetic_energy(self, positions, strengths, radii):
        x, a, s = _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        return float(self._fn("total_kinetic_energy")(_p(x), _p(a), _p(s), len(x)))

    def get_total_helicity(self, positions, strengths, radii, ref_extra_4pi=True):
        x, a, s = _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        if self._prefix == "cpu":
            return float(self._fn("total_helicity")(_p(x), _p(a), _p(s), len(x)))
        return float(self._fn("total_helicity")(_p(x), _p(a), _p(s), len(x), int(ref_extra_4pi)))

    def get_total_enstrophy(self, positions, strengths, radii, ref_extra_4pi=True):
        x, a, s = _f64(positions, 3), _f64(strengths, 3), _f64(radii)
        if self._prefix == "cpu":
            return float(self._fn("total_enstrophy")(_p(x), _p(a), _p(s), len(x)))
        return float(self._fn("total_enstrophy")(_p(x), _p(a), _p(s), len(x), int(ref_extra_4pi)))


#: GPU semantics (ParticlesPhysicsCuda.py), strict arithmetic: the parity oracle.
gpu = _Module("gpu", fast=False)
#: CPU semantics (ParticlesPhysics.py), strict arithmetic.
cpu = _Module("cpu", fast=False)
#: CPU semantics, fast-math build: the timed CPU baseline.
cpu_fast = _Module("cpu", fast=True)
#: GPU semantics, fast-math build.
gpu_fast = _Module("gpu", fast=True)


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def set_num_threads(n: int) -> None:
    lib().oracle_set_num_threads(int(n))
    lib(fast=True).oracle_set_num_threads(int(n))
