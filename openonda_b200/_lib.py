"""ctypes binding of ``libvpm_b200.so`` (the C ABI in ``include/vpm_b200.h``).

The library is built in-tree by :mod:`openonda_b200.build`.  There is no fallback: if
the shared library is missing or cannot be loaded, every compute call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libvpm_b200.so")

VPM_OK = 0
VPM_ERR_ARG = 1
VPM_ERR_ALIGN = 2
VPM_ERR_WORKSPACE = 3
VPM_ERR_CUDA = 4
VPM_ERR_ARCH = 5

PRECISIONS = {"fp64": 0, "fp32c": 1, "fp32c_refined": 2}

OPS = {
    "selfinduced_velocity": 0,
    "induced_velocity_at": 1,
    "vorticity_field_at": 2,
    "strength_gradients": 3,
    "strength_gradients_pse": 4,
    "total_kinetic_energy": 5,
    "total_helicity": 6,
    "total_enstrophy": 7,
    "velocity_and_strength_gradients": 8,
    "rhs_vjp": 9,
    "rhs_vjp_pse": 10,
    "kinetic_energy_grad": 11,
    "les_step_sums": 12,
    "les_test_filter": 13,
}

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I = ctypes.c_int
_SZ = ctypes.c_size_t
_D = ctypes.c_double

# name -> (argtypes, restype)
SIGNATURES = {
    "vpm_abi_version": ([], _I),
    "vpm_last_error": ([], ctypes.c_char_p),
    "vpm_check_device": ([], _I),
    "vpm_binary_info": ([ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "vpm_device_errors": ([ctypes.POINTER(_I), _I], _I),
    "vpm_selftest_bounded_wait": ([_P, _P], _I),
    "vpm_workspace_bytes": ([_I, _I, _I64, _I64], _SZ),
    "vpm_plan_info": ([_I, _I, _I64, _I64, ctypes.POINTER(_I64), ctypes.POINTER(_I),
                       ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "vpm_induced_velocity_at": ([_P, _I64, _P, _P, _P, _I64, _P, _I, _P, _SZ, _P], _I),
    "vpm_selfinduced_velocity": ([_P, _P, _P, _I64, _P, _I, _P, _SZ, _P], _I),
    "vpm_vorticity_field_at": ([_P, _I64, _P, _P, _P, _I64, _P, _I, _P, _SZ, _P], _I),
    "vpm_strength_gradients": ([_P, _P, _P, _I64, _P, _I, _P, _SZ, _P], _I),
    "vpm_strength_gradients_pse": ([_P, _P, _P, _P, _I64, _P, _I, _P, _SZ, _P], _I),
    "vpm_total_kinetic_energy": ([_P, _P, _P, _I64, _P, _I, _P, _SZ, _P], _I),
    "vpm_total_helicity": ([_P, _P, _P, _I64, _I, _P, _I, _P, _SZ, _P], _I),
    "vpm_total_enstrophy": ([_P, _P, _P, _I64, _I, _P, _I, _P, _SZ, _P], _I),
    "vpm_velocity_and_strength_gradients": ([_P, _P, _P, _I64, _P, _P, _I, _P, _SZ, _P], _I),
    "vpm_set_symmetric_min_n": ([_I64], _I64),
    "vpm_sweep_launches": ([_I, _I, _I64, _I64], _I64),
    "vpm_les_step_sums": ([_P, _P, _P, _I64, _P, _P, _P, _P, _I, _I, _P, _SZ, _P], _I),
    "vpm_rhs_vjp": ([_P, _P, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _I, _P, _SZ, _P], _I),
    "vpm_kinetic_energy_grad": ([_P, _P, _P, _I64, _P, _P, _P, _I, _P, _SZ, _P], _I),
    "vpm_record_bytes": ([_I], _SZ),
    "vpm_pack_records": ([_P, _P, _P, _P, _I64, _I, _P, _P], _I),
    "vpm_sweep_records": ([_I, _P, _I64, _I64, _I64, _I, _P, _P, _I, _P, _SZ, _P], _I),
    "vpm_pairs_layout": ([_I, _I, _I64, _P, _P, _P, _P, _P], _I),
    "vpm_sweep_pairs_partial": ([_I, _P, _I64, _I64, _I64, _I64, _I64, _P, _I, _P, _SZ, _P],
                                _I),
    "vpm_finalize_pairs_partial": ([_I, _P, _P, _I64, _I64, _P, _P, _I, _P], _I),
    "vpm_selfinduced_velocity_noalloc": ([_P, _P, _P, _I64, _P, _I, _P], _I),
    "vpm_axpy": ([_P, _P, ctypes.c_double, _I64, _P, _P], _I),
    "vpm_rk4_combine": ([_P, _P, _P, _P, _P, ctypes.c_double, _I64, _P, _P], _I),
    "vpm_bdf_update": ([_P, _P, _P, _P, _P, _I64, _I, ctypes.c_double, _P], _I),
    "vpm_core_spreading": ([_P, _P, _P, _I64, ctypes.c_double, ctypes.c_double, _P], _I),
    "vpm_les_workspace_bytes": ([_I64], _SZ),
    "vpm_les_update": ([_P, _P, _P, _I64, _I, _P, _P, _P, _P, _SZ, _P], _I),
    "vpm_les_test_filter": ([_P, _P, _P, _P, _I64, _P, _P, _I, _P, _SZ, _P], _I),
    "vpm_les_lsq_weights": ([_P, _P, _P, _P, _I64, _P, _P], _I),
    "vpm_les_lsq_update": ([_P, _P, _P, _P, _I64, _P, _P, _P], _I),
    "vpm_relax_strengths": ([_P, _P, _I64, ctypes.c_double, _P], _I),
    "vpm_particle_diagnostics": ([_P, _P, _I64, _P, _P], _I),
    "vpm_ic_workspace_bytes": ([_I64], _SZ),
    "vpm_ic_vortex_ring": ([_P, _P, _I64] + [_D] * 11 + [_P, _P, _P, _P, _SZ, _P], _I),
    "vpm_ic_lamb_oseen": ([_P, _P, _I64] + [_D] * 10 + [_P, _P, _P, _P], _I),
    "vpm_lattice_rectangular": ([_P, _D, _I, _P, _P, _I64, ctypes.POINTER(_I64), _P], _I),
    "vpm_lattice_hexagonal": ([_P, _D, _P, _P, _I64, ctypes.POINTER(_I64), _P], _I),
    "vpm_lattice_cylindrical": ([_D, _D, _D, _P, _I, _P, _P, _I64, ctypes.POINTER(_I64), _P],
                                _I),
    "vpm_launch_fma_peak": ([_I, _I, _I, _I, _P, _P], _I),
}

_lock = threading.Lock()
_lib = None


class VPMError(RuntimeError):
    """Raised when a libvpm_b200 entry point returns a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"libvpm_b200 error {code}: {message}")
        self.code = code


def load() -> ctypes.CDLL:
    """Load the library once; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `python -m openonda_b200.build` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def check(rc: int) -> None:
    if rc != VPM_OK:
        msg = load().vpm_last_error()
        raise VPMError(rc, msg.decode() if msg else "")


UNIFORM_CORE = 0x100  # VPM_UNIFORM_CORE: every particle has the same core radius


def precision_code(precision: str, uniform_core: bool = False) -> int:
    try:
        code = PRECISIONS[precision]
    except KeyError:
        raise ValueError(f"unknown precision {precision!r}; choose from {sorted(PRECISIONS)}")
    return code | (UNIFORM_CORE if uniform_core else 0)
