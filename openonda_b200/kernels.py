"""Tensor-level access to the B200 pair-sum kernels.

Every function takes CUDA ``torch.float64`` tensors in the reference's layout
(positions/strengths ``(n,3)``, radii/viscosities ``(n,)``), runs on the current CUDA
stream, and returns new CUDA tensors (scalars as 0-d tensors, without a host sync).

``precision``:

* ``"fp64"``  -- FP64 arithmetic, the exact drop-in for the reference's Numba-CUDA
  kernels (agreement to 1e-12 relative).
* ``"fp32c"`` -- pair terms in FP32 (inputs rounded to FP32 once), FP32 partial sums over
  windows of 32 sources carried in FP64, FP64 outputs.
* ``"fp32c_refined"`` -- as ``fp32c`` with one Newton step on the hardware rsqrt.

``uniform_core=True`` (self sums): the caller guarantees that all radii are equal; the pair
core is then sigma_i and the sweeps skip forming it (same values, 2 FP32 operations fewer per
pair).  The library checks the claim while packing and reports a false one through
:func:`device_errors` (bit 1).  ``ParticleSystem`` sets it by itself when its cores are equal.

Scratch space comes from PyTorch's caching allocator and is handed to the C ABI.
"""
from __future__ import annotations

import torch

from . import _lib

_F64 = torch.float64


def _check_vec(name, t, n=None):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must be a CUDA tensor (got {t.device})")
    if t.dtype != _F64:
        raise TypeError(f"{name} must be float64 (got {t.dtype})")
    if t.dim() != 2 or t.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n, 3), got {tuple(t.shape)}")
    if n is not None and t.shape[0] != n:
        raise ValueError(f"{name} has {t.shape[0]} rows, expected {n}")
    return t.contiguous()


def _check_scalar(name, t, n):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must be a CUDA tensor (got {t.device})")
    if t.dtype != _F64:
        raise TypeError(f"{name} must be float64 (got {t.dtype})")
    t = t.reshape(-1)
    if t.shape[0] != n:
        raise ValueError(f"{name} has {t.shape[0]} entries, expected {n}")
    return t.contiguous()


def _same_device(*ts):
    dev = ts[0].device
    for t in ts[1:]:
        if t.device != dev:
            raise ValueError("all tensors must be on the same CUDA device")
    return dev


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def workspace_bytes(op: str, precision: str, m: int, n: int, uniform_core: bool = False) -> int:
    lib = _lib.load()
    nbytes = lib.vpm_workspace_bytes(_lib.OPS[op], _lib.precision_code(precision, uniform_core),
                                     int(m), int(n))
    if nbytes == 0 and m > 0 and n > 0:
        msg = lib.vpm_last_error()
        raise _lib.VPMError(_lib.VPM_ERR_CUDA, msg.decode() if msg else "workspace query failed")
    return int(nbytes)


def plan_info(op: str, precision: str, m: int, n: int, uniform_core: bool = False) -> dict:
    import ctypes

    lib = _lib.load()
    tb, sp, th, r = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _lib.check(lib.vpm_plan_info(_lib.OPS[op], _lib.precision_code(precision, uniform_core),
                                 int(m), int(n),
                                 ctypes.byref(tb), ctypes.byref(sp), ctypes.byref(th),
                                 ctypes.byref(r)))
    return dict(target_blocks=tb.value, splits=sp.value, threads=th.value,
                targets_per_thread=r.value)


def _workspace(op, precision, m, n, dev, uniform_core=False):
    nbytes = workspace_bytes(op, precision, m, n, uniform_core)
    return torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev), nbytes


def _self_inputs(positions, strengths, radii):
    positions = _check_vec("positions", positions)
    n = positions.shape[0]
    strengths = _check_vec("strengths", strengths, n)
    radii = _check_scalar("radii", radii, n)
    dev = _same_device(positions, strengths, radii)
    return positions, strengths, radii, n, dev


def selfinduced_velocity(positions, strengths, radii, precision="fp64", uniform_core=False):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    out = torch.empty((n, 3), dtype=_F64, device=dev)
    ws, nb = _workspace("selfinduced_velocity", precision, n, n, dev, uniform_core)
    _lib.check(_lib.load().vpm_selfinduced_velocity(
        _ptr(x), _ptr(a), _ptr(s), n, _ptr(out),
        _lib.precision_code(precision, uniform_core), _ptr(ws),
        ws.numel(), _stream(dev)))
    return out


def strength_gradients(positions, strengths, radii, precision="fp64", uniform_core=False):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    out = torch.empty((n, 3), dtype=_F64, device=dev)
    ws, nb = _workspace("strength_gradients", precision, n, n, dev, uniform_core)
    _lib.check(_lib.load().vpm_strength_gradients(
        _ptr(x), _ptr(a), _ptr(s), n, _ptr(out),
        _lib.precision_code(precision, uniform_core), _ptr(ws),
        ws.numel(), _stream(dev)))
    return out


def velocity_and_strength_gradients(positions, strengths, radii,
                                    precision="fp64", uniform_core=False):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    u = torch.empty((n, 3), dtype=_F64, device=dev)
    g = torch.empty((n, 3), dtype=_F64, device=dev)
    ws, nb = _workspace("velocity_and_strength_gradients", precision, n, n, dev, uniform_core)
    _lib.check(_lib.load().vpm_velocity_and_strength_gradients(
        _ptr(x), _ptr(a), _ptr(s), n, _ptr(u), _ptr(g),
        _lib.precision_code(precision, uniform_core),
        _ptr(ws), ws.numel(), _stream(dev)))
    return u, g


def les_step_sums(positions, strengths, radii, ref_extra_4pi=True,
                  precision="fp64", uniform_core=False):
    """Velocity, stretching, particle vorticity and the enstrophy filter sum of one
    dynamic-LES step, from one sweep over the same state.  Returns (u, dalpha_dt, omega,
    enstrophy) with the enstrophy as a 0-d tensor."""
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    u = torch.empty((n, 3), dtype=_F64, device=dev)
    g = torch.empty((n, 3), dtype=_F64, device=dev)
    w = torch.empty((n, 3), dtype=_F64, device=dev)
    e = torch.empty((), dtype=_F64, device=dev)
    ws, nb = _workspace("les_step_sums", precision, n, n, dev, uniform_core)
    _lib.check(_lib.load().vpm_les_step_sums(
        _ptr(x), _ptr(a), _ptr(s), n, _ptr(u), _ptr(g), _ptr(w), _ptr(e),
        int(bool(ref_extra_4pi)),
        _lib.precision_code(precision, uniform_core), _ptr(ws), ws.numel(),
        _stream(dev)))
    return u, g, w, e


def les_test_filter(positions, strengths, test_radii, fields, precision="fp64"):
    """The two test-filter sums of the least-squares LES coefficient in one sweep: the
    vorticity filter sum with cores ``test_radii`` and the same filter applied to the first two
    columns of ``fields`` (n, 3).  Returns (test_vorticity, test_filtered), both (n, 3)."""
    x, a, s, n, dev = _self_inputs(positions, strengths, test_radii)
    f = _check_vec("fields", fields, n)
    _same_device(x, f)
    w = torch.empty((n, 3), dtype=_F64, device=dev)
    fh = torch.empty((n, 3), dtype=_F64, device=dev)
    ws, nb = _workspace("les_test_filter", precision, n, n, dev)
    _lib.check(_lib.load().vpm_les_test_filter(
        _ptr(x), _ptr(a), _ptr(s), _ptr(f), n, _ptr(w), _ptr(fh),
        _lib.precision_code(precision), _ptr(ws), ws.numel(), _stream(dev)))
    return w, fh


def strength_gradients_pse(positions, strengths, radii, viscosities,
                           precision="fp64", uniform_core=False):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    v = _check_scalar("viscosities", viscosities, n)
    _same_device(x, v)
    out = torch.empty((n, 3), dtype=_F64, device=dev)
    ws, nb = _workspace("strength_gradients_pse", precision, n, n, dev, uniform_core)
    _lib.check(_lib.load().vpm_strength_gradients_pse(
        _ptr(x), _ptr(a), _ptr(s), _ptr(v), n, _ptr(out),
        _lib.precision_code(precision, uniform_core),
        _ptr(ws), ws.numel(), _stream(dev)))
    return out


def _probe(fn_name, op, targets, positions, strengths, radii, precision):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    t = _check_vec("targets", targets)
    _same_device(x, t)
    m = t.shape[0]
    out = torch.empty((m, 3), dtype=_F64, device=dev)
    ws, nb = _workspace(op, precision, m, n, dev)
    fn = getattr(_lib.load(), fn_name)
    _lib.check(fn(_ptr(t), m, _ptr(x), _ptr(a), _ptr(s), n, _ptr(out),
                  _lib.precision_code(precision), _ptr(ws), ws.numel(), _stream(dev)))
    return out


def induced_velocity_at(targets, positions, strengths, radii, precision="fp64"):
    return _probe("vpm_induced_velocity_at", "induced_velocity_at", targets, positions,
                  strengths, radii, precision)


def vorticity_field_at(targets, positions, strengths, radii, precision="fp64"):
    return _probe("vpm_vorticity_field_at", "vorticity_field_at", targets, positions,
                  strengths, radii, precision)


def total_kinetic_energy(positions, strengths, radii, precision="fp64"):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    out = torch.empty((), dtype=_F64, device=dev)
    ws, nb = _workspace("total_kinetic_energy", precision, n, n, dev)
    _lib.check(_lib.load().vpm_total_kinetic_energy(
        _ptr(x), _ptr(a), _ptr(s), n, _ptr(out), _lib.precision_code(precision), _ptr(ws),
        ws.numel(), _stream(dev)))
    return out


def total_helicity(positions, strengths, radii, ref_extra_4pi=True, precision="fp64"):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    out = torch.empty((), dtype=_F64, device=dev)
    ws, nb = _workspace("total_helicity", precision, n, n, dev)
    _lib.check(_lib.load().vpm_total_helicity(
        _ptr(x), _ptr(a), _ptr(s), n, int(bool(ref_extra_4pi)), _ptr(out),
        _lib.precision_code(precision), _ptr(ws), ws.numel(), _stream(dev)))
    return out


def total_enstrophy(positions, strengths, radii, ref_extra_4pi=True,
                    precision="fp64", uniform_core=False):
    x, a, s, n, dev = _self_inputs(positions, strengths, radii)
    out = torch.empty((), dtype=_F64, device=dev)
    ws, nb = _workspace("total_enstrophy", precision, n, n, dev, uniform_core)
    _lib.check(_lib.load().vpm_total_enstrophy(
        _ptr(x), _ptr(a), _ptr(s), n, int(bool(ref_extra_4pi)), _ptr(out),
        _lib.precision_code(precision, uniform_core), _ptr(ws), ws.numel(), _stream(dev)))
    return out


def set_symmetric_min_n(n: int) -> int:
    """Particle count from which the FP32-compensated self sums (velocity + stretching,
    velocity, PSE, the LES step sums) and the adjoint of (u, S [+ P]) evaluate each unordered
    pair once for both particles; returns the previous value."""
    return int(_lib.load().vpm_set_symmetric_min_n(int(n)))


def sweep_launches(op: str, precision: str, m: int, n: int, uniform_core: bool = False) -> int:
    """Kernel launches of one sweep of ``op`` (sweep and finalize) under the current plan."""
    v = int(_lib.load().vpm_sweep_launches(_lib.OPS[op],
                                           _lib.precision_code(precision, uniform_core),
                                           int(m), int(n)))
    if v < 0:
        raise _lib.VPMError(_lib.VPM_ERR_ARG, f"no plan for {op} at m={m}, n={n}")
    return v


def device_errors(clear: bool = True) -> int:
    import ctypes

    v = ctypes.c_int(0)
    _lib.check(_lib.load().vpm_device_errors(ctypes.byref(v), int(clear)))
    return v.value


def launch_fma_peak(fp64, blocks: int, threads: int, iters: int, sink: torch.Tensor):
    """fp64: False/0 = FP32 FMA, True/1 = FP64 FMA, 2 = FP32 MUFU rsqrt (SFU),
    3 = packed FP32x2 FMA (FFMA2)."""
    _lib.check(_lib.load().vpm_launch_fma_peak(int(fp64), blocks, threads, iters,
                                               sink.data_ptr(), _stream(sink.device)))
