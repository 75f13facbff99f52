"""Drop-in physics module for ``vpmModule.ParticleSystem``.

Exports the eight module-level functions that ``ParticleSystem`` calls on
``self.physics`` (OpenONDA/solvers/VPM/vpmModule.py:141-154 selects the module; call
sites at vpmModule.py:259,293,302,321,333,343,607,640,644,677,681,685,704,753,759,765,
774,803,810,817,827), with the same names, positional arguments and return types as
OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py:

* numpy float64 inputs (or host torch tensors) -> numpy arrays (host tensors), scalars
  as Python floats, with one
  host->device copy per input and one device->host copy of the result, as the reference
  wrapper does (ParticlesPhysicsCuda.py:16-34);
* CUDA torch tensors -> CUDA torch tensors (scalars as 0-d tensors, no host sync).

The arithmetic is the library's FP64 path by default (the exact drop-in).  Select the
FP32-compensated path with ``set_precision("fp32c")`` or per call with
``precision="fp32c"``.  There is no CPU fallback: without the CUDA library or a B200
the functions raise.

Host radii that are all equal select the library's uniform-core sweeps (same values, fewer
operations).  Reference behaviours kept: probe sums skip pairs with r^2 <= 1e-8; self sums skip
j == i and use the pair core (sigma_i + sigma_j)/2; PSE uses the target's viscosity;
helicity and enstrophy keep the wrapper's extra 1/(4 pi) (``set_reference_scaling``
turns it off).  Reference defects not kept: scalar accumulators start at zero (the
reference leaves them uninitialised, ParticlesPhysicsCuda.py:545,655,764) and
``get_vorticity_field_at`` returns one row per target (ParticlesPhysicsCuda.py:200,207
size the result by the number of sources).
"""
from __future__ import annotations

import numpy as np
import torch

from .. import kernels

_state = {"precision": "fp64", "ref_extra_4pi": True, "device": None}


def set_precision(precision: str) -> None:
    """Module-wide arithmetic: "fp64" (default), "fp32c" or "fp32c_refined"."""
    from .._lib import precision_code

    precision_code(precision)
    _state["precision"] = precision


def get_precision() -> str:
    return _state["precision"]


def set_reference_scaling(extra_4pi: bool) -> None:
    """Keep (True, default) or drop the wrappers' second 1/(4 pi) on helicity/enstrophy."""
    _state["ref_extra_4pi"] = bool(extra_4pi)


def set_device(device) -> None:
    _state["device"] = torch.device(device) if device is not None else None


def _device():
    if _state["device"] is not None:
        return _state["device"]
    if not torch.cuda.is_available():
        raise RuntimeError("ParticlesPhysicsB200 needs a CUDA device (B200); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def _prep(args):
    """Move inputs to the device; return (tensors, mode).

    mode "cuda": every input is a CUDA tensor, results stay on the device;
    mode "torch": host torch tensors (pinned ones copy fastest), results come back as host
    tensors; mode "numpy": anything else, results come back as numpy arrays."""
    if all(isinstance(a, torch.Tensor) and a.is_cuda for a in args):
        return list(args), "cuda"
    dev = _device()
    mode = "torch" if all(isinstance(a, torch.Tensor) for a in args) else "numpy"
    out = []
    for a in args:
        if isinstance(a, torch.Tensor):
            t = a.to(device=dev, dtype=torch.float64, non_blocking=True)
        else:
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64))).to(dev)
        out.append(t)
    return out, mode


def _ret(t, mode):
    if mode == "cuda":
        return t
    if t.dim() == 0:
        return float(t.item())
    if mode == "torch":
        # host tensors in, host tensors out: copy into page-locked memory (the caching host
        # allocator reuses it), which the copy engine fills at full PCIe/C2C speed
        out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        out.copy_(t, non_blocking=True)
        torch.cuda.current_stream(t.device).synchronize()
        return out
    return t.cpu().numpy()


def _prec(precision):
    return _state["precision"] if precision is None else precision


def _uniform(radii):
    """Host radii that are all equal select the uniform-core sweeps (same pair values, 2 FP32
    operations fewer per pair); device radii are not inspected (that would need a sync)."""
    if isinstance(radii, torch.Tensor):
        if radii.is_cuda:
            return False
        radii = radii.numpy()
    r = np.asarray(radii).reshape(-1)
    return bool(r.size) and bool(np.all(r == r[0]))


def get_induced_velocity_at(target_positions, particles_positions, particles_strengths,
                            particles_radii, precision=None):
    (t, x, a, s), np_mode = _prep((target_positions, particles_positions, particles_strengths,
                                   particles_radii))
    return _ret(kernels.induced_velocity_at(t, x, a, s, precision=_prec(precision)), np_mode)


def get_selfinduced_velocity(particles_positions, particles_strengths, particles_radii,
                             precision=None):
    uc = _uniform(particles_radii)
    (x, a, s), np_mode = _prep((particles_positions, particles_strengths, particles_radii))
    return _ret(kernels.selfinduced_velocity(x, a, s, precision=_prec(precision),
                                             uniform_core=uc), np_mode)


def get_vorticity_field_at(target_positions, particle_positions, particle_strengths,
                           particle_radii, precision=None):
    (t, x, a, s), np_mode = _prep((target_positions, particle_positions, particle_strengths,
                                   particle_radii))
    return _ret(kernels.vorticity_field_at(t, x, a, s, precision=_prec(precision)), np_mode)


def get_strength_gradients(particle_positions, particle_strengths, particle_radii,
                           precision=None):
    uc = _uniform(particle_radii)
    (x, a, s), np_mode = _prep((particle_positions, particle_strengths, particle_radii))
    return _ret(kernels.strength_gradients(x, a, s, precision=_prec(precision),
                                           uniform_core=uc), np_mode)


def get_strength_gradients_PSE(positions, strengths, radii, viscosities, precision=None):
    uc = _uniform(radii)
    (x, a, s, v), np_mode = _prep((positions, strengths, radii, viscosities))
    return _ret(kernels.strength_gradients_pse(x, a, s, v, precision=_prec(precision),
                                               uniform_core=uc), np_mode)


def get_total_kinetic_energy(particles_positions, particles_strengths, particles_radii,
                             precision=None):
    (x, a, s), np_mode = _prep((particles_positions, particles_strengths, particles_radii))
    return _ret(kernels.total_kinetic_energy(x, a, s, precision=_prec(precision)), np_mode)


def get_total_helicity(particles_positions, particles_strengths, particles_radii,
                       precision=None):
    (x, a, s), np_mode = _prep((particles_positions, particles_strengths, particles_radii))
    return _ret(kernels.total_helicity(x, a, s, ref_extra_4pi=_state["ref_extra_4pi"],
                                       precision=_prec(precision)), np_mode)


def get_total_enstrophy(particles_positions, particles_strengths, particles_radii,
                        precision=None):
    uc = _uniform(particles_radii)
    (x, a, s), np_mode = _prep((particles_positions, particles_strengths, particles_radii))
    return _ret(kernels.total_enstrophy(x, a, s, ref_extra_4pi=_state["ref_extra_4pi"],
                                        precision=_prec(precision), uniform_core=uc), np_mode)


def get_selfinduced_velocity_and_strength_gradients(particles_positions, particles_strengths,
                                                    particles_radii, precision=None):
    """Fused ``get_selfinduced_velocity`` + ``get_strength_gradients`` (one sweep)."""
    uc = _uniform(particles_radii)
    (x, a, s), np_mode = _prep((particles_positions, particles_strengths, particles_radii))
    u, g = kernels.velocity_and_strength_gradients(x, a, s, precision=_prec(precision),
                                                   uniform_core=uc)
    return _ret(u, np_mode), _ret(g, np_mode)
