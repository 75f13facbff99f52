"""Particle lattices generated on the GPU.

Same functions, arguments and return values as OpenONDA/utilities/vpm_solver_helper.py
(``get_rectangular_point_distribuition`` :21-68, ``get_2D_rectangular_point_distribuition``
:71-117, ``get_hexagonal_point_distribution`` :120-161,
``get_cylindrical_point_distribuition`` :164-253): ``(points (n,3), volumes (n,))`` as numpy
arrays, or as CUDA tensors when ``device`` names a CUDA device.  Sizes are computed on the
host with the reference's arithmetic; the points are written by the library kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import _lib
from ._dev import cuda_device, stream

epsilon = 1e-9


def gaussian(r, omega_0, a):
    """vpm_solver_helper.py:5-6."""
    return omega_0 * np.exp(-(r ** 2) / a ** 2)


def compute_min_max(x, y, z):
    """vpm_solver_helper.py:10-16 (numpy or tensors)."""
    mm = (lambda t: (float(t.min()), float(t.max())))
    return (*mm(x), *mm(y), *mm(z))


def _run(fn, args_before, args_after, device):
    dev = cuda_device(device)
    lib = _lib.load()
    count = ctypes.c_int64(0)
    _lib.check(getattr(lib, fn)(*args_before, None, None, 0, ctypes.byref(count), *args_after,
                                None))
    n = count.value
    pts = torch.empty((n, 3), dtype=torch.float64, device=dev)
    vols = torch.empty(n, dtype=torch.float64, device=dev)
    if n:
        _lib.check(getattr(lib, fn)(*args_before, pts.data_ptr(), vols.data_ptr(), n,
                                    ctypes.byref(count), *args_after, stream(dev)))
    if device is None:
        return pts.cpu().numpy(), vols.cpu().numpy()
    return pts, vols


def _box(box_limits):
    b = np.ascontiguousarray(np.asarray(box_limits, dtype=np.float64).reshape(-1))
    if b.shape[0] != 6:
        raise ValueError("box_limits must be [xmin, xmax, ymin, ymax, zmin, zmax]")
    return b


def get_rectangular_point_distribuition(box_limits, spacing: float, device=None):
    b = _box(box_limits)
    return _run("vpm_lattice_rectangular", (b.ctypes.data, float(spacing), 3), (), device)


def get_2D_rectangular_point_distribuition(box_limits, spacing: float, device=None):
    b = _box(box_limits)
    return _run("vpm_lattice_rectangular", (b.ctypes.data, float(spacing), 2), (), device)


def get_hexagonal_point_distribution(box_limits, spacing: float, device=None):
    b = _box(box_limits)
    return _run("vpm_lattice_hexagonal", (b.ctypes.data, float(spacing)), (), device)


_AXES = {"x": 0, "y": 1, "z": 2}


def get_cylindrical_point_distribuition(particle_distance: float, radius=1.0, height=2.0,
                                        center=np.array([0, 0, 0]), axis="x", device=None):
    if axis not in _AXES:
        raise ValueError("Invalid axis. Choose from 'x', 'y', or 'z'.")
    c = np.ascontiguousarray(np.asarray(center, dtype=np.float64).reshape(3))
    return _run("vpm_lattice_cylindrical",
                (float(particle_distance), float(radius), float(height), c.ctypes.data,
                 _AXES[axis]), (), device)
