"""Shared plumbing of the device generators: numpy in -> numpy out, CUDA tensors in ->
CUDA tensors out; the work always runs on the GPU (no host path)."""
from __future__ import annotations

import numpy as np
import torch

_F64 = torch.float64


def cuda_device(device=None):
    if not torch.cuda.is_available():
        raise RuntimeError("openonda_b200 initial conditions need a CUDA device (B200)")
    dev = torch.device(device) if device is not None else torch.device("cuda")
    if dev.type != "cuda":
        raise ValueError(f"device must be a CUDA device, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def to_device(arr, dev, shape_tail, name):
    if isinstance(arr, torch.Tensor):
        t = arr.to(device=dev, dtype=_F64)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(arr, dtype=np.float64))).to(dev)
    if tuple(t.shape[1:]) != shape_tail or (not shape_tail and t.dim() != 1):
        raise ValueError(f"{name} has shape {tuple(t.shape)}")
    return t.contiguous()


def stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream
