"""Target-sharded sweeps across GPUs (one process per GPU, torch.distributed).

Each rank owns a contiguous shard of the particles.  One sweep is:

1. pack the rank's own shard into compute-precision records (64 B each in both precisions:
   FP64 values, or FP32 values stored twice for the paired FP32 instructions),
2. all-gather the records of every shard (NCCL over NVLink; the only exchange step of the
   all-pairs sum -- 64 MB at N = 2^20),
3. sweep the rank's own targets against all gathered sources with ``vpm_sweep_records``.

Targets are independent, so nothing else crosses GPUs; the outputs stay sharded.  The
host-side logic (shard ranges, padding and compaction of uneven shards) is backend
agnostic and is tested with ``gloo`` ranks on CPU.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from . import _lib, kernels


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's shard: sizes differ by at most one, larger shards first."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, rem = divmod(int(n), int(world))
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def gather_shards(local: torch.Tensor, n_rows: int, group=None) -> torch.Tensor:
    """All-gather row shards (shard_range layout) of a 2-D tensor into the full array.

    Shards are padded to the largest shard for the collective and compacted afterwards,
    so uneven ``n_rows`` is allowed.  Works for any backend (nccl on GPUs, gloo on CPU).
    """
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    width = local.shape[1]
    smax = shard_range(n_rows, 0, world)[1]  # shard 0 is the largest
    start, stop = shard_range(n_rows, rank, world)
    if local.shape[0] != stop - start:
        raise ValueError(f"rank {rank} holds {local.shape[0]} rows, expected {stop - start}")
    if n_rows % world == 0:
        out = torch.empty((n_rows, width), dtype=local.dtype, device=local.device)
        dist.all_gather_into_tensor(out, local.contiguous(), group=group)
        return out
    padded = torch.zeros((smax, width), dtype=local.dtype, device=local.device)
    padded[: local.shape[0]] = local
    buf = torch.empty((world * smax, width), dtype=local.dtype, device=local.device)
    dist.all_gather_into_tensor(buf, padded, group=group)
    out = torch.empty((n_rows, width), dtype=local.dtype, device=local.device)
    for r in range(world):
        a, b = shard_range(n_rows, r, world)
        out[a:b] = buf[r * smax: r * smax + (b - a)]
    return out


class ShardedVelocityStretching:
    """Fused velocity + stretching of this rank's targets against all ranks' particles."""

    def __init__(self, n_total: int, precision: str = "fp32c", group=None):
        self.n = int(n_total)
        self.precision = precision
        self.pcode = _lib.precision_code(precision)
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.start, self.stop = shard_range(self.n, self.rank, self.world)
        self.m = self.stop - self.start
        lib = _lib.load()
        self.rec_bytes = int(lib.vpm_record_bytes(self.pcode))
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        # records as float rows so the collective moves whole records
        words = self.rec_bytes // 4
        self.local = torch.empty((self.m, words), dtype=torch.float32, device=dev)
        self.ws_bytes = kernels.workspace_bytes("velocity_and_strength_gradients", precision,
                                                self.m, self.n)
        self.ws = torch.empty(max(self.ws_bytes, 256), dtype=torch.uint8, device=dev)
        self.u = torch.empty((self.m, 3), dtype=torch.float64, device=dev)
        self.g = torch.empty((self.m, 3), dtype=torch.float64, device=dev)
        # pack, then the sweep's own launches (one-sided: sweep + finalize; both-sides sweep
        # over all particles: zero, diagonal tiles, diagonal-pair launches, finalize)
        self.sweep_launches = int(lib.vpm_sweep_launches(
            _lib.OPS["velocity_and_strength_gradients"], self.pcode, self.m, self.n))
        self.both_sides = self.sweep_launches > 2
        self.kernel_launches_per_call = 1 + self.sweep_launches

    def pack(self, positions, strengths, radii):
        x = kernels._check_vec("positions", positions, self.m)
        a = kernels._check_vec("strengths", strengths, self.m)
        s = kernels._check_scalar("radii", radii, self.m)
        _lib.check(_lib.load().vpm_pack_records(
            x.data_ptr(), a.data_ptr(), s.data_ptr(), None, self.m, self.pcode,
            self.local.data_ptr(), kernels._stream(self.device)))
        return self.local

    def exchange(self):
        if self.world == 1:
            return self.local
        return gather_shards(self.local, self.n, self.group)

    def sweep(self, records):
        _lib.check(_lib.load().vpm_sweep_records(
            _lib.OPS["velocity_and_strength_gradients"], records.data_ptr(), self.n, self.start,
            self.m, 0, self.u.data_ptr(), self.g.data_ptr(), self.pcode, self.ws.data_ptr(),
            self.ws.numel(), kernels._stream(self.device)))
        return self.u, self.g

    def __call__(self, positions, strengths, radii):
        self.pack(positions, strengths, radii)
        return self.sweep(self.exchange())
