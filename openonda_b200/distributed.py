"""Sweeps across GPUs (one process per GPU, torch.distributed).

Each rank owns a contiguous shard of the particles.  One sweep is:

1. pack the rank's own shard into compute-precision records (64 B each in both precisions:
   FP64 values, or FP32 values stored twice for the paired FP32 instructions),
2. all-gather the records of every shard (NCCL over NVLink -- 64 MB at N = 2^20),
3. either (target shards) sweep the rank's own targets against all gathered sources with
   ``vpm_sweep_records``; nothing else crosses GPUs,
   or (pair shards, sizes that take the both-sides schedule) run the rank's share of
   that schedule's tiles and diagonal pairs over all particles with
   ``vpm_sweep_pairs_partial``, reduce-scatter the (n, 9) FP64 partial sums by row ranges
   (72 MB at N = 2^20) and finalize the rank's own rows with
   ``vpm_finalize_pairs_partial``.  Each unordered pair is then evaluated once for both of
   its particles, wherever they live, at the cost of the one extra exchange.

The outputs stay sharded either way.  The host-side logic (shard and schedule ranges,
padding and compaction of uneven shards, the row reduce-scatter) is backend agnostic and is
tested with ``gloo`` ranks on CPU.
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


def balanced_ranges(weights, world: int) -> list[tuple[int, int]]:
    """Split items 0..len(weights)-1 into ``world`` contiguous ranges of near-equal total
    weight: range r ends at the first item whose running total reaches (r + 1) / world of
    the whole."""
    total = float(sum(weights))
    bounds = [0]
    run = 0.0
    i = 0
    for r in range(1, world):
        goal = total * r / world
        while i < len(weights) and run + weights[i] / 2.0 <= goal:
            run += weights[i]
            i += 1
        bounds.append(i)
    bounds.append(len(weights))
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def pair_shard_ranges(n_tiles: int, n_pairs: int, rank: int, world: int):
    """(tile_begin, tile_end, pair_begin, pair_end) of rank's share of the both-sides
    schedule: the diagonal tiles by even counts, the diagonal pairs (index p = diagonal
    p + 1) by their CTA counts -- n_tiles each, except the middle diagonal of an even tile
    count, which has n_tiles / 2."""
    t0, t1 = shard_range(n_tiles, rank, world)
    w = [n_tiles // 2 if 2 * (p + 1) == n_tiles else n_tiles for p in range(n_pairs)]
    p0, p1 = balanced_ranges(w, world)[rank]
    return t0, t1, p0, p1


def reduce_scatter_rows(rows: torch.Tensor, n_rows: int, group=None) -> torch.Tensor:
    """Sum of every rank's (n_rows, width) ``rows`` over the ranks, each rank receiving its
    shard_range rows.  Uneven shards are padded to the largest shard for the collective."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    width = rows.shape[1]
    start, stop = shard_range(n_rows, rank, world)
    if n_rows % world == 0:
        out = torch.empty((stop - start, width), dtype=rows.dtype, device=rows.device)
        dist.reduce_scatter_tensor(out, rows.contiguous(), group=group)
        return out
    smax = shard_range(n_rows, 0, world)[1]
    buf = torch.zeros((world * smax, width), dtype=rows.dtype, device=rows.device)
    for r in range(world):
        a, b = shard_range(n_rows, r, world)
        buf[r * smax: r * smax + (b - a)] = rows[a:b]
    out = torch.empty((smax, width), dtype=rows.dtype, device=rows.device)
    dist.reduce_scatter_tensor(out, buf, group=group)
    return out[: stop - start]


def pairs_layout(n: int, precision: str = "fp32c", uniform_core: bool = False):
    """(tiles, diagonal pairs, diagonal pairs per launch, values per row, workspace bytes) of
    the fused sum's both-sides plan for n particles, or None where n does not take it."""
    import ctypes

    lib = _lib.load()
    nt, npairs, per, nv, wsb = (ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int(),
                                ctypes.c_int(), ctypes.c_size_t())
    rc = lib.vpm_pairs_layout(_lib.OPS["velocity_and_strength_gradients"],
                              _lib.precision_code(precision, uniform_core), int(n),
                              ctypes.byref(nt), ctypes.byref(npairs), ctypes.byref(per),
                              ctypes.byref(nv), ctypes.byref(wsb))
    if rc != 0:
        return None
    return nt.value, npairs.value, per.value, nv.value, wsb.value


def sweep_pairs_partial(records, n, tiles, pairs, rows, workspace, precision="fp32c",
                        uniform_core=False):
    """One rank's share of the fused sum's both-sides schedule over all n packed records:
    the diagonal tiles range ``tiles`` and the diagonal pairs range ``pairs``, summed into
    ``rows`` (n, values) FP64 (overwritten)."""
    _lib.check(_lib.load().vpm_sweep_pairs_partial(
        _lib.OPS["velocity_and_strength_gradients"], records.data_ptr(), int(n),
        int(tiles[0]), int(tiles[1]), int(pairs[0]), int(pairs[1]), rows.data_ptr(),
        _lib.precision_code(precision, uniform_core), workspace.data_ptr(), workspace.numel(),
        kernels._stream(rows.device)))
    return rows


def finalize_pairs_partial(rows, records, start, u, g, precision="fp32c",
                           uniform_core=False):
    """Velocities and stretching of targets records[start, start + len(rows)) from their
    summed rows."""
    _lib.check(_lib.load().vpm_finalize_pairs_partial(
        _lib.OPS["velocity_and_strength_gradients"], rows.data_ptr(), records.data_ptr(),
        int(start), rows.shape[0], u.data_ptr(), g.data_ptr(),
        _lib.precision_code(precision, uniform_core), kernels._stream(rows.device)))
    return u, g


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
        self.u = torch.empty((self.m, 3), dtype=torch.float64, device=dev)
        self.g = torch.empty((self.m, 3), dtype=torch.float64, device=dev)
        # pair shards: several ranks and a size that takes the both-sides schedule
        self.pairs = self._pair_plan(lib) if self.world > 1 else None
        if self.pairs is not None:
            nt, npairs, per_launch, nv, wsb, (t0, t1, p0, p1) = self.pairs
            self.both_sides = True
            self.ws_bytes = wsb
            self.rows = torch.empty((self.n, nv), dtype=torch.float64, device=dev)
            launches = -(-(p1 - p0) // per_launch)
            # zero, diagonal tiles, diagonal-pair launches, rows, finalize (+ pack)
            self.sweep_launches = 1 + (1 if t1 > t0 else 0) + launches + 2
        else:
            self.ws_bytes = kernels.workspace_bytes("velocity_and_strength_gradients",
                                                    precision, self.m, self.n)
            # the sweep's own launches (one-sided: sweep + finalize; both-sides sweep over all
            # particles: zero, diagonal tiles, diagonal-pair launches, finalize)
            self.sweep_launches = int(lib.vpm_sweep_launches(
                _lib.OPS["velocity_and_strength_gradients"], self.pcode, self.m, self.n))
            self.both_sides = self.sweep_launches > 2
        self.ws = torch.empty(max(self.ws_bytes, 256), dtype=torch.uint8, device=dev)
        self.kernel_launches_per_call = 1 + self.sweep_launches  # + the pack

    def _pair_plan(self, lib):
        layout = pairs_layout(self.n, self.precision)
        if layout is None:
            return None  # below the both-sides size: target shards
        nt, npairs = layout[0], layout[1]
        return (*layout, pair_shard_ranges(nt, npairs, self.rank, self.world))

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
        if self.pairs is not None:
            return self._sweep_pairs(records)
        _lib.check(_lib.load().vpm_sweep_records(
            _lib.OPS["velocity_and_strength_gradients"], records.data_ptr(), self.n, self.start,
            self.m, 0, self.u.data_ptr(), self.g.data_ptr(), self.pcode, self.ws.data_ptr(),
            self.ws.numel(), kernels._stream(self.device)))
        return self.u, self.g

    def _sweep_pairs(self, records):
        t0, t1, p0, p1 = self.pairs[5]
        sweep_pairs_partial(records, self.n, (t0, t1), (p0, p1), self.rows, self.ws,
                            self.precision)
        mine = reduce_scatter_rows(self.rows, self.n, self.group)
        return finalize_pairs_partial(mine, records, self.start, self.u, self.g,
                                      self.precision)

    def __call__(self, positions, strengths, radii):
        self.pack(positions, strengths, radii)
        return self.sweep(self.exchange())
