"""Multi-rank host logic of the target-sharded sweep, on CPU with gloo (world size 2 and 3).

Each rank holds one shard of the particles (shard_range), all-gathers the shards with
gather_shards (padding + compaction for uneven sizes), computes its own targets against all
gathered sources with the oracle, and the concatenation over ranks must equal the oracle's
full sweep bit for bit."""
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from openonda_b200.distributed import (balanced_ranges, gather_shards, pair_shard_ranges,
                                       reduce_scatter_rows, shard_range)


def test_shard_range_partitions():
    for n in [0, 1, 7, 8, 1000, 1 << 20]:
        for world in [1, 2, 3, 8]:
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
            assert sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _worker(rank, world, n, init_file, out_dir):
    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank,
                            world_size=world)
    try:
        import oracle
        from openonda_b200 import configs

        f = configs.random_cloud(n, seed=123)
        f.radii *= 6
        a, b = shard_range(n, rank, world)
        # this rank only owns its shard of the state
        local = torch.from_numpy(np.concatenate(
            [f.positions[a:b], f.strengths[a:b], f.radii[a:b, None]], axis=1))
        full = gather_shards(local, n).numpy()
        x, s_, r_ = full[:, 0:3], full[:, 3:6], full[:, 6]
        u = oracle.gpu.selfinduced_velocity_range(x, s_, r_, a, b)
        g = oracle.gpu.strength_gradients_range(x, s_, r_, a, b)
        np.save(os.path.join(out_dir, f"u{rank}.npy"), u)
        np.save(os.path.join(out_dir, f"g{rank}.npy"), g)
        np.save(os.path.join(out_dir, f"full{rank}.npy"), full)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 1000), (3, 1001), (2, 7)])
def test_gloo_sharded_sweep_matches_full(world, n):
    import oracle
    from openonda_b200 import configs

    with tempfile.TemporaryDirectory() as td:
        init_file = os.path.join(td, "init")
        mp.start_processes(_worker, args=(world, n, init_file, td), nprocs=world, join=True,
                           start_method="spawn")
        f = configs.random_cloud(n, seed=123)
        f.radii *= 6
        ref = np.concatenate([f.positions, f.strengths, f.radii[:, None]], axis=1)
        for r in range(world):
            assert np.array_equal(np.load(os.path.join(td, f"full{r}.npy")), ref)
        u = np.concatenate([np.load(os.path.join(td, f"u{r}.npy")) for r in range(world)])
        g = np.concatenate([np.load(os.path.join(td, f"g{r}.npy")) for r in range(world)])
        assert np.array_equal(u, oracle.gpu.get_selfinduced_velocity(f.positions, f.strengths,
                                                                     f.radii))
        assert np.array_equal(g, oracle.gpu.get_strength_gradients(f.positions, f.strengths,
                                                                   f.radii))


def test_pair_shard_ranges_partition_and_balance():
    """Pair shards: the diagonal tiles and the diagonal pairs of the both-sides schedule are
    each split into contiguous, disjoint ranges that cover them, and the CTA counts of the
    pair ranges differ by at most one diagonal's."""
    for nt in [2, 3, 10, 11, 64, 171, 1366]:
        npairs = nt // 2
        weights = [nt // 2 if 2 * (p + 1) == nt else nt for p in range(npairs)]
        for world in [1, 2, 3, 8]:
            spans = [pair_shard_ranges(nt, npairs, r, world) for r in range(world)]
            for lo, hi, total in ((0, 1, nt), (2, 3, npairs)):
                assert spans[0][lo] == 0 and spans[-1][hi] == total
                for a, b in zip(spans, spans[1:]):
                    assert a[hi] == b[lo] and a[lo] <= a[hi]
            loads = [sum(weights[s[2]:s[3]]) for s in spans]
            assert sum(loads) == sum(weights)
            assert max(loads) - min(loads) <= max(weights, default=0), (nt, world, loads)
    assert balanced_ranges([], 3) == [(0, 0)] * 3


def _rs_worker(rank, world, n, init_file, out_dir):
    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank,
                            world_size=world)
    try:
        rows = torch.arange(n * 9, dtype=torch.float64).reshape(n, 9) * (rank + 1) + rank
        mine = reduce_scatter_rows(rows, n)
        np.save(os.path.join(out_dir, f"rs{rank}.npy"), mine.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 1000), (3, 1001), (2, 7), (3, 2)])
def test_gloo_reduce_scatter_rows(world, n):
    """The row reduce-scatter of pair shards: rank r receives the sum over ranks of its
    shard_range rows (uneven shards padded for the collective)."""
    with tempfile.TemporaryDirectory() as td:
        init_file = os.path.join(td, "init")
        mp.start_processes(_rs_worker, args=(world, n, init_file, td), nprocs=world,
                           join=True, start_method="spawn")
        base = np.arange(n * 9, dtype=np.float64).reshape(n, 9)
        total = sum(base * (r + 1) + r for r in range(world))
        for r in range(world):
            a, b = shard_range(n, r, world)
            got = np.load(os.path.join(td, f"rs{r}.npy"))
            assert got.shape == (b - a, 9)
            assert np.array_equal(got, total[a:b])

