"""Pair shards of the fused velocity + stretching sum (the multi-GPU form of the both-sides
schedule, openonda_b200/distributed.py), emulated on one GPU.

Each rank's share -- vpm_sweep_pairs_partial over its diagonal-tile and diagonal-pair
ranges, on all n records -- runs in turn on the same GPU; the rows are summed over the ranks
in rank order (what the reduce-scatter between GPUs sums), and every rank's targets are
finalized from their summed rows with vpm_finalize_pairs_partial.  The result must equal the
single-GPU both-sides sweep up to the order of the FP64 additions, and hold the FP32c bars
against the FP64 sweep (FP64 pair shards: 1e-12).  No collective and no wait between ranks
runs on the GPU: the ranks' kernels are independent launches, one after the other."""
import numpy as np
import pytest
import torch

from conftest import normwise

pytestmark = pytest.mark.gpu


def _records(x, a, s, code):
    from openonda_b200 import _lib

    lib = _lib.load()
    n = x.shape[0]
    rec = torch.empty((n, int(lib.vpm_record_bytes(code)) // 4), dtype=torch.float32,
                      device=x.device)
    _lib.check(lib.vpm_pack_records(x.data_ptr(), a.data_ptr(), s.data_ptr(), None, n, code,
                                    rec.data_ptr(), torch.cuda.current_stream().cuda_stream))
    return rec


@pytest.mark.parametrize("n,world,uniform_core,precision",
                         [(50000, 2, False, "fp32c"), (50000, 3, True, "fp32c"),
                          (32768, 4, False, "fp32c"), (131072, 8, False, "fp32c"),
                          (50000, 3, False, "fp64")])
def test_pair_shards_sum_to_the_single_gpu_sweep(n, world, uniform_core, precision):
    from openonda_b200 import _lib, configs, kernels
    from openonda_b200.distributed import (finalize_pairs_partial, pair_shard_ranges,
                                           pairs_layout, shard_range, sweep_pairs_partial)

    f = configs.random_cloud(n, seed=5)
    if uniform_core:
        f.radii[:] = f.radii[0]
    x, a, s = (torch.from_numpy(np.asarray(z, np.float32).astype(np.float64)).cuda()
               for z in (f.positions, f.strengths, f.radii))
    layout = pairs_layout(n, precision, uniform_core)
    assert layout is not None
    nt, npairs, per_launch, nv, wsb = layout
    assert nv == 9 and npairs == nt // 2 and per_launch >= 1
    rec = _records(x, a, s, _lib.precision_code(precision, uniform_core))
    ws = torch.empty(max(wsb, 256), dtype=torch.uint8, device=x.device)
    rows = torch.empty((n, nv), dtype=torch.float64, device=x.device)
    total = torch.zeros((n, nv), dtype=torch.float64, device=x.device)
    for r in range(world):
        t0, t1, p0, p1 = pair_shard_ranges(nt, npairs, r, world)
        sweep_pairs_partial(rec, n, (t0, t1), (p0, p1), rows, ws, precision, uniform_core)
        total += rows
    u = torch.empty((n, 3), dtype=torch.float64, device=x.device)
    g = torch.empty_like(u)
    for r in range(world):
        lo, hi = shard_range(n, r, world)
        finalize_pairs_partial(total[lo:hi].contiguous(), rec, lo, u[lo:hi], g[lo:hi],
                               precision, uniform_core)
    one = kernels.velocity_and_strength_gradients(x, a, s, precision=precision,
                                                  uniform_core=uniform_core)
    ref = kernels.velocity_and_strength_gradients(x, a, s, precision="fp64")
    for k, got in enumerate((u, g)):
        e_one = normwise(got.cpu().numpy(), one[k].cpu().numpy())
        e_ref = normwise(got.cpu().numpy(), ref[k].cpu().numpy())
        print(f"n={n} world={world} uc={uniform_core} {precision} k={k}: vs single GPU "
              f"{e_one:.2e}, vs FP64 {e_ref:.2e}")
        assert e_one <= 1e-11, (k, e_one)
        bar = 1e-12 if precision == "fp64" else (1e-6 if k == 0 else 2e-6)
        assert e_ref <= bar, (k, e_ref)
    assert kernels.device_errors() == 0


def test_pair_shards_need_the_both_sides_size():
    """Below the both-sides schedule's size there are no pair shards (the sharded sweep keeps
    target shards there)."""
    from openonda_b200.distributed import pairs_layout

    assert pairs_layout(1000, "fp32c") is None
    assert pairs_layout(1000, "fp64") is None
    assert pairs_layout(1 << 16, "fp32c") is not None
    assert pairs_layout(1 << 16, "fp64")[3] == 9
