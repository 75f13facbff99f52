#!/usr/bin/env python
"""Benchmark of the VPM all-pairs hot path on B200.

Metric: Biot-Savart Gpairs/s at N = 1M -- one fused self-induced velocity + velocity
gradient (vortex stretching) evaluation of N = 2^20 particles in the FP32-compensated
form, with the FP64 form and its relative error reported beside it.

Workload: seeded random cloud (positions U[-1,1]^3, strengths N(0, 1e-3) per component,
cores U(0.02, 0.05)), the throughput-sweep configuration at N = 2^20.  A step = one
evaluation; pairs per step = N^2.  With --gpus P the targets are sharded over P ranks and
the packed source records are all-gathered (NCCL) inside every step; `value` is the
whole-job rate N^2 / (max over ranks of the step time).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Biot-Savart Gpairs/s at N=1M: FP32-compensated vs FP64 at <=1e-6 rel err"
UNIT = "Gpairs/s"
# FP32-pipe work per ordered pair of the fused velocity + stretching sweep, counted from the
# pair operators (OpVelStretch in csrc/vpm_pairs.cuh, OpVelStretchBoth in csrc/vpm_rot.cuh).
# One-sided: 38 FP32 lane-ops = 19 FFMA + 12 FMUL + 7 FADD -> 57 flops (FMA = 2), 1 MUFU.RSQ.
# Both-sides (each unordered pair once for both particles): 53 lane-ops = 31 FFMA + 15 FMUL
# + 7 FADD -> 84 flops and 1 MUFU per unordered pair, i.e. 26.5 lane-ops, 42 flops and 0.5
# MUFU per ordered pair.
FLOPS_PER_PAIR_FUSED = 57
FP32_OPS_PER_PAIR_FUSED = 38
FLOPS_PER_PAIR_BOTH = 42
FP32_OPS_PER_PAIR_BOTH = 26.5
# Algorithmic work of one ordered pair of the fused sum, whatever the schedule: the pair math
# of ParticlesPhysicsCuda.py:133-191 and :375-445 with the target terms hoisted is 43 FP32-pipe
# ops, 21 of them FMA -> 64 flops (FMA = 2), and one rsqrt.  roofline.achieved counts these;
# the both-sides schedule executes 42 flops per ordered pair (each unordered pair once for
# both particles), reported beside it.
ALGO_FLOPS_PER_PAIR = 64
L2_FLUSH_BYTES = 512 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp32c_refined"])
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=0)
    return ap.parse_args()


def workload(n, seed):
    from openonda_b200 import configs

    return configs.random_cloud(n, seed=seed)


def workload_name(n, seed):
    return (f"random cloud N={n} (x~U[-1,1]^3, alpha~N(0,1e-3), sigma~U(0.02,0.05), "
            f"seed={seed}); one fused velocity + stretching evaluation")


# ----------------------------------------------------------------------------------------
# CPU baseline (the oracle's port of the reference's CPU module, all host threads)
# ----------------------------------------------------------------------------------------
def cpu_port_rate(field, seconds):
    """Gpairs/s of velocity + stretching (CPU semantics) on a target subset x all sources."""
    import oracle

    x, a, s = field.positions, field.strengths, field.radii
    n = len(x)
    mod = oracle.cpu_fast
    m = 16
    t0 = time.perf_counter()
    mod.selfinduced_velocity_range(x, a, s, 0, m)
    mod.strength_gradients_range(x, a, s, 0, m)
    dt = time.perf_counter() - t0
    rate = m * n / max(dt, 1e-9)
    m = int(max(16, min(n, rate * seconds / n)))
    t0 = time.perf_counter()
    mod.selfinduced_velocity_range(x, a, s, 0, m)
    mod.strength_gradients_range(x, a, s, 0, m)
    dt = time.perf_counter() - t0
    return m * n / dt / 1e9, m, dt, oracle.num_threads()


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    """Reference arm: the reference's CPU path (oracle port, FP64, fast-math, all threads)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle

    f = workload(args.n, args.seed)
    x, a, s = f.positions, f.strengths, f.radii
    n = len(x)
    mod = oracle.cpu_fast
    # size one step to ~6 s of CPU work so the whole run ends within a few minutes
    m = 16
    t0 = time.perf_counter()
    mod.selfinduced_velocity_range(x, a, s, 0, m)
    mod.strength_gradients_range(x, a, s, 0, m)
    rate = m * n / max(time.perf_counter() - t0, 1e-9)
    m = int(max(16, min(n, rate * 6.0 / n)))
    times = []
    for k in range(args.warmup + args.steps):
        off = (k * m) % max(1, n - m)
        t0 = time.perf_counter()
        mod.selfinduced_velocity_range(x, a, s, off, off + m)
        mod.strength_gradients_range(x, a, s, off, off + m)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    value = m * n / t / 1e9
    sample = (f"{m} targets x {n} sources per step (velocity + stretching, CPU semantics of "
              f"ParticlesPhysics.py), {oracle.num_threads()} threads, {cpu_model()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(args.n, args.seed), "n": args.n,
                   "sample": sample},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": oracle.num_threads(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------------------
# clocks sampler
# ----------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------------------
# B200 arm
# ----------------------------------------------------------------------------------------
def measure_fp32_peak(torch, kernels, dev, kind=0, iters=1 << 15):
    """Throughput of one pipe by microbenchmark: kind 0 = FP32 FFMA, 3 = packed FFMA2 (both
    in TFLOP/s, a lane FMA = 2 flops), kind 2 = MUFU rsqrt (T rsqrt/s)."""
    props = torch.cuda.get_device_properties(dev)
    blocks, threads = props.multi_processor_count * 8, 256
    sink = torch.empty(blocks * threads, dtype=torch.float32, device=dev)
    kernels.launch_fma_peak(kind, blocks, threads, 64, sink)
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        kernels.launch_fma_peak(kind, blocks, threads, iters, sink)
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        best = t if best is None else min(best, t)
    ops = blocks * threads * iters * 16
    return {0: 2.0, 2: 1.0, 3: 4.0}[kind] * ops / best / 1e12


def reference_gpu(torch, kernels, dev, x_h, a_h, s_h, n):
    """The reference's Numba-CUDA velocity and stretching kernels on this GPU (FP64, one thread
    per target, 512 threads per block), N = n: kernel time by CUDA events around the two
    launches, and end to end through its module functions (per-call H2D, launch, D2H), in
    Gpairs/s counting N^2 pairs for the pair of sweeps, as the headline counts one fused
    evaluation.  Returns {"unavailable": why} when the reference or Numba's CUDA target is
    missing."""
    try:
        sys.path.insert(0, os.path.join(HERE, "baseline"))
        from install_ref import load_reference_module

        import numba
        from numba import cuda

        mod = load_reference_module("ParticlesPhysicsCuda")
        x, a, s = (np.ascontiguousarray(z[:n]) for z in (x_h, a_h, s_h))
        xd, ad, sd = cuda.to_device(x), cuda.to_device(a), cuda.to_device(s)
        ud, gd = cuda.device_array_like(x), cuda.device_array_like(x)
        tpb = mod.threads_per_block
        blocks = (n + tpb - 1) // tpb

        def launch():
            mod.get_selfinduced_velocity_kernel[blocks, tpb](xd, ad, sd, ud)
            mod.get_strength_gradients_kernel[blocks, tpb](xd, ad, sd, gd)

        launch()
        cuda.synchronize()
        e0, e1 = cuda.event(), cuda.event()
        e0.record()
        launch()
        e1.record()
        e1.synchronize()
        t_kernel = cuda.event_elapsed_time(e0, e1) / 1e3
        t0 = time.perf_counter()
        u_ref = mod.get_selfinduced_velocity(x, a, s)
        g_ref = mod.get_strength_gradients(x, a, s)
        t_e2e = time.perf_counter() - t0
    except Exception as e:  # noqa: BLE001 -- the bench reports why and goes on
        msg = str(e).splitlines()[0] if str(e) else ""
        return {"unavailable": f"{type(e).__name__}: {msg}"}
    xt, at, st = (torch.from_numpy(z).to(dev) for z in (x, a, s))
    u, g = kernels.velocity_and_strength_gradients(xt, at, st, precision="fp64")
    return {"n": n, "numba": numba.__version__,
            "kernel_gpairs_s": round(float(n) * n / t_kernel / 1e9, 3),
            "e2e_gpairs_s": round(float(n) * n / t_e2e / 1e9, 3),
            "rel_diff_fp64_vs_reference": {"velocity": normwise(u.cpu(), torch.from_numpy(u_ref)),
                                           "stretching": normwise(g.cpu(),
                                                                  torch.from_numpy(g_ref))},
            "kernels": "get_selfinduced_velocity_kernel + get_strength_gradients_kernel "
                       "(ParticlesPhysicsCuda.py:133-191, :375-445), Numba-CUDA, FP64"}


def reference_cpu(x_h, a_h, s_h, n, seconds=4.0):
    """The reference's own CPU module (ParticlesPhysics.py, Numba njit with prange, unmodified,
    from baseline/_ref) on all host threads, FP64: velocity through get_induced_velocity_at on
    a bounded number of target rows against all n sources (exact per-pair work), and the
    stretching sweep, which has no target-subset entry point, on the first 16384 particles.
    The fused-equivalent rate (one velocity and one stretching evaluation per pair, as the
    headline counts one fused evaluation) is 1 / (1 / velocity rate + 1 / stretching rate).
    Returns {"unavailable": why} when the reference or Numba is missing."""
    try:
        sys.path.insert(0, os.path.join(HERE, "baseline"))
        from install_ref import load_reference_module

        import numba

        mod = load_reference_module("ParticlesPhysics")
        x, a, s = (np.ascontiguousarray(z[:n]) for z in (x_h, a_h, s_h))
        t0 = time.perf_counter()
        mod.get_induced_velocity_at(x[:64], x[:64], a[:64], s[:64])  # JIT
        mod.get_strength_gradients(x[:64], a[:64], s[:64])
        jit_s = time.perf_counter() - t0
        m = 64
        t0 = time.perf_counter()
        mod.get_induced_velocity_at(x[:m], x, a, s)
        rate = m * n / (time.perf_counter() - t0)
        m = int(min(n, max(64, rate * seconds / n)))
        t0 = time.perf_counter()
        mod.get_induced_velocity_at(x[:m], x, a, s)
        t_vel = time.perf_counter() - t0
        ns = min(n, 16384)
        t0 = time.perf_counter()
        mod.get_strength_gradients(x[:ns], a[:ns], s[:ns])
        t_str = time.perf_counter() - t0
    except Exception as e:  # noqa: BLE001 -- the bench reports why and goes on
        msg = str(e).splitlines()[0] if str(e) else ""
        return {"unavailable": f"{type(e).__name__}: {msg}"}
    r_vel = m * float(n) / t_vel / 1e9
    r_str = float(ns) * ns / t_str / 1e9
    return {"module": "ParticlesPhysics.py (Numba CPU, FP64)", "numba": numba.__version__,
            "threads": numba.get_num_threads(), "jit_s": round(jit_s, 1),
            "velocity_gpairs_s": round(r_vel, 4),
            "velocity_sample": f"{m} targets x {n} sources, {t_vel:.1f} s",
            "stretching_gpairs_s": round(r_str, 4),
            "stretching_sample": f"{ns} x {ns}, {t_str:.1f} s",
            "fused_equivalent_gpairs_s": round(1.0 / (1.0 / r_vel + 1.0 / r_str), 4)}


def load_traffic():
    path = os.path.join(HERE, "profiles", "ncu_traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return None


def normwise(got, ref):
    d = (got - ref).abs().max()
    r = ref.abs().max()
    return float(d / r) if float(r) > 0 else float(d)


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    from openonda_b200 import kernels
    from openonda_b200.distributed import ShardedVelocityStretching, shard_range
    from openonda_b200.vpm import ParticlesPhysicsB200 as pp

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    f = workload(args.n, args.seed)
    n = f.n
    start, stop = shard_range(n, rank, world)
    # Inputs rounded to FP32 once, so that the FP64 run sees exactly the FP32 inputs.
    x_h = f.positions.astype(np.float32).astype(np.float64)
    a_h = f.strengths.astype(np.float32).astype(np.float64)
    s_h = f.radii.astype(np.float32).astype(np.float64)
    xs = torch.from_numpy(x_h[start:stop]).to(dev)
    as_ = torch.from_numpy(a_h[start:stop]).to(dev)
    ss = torch.from_numpy(s_h[start:stop]).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def timed(op, steps, warmup, sampler=None):
        for _ in range(warmup):
            op()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        evs = []
        for _ in range(steps):
            flush.fill_(1)  # L2 flush between timed steps, outside the events
            e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            e[0].record()
            out = op()
            e[1].record()
            evs.append(e)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        t = sum(e[0].elapsed_time(e[1]) for e in evs) / 1e3
        return max_over_ranks(t), out, clocks

    # ---- FP32-compensated (headline) ----
    sweep32 = ShardedVelocityStretching(n, precision=args.precision)
    sweep_events = []

    def step32():
        sweep32.pack(xs, as_, ss)
        rec = sweep32.exchange()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        e[0].record()
        out = sweep32.sweep(rec)
        e[1].record()
        sweep_events.append(e)
        return out

    peak = measure_fp32_peak(torch, kernels, dev)
    sfu_peak = measure_fp32_peak(torch, kernels, dev, kind=2, iters=1 << 13)
    ffma2_peak = measure_fp32_peak(torch, kernels, dev, kind=3, iters=1 << 14)
    sampler = ClockSampler(local_rank) if rank == 0 else None
    t32, (u32, g32), clocks = timed(step32, args.steps, args.warmup, sampler)
    sweep_events = sweep_events[-args.steps:]
    t_sweep = sum(e[0].elapsed_time(e[1]) for e in sweep_events) / 1e3 / args.steps
    t_sweep = max_over_ranks(t_sweep)
    u32, g32 = u32.clone(), g32.clone()
    ms32 = t32 / args.steps * 1e3
    value = float(n) * n / (t32 / args.steps) / 1e9

    # ---- FP64 fused and FP64 drop-in (two separate sweeps, as the reference calls them) ----
    sweep64 = ShardedVelocityStretching(n, precision="fp64")
    t64, (u64, g64), _ = timed(lambda: sweep64(xs, as_, ss), args.fp64_steps, 1)
    fp64_fused = float(n) * n / (t64 / args.fp64_steps) / 1e9
    err_u = max_over_ranks(normwise(u32, u64))
    err_g = max_over_ranks(normwise(g32, g64))
    fp64_dropin = fp64_one_sided = fp64_dropin_shipped = None
    if world == 1:
        xa = torch.from_numpy(x_h).to(dev)
        aa = torch.from_numpy(a_h).to(dev)
        sa = torch.from_numpy(s_h).to(dev)

        def dropin():
            return (kernels.selfinduced_velocity(xa, aa, sa, precision="fp64"),
                    kernels.strength_gradients(xa, aa, sa, precision="fp64"))

        # the drop-in as shipped (its velocity sweep takes the both-sides schedule here)
        tdi, _, _ = timed(dropin, 1, 1)
        fp64_dropin_shipped = float(n) * n / tdi / 1e9
        # the plain FP64 kernels, one-sided (each ordered pair evaluated for its target only)
        # as the reference's kernels evaluate them: the fused sum, and the two separate
        # sweeps the reference calls
        prev = kernels.set_symmetric_min_n(1 << 40)
        try:
            tos, _, _ = timed(lambda: kernels.velocity_and_strength_gradients(
                xa, aa, sa, precision="fp64"), 1, 1)
            tdp, _, _ = timed(dropin, 1, 1)
        finally:
            kernels.set_symmetric_min_n(prev)
        fp64_one_sided = float(n) * n / tos / 1e9
        fp64_dropin = float(n) * n / tdp / 1e9
        del xa, aa, sa

    # ---- the reference's own Numba-CUDA kernels (ParticlesPhysicsCuda.py, unmodified, from
    # baseline/_ref) on this GPU: velocity + stretching, as the reference calls them ----
    ref_gpu = None
    if world == 1:
        ref_gpu = reference_gpu(torch, kernels, dev, x_h, a_h, s_h, min(n, 131072))
    ref_cpu = None
    if world == 1 and not args.no_cpu_baseline:
        ref_cpu = reference_cpu(x_h, a_h, s_h, n)
    # ---- adjoint: one VJP sweep of the right-hand side (u, S [+ P]) against one forward
    # evaluation of it, N = 65536 random cloud, cotangents N(0,1) ----
    adjoint = None
    if world == 1:
        from openonda_b200 import autodiff

        na = min(n, 65536)
        xa = torch.from_numpy(x_h[:na]).to(dev)
        aa = torch.from_numpy(a_h[:na]).to(dev)
        sa = torch.from_numpy(s_h[:na]).to(dev)
        nua = torch.full((na,), 1e-4, dtype=torch.float64, device=dev)
        gen = torch.Generator().manual_seed(1)
        gu = torch.randn((na, 3), generator=gen, dtype=torch.float64).to(dev)
        gr = torch.randn((na, 3), generator=gen, dtype=torch.float64).to(dev)
        adjoint = {"n": na, "steps": 3}
        grads = {}
        for prec in ("fp32c", "fp64"):
            def fwd():
                return kernels.velocity_and_strength_gradients(xa, aa, sa, precision=prec)

            def fwd_pse():
                return (fwd(), kernels.strength_gradients_pse(xa, aa, sa, nua, precision=prec))

            tf, _, _ = timed(fwd, 3, 1)
            tb, grads[prec], _ = timed(
                lambda: autodiff.rhs_vjp(xa, aa, sa, None, gu, gr, precision=prec), 3, 1)
            tfp, _, _ = timed(fwd_pse, 3, 1)
            tbp, _, _ = timed(
                lambda: autodiff.rhs_vjp(xa, aa, sa, nua, gu, gr, precision=prec), 3, 1)
            adjoint[prec] = {"forward_ms": round(tf / 3 * 1e3, 3),
                             "vjp_ms": round(tb / 3 * 1e3, 3),
                             "vjp_over_forward": round(tb / tf, 3),
                             "forward_pse_ms": round(tfp / 3 * 1e3, 3),
                             "vjp_pse_ms": round(tbp / 3 * 1e3, 3),
                             "vjp_pse_over_forward_pse": round(tbp / tfp, 3)}
        adjoint["grad_rel_err_fp32c_vs_fp64"] = {
            k: normwise(grads["fp32c"][i], grads["fp64"][i])
            for i, k in enumerate(("positions", "strengths", "radii"))}
        del xa, aa, sa, nua, gu, gr, grads

    # ---- end to end through the public API, host buffers (pinned), copies timed ----
    xp = torch.from_numpy(x_h[start:stop]).pin_memory()
    ap_ = torch.from_numpy(a_h[start:stop]).pin_memory()
    sp = torch.from_numpy(s_h[start:stop]).pin_memory()

    def e2e_step():
        if world == 1:
            u, g = pp.get_selfinduced_velocity_and_strength_gradients(
                xp, ap_, sp, precision=args.precision)
        else:
            u, g = sweep32(xp.to(dev, non_blocking=True), ap_.to(dev, non_blocking=True),
                           sp.to(dev, non_blocking=True))
            u, g = u.cpu(), g.cpu()
        return u, g

    for _ in range(1):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    barrier()
    e2e_value = float(n) * n / (t_e2e / args.e2e_steps) / 1e9
    m_local = stop - start
    h2d = m_local * (3 + 3 + 1) * 8
    d2h = m_local * 6 * 8

    # ---- CPU baseline (rank 0, single GPU only) ----
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        rate, m, dt, cores = cpu_port_rate(f, args.cpu_seconds)
        cpu = {"value": round(rate, 4), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{m} targets x {n} sources, velocity + stretching (CPU semantics), "
                         f"{dt:.1f} s, {cpu_model()}"}

    if rank == 0:
        pairs_per_launch = float(m_local) * n
        both = sweep32.both_sides
        flops_pp = FLOPS_PER_PAIR_BOTH if both else FLOPS_PER_PAIR_FUSED
        ops_pp = FP32_OPS_PER_PAIR_BOTH if both else FP32_OPS_PER_PAIR_FUSED
        rsqrt_pp = 0.5 if both else 1.0
        executed = flops_pp * pairs_per_launch / t_sweep / 1e12
        achieved = ALGO_FLOPS_PER_PAIR * pairs_per_launch / t_sweep / 1e12
        traffic = load_traffic()
        tr = None
        if traffic and both and traffic.get("both_sides"):
            # both-sides sweep: accumulator read-modify-writes per tile pair, ~N^2
            tr = round(traffic["both_sides"]["bytes_per_pair"] * float(m_local) * n)
        elif traffic and traffic.get("kernel_traffic_bytes_per_particle") is not None:
            # one-sided sweep: DRAM traffic grows with the particle count, not with N^2
            tr = round(traffic["kernel_traffic_bytes_per_particle"] * n)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms32, 3),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 pair terms + f64 carries", "data": "synthetic",
            "config": {"workload": workload_name(n, args.seed), "n": n,
                       "precision": args.precision,
                       "parallelism": (f"pair shards x{world}, records all-gathered, "
                                       "FP64 rows reduce-scattered" if sweep32.pairs is not None
                                       else f"target shards x{world}, sources all-gathered"),
                       "l2": "flushed between timed steps (512 MiB write)"},
            "fp64": {"fused_gpairs_s": round(fp64_fused, 3),
                     "fused_path": "both-sides" if sweep64.both_sides else "one-sided",
                     "one_sided_gpairs_s":
                         None if fp64_one_sided is None else round(fp64_one_sided, 3),
                     "speedup_vs_fp64_one_sided":
                         None if fp64_one_sided is None else round(value / fp64_one_sided, 3),
                     "dropin_two_sweeps_gpairs_s":
                         None if fp64_dropin is None else round(fp64_dropin, 3),
                     "speedup_vs_fp64_fused": round(value / fp64_fused, 3),
                     "speedup_vs_fp64_dropin":
                         None if fp64_dropin is None else round(value / fp64_dropin, 3),
                     "dropin_shipped_gpairs_s":
                         None if fp64_dropin_shipped is None
                         else round(fp64_dropin_shipped, 3),
                     "speedup_vs_fp64_dropin_shipped":
                         None if fp64_dropin_shipped is None
                         else round(value / fp64_dropin_shipped, 3)},
            "rel_err_vs_fp64": {"velocity": err_u, "stretching": err_g},
            "reference_gpu": ref_gpu,
            "reference_cpu": ref_cpu,
            "speedup_vs_reference_cpu":
                None if not ref_cpu or "fused_equivalent_gpairs_s" not in ref_cpu
                else round(e2e_value / ref_cpu["fused_equivalent_gpairs_s"], 1),
            "speedup_vs_reference_gpu":
                None if not ref_gpu or "kernel_gpairs_s" not in ref_gpu
                else {"kernel": round(value / ref_gpu["kernel_gpairs_s"], 1),
                      "e2e": round(e2e_value / ref_gpu["e2e_gpairs_s"], 1)},
            "adjoint": adjoint,
            "roofline": {"bound": "fp32", "achieved": round(achieved, 3),
                         "peak": round(peak, 3), "unit": "TFLOP/s",
                         "frac": round(achieved / peak, 4), "traffic": tr,
                         "peak_source": "FFMA microbenchmark measured in this run",
                         "kernel": ("both-sides sweep, " if both else "one-sided sweep, ")
                                   + f"{sweep32.sweep_launches} launches per call",
                         "flops_per_pair": ALGO_FLOPS_PER_PAIR,
                         "executed_flops_per_pair": flops_pp,
                         "executed": round(executed, 3),
                         "executed_frac": round(executed / peak, 4),
                         "fp32_pipe_frac": round(executed / peak * 2 * ops_pp / flops_pp, 4),
                         "packed_ffma2_peak": round(ffma2_peak, 3),
                         # FP32 lane-ops (x2, the FMA flop convention) against the packed-FFMA2
                         # microbenchmark: the ceiling of this instruction mix
                         "fp32_pipe_frac_of_packed_peak": round(
                             executed / ffma2_peak * 2 * ops_pp / flops_pp, 4),
                         "sfu": {"rsqrt_per_pair": rsqrt_pp,
                                 "achieved_t_per_s": round(
                                     rsqrt_pp * pairs_per_launch / t_sweep / 1e12, 4),
                                 "peak_t_per_s": round(sfu_peak, 4),
                                 "frac": round(rsqrt_pp * pairs_per_launch / t_sweep / 1e12
                                               / sfu_peak, 4),
                                 "peak_source": "MUFU rsqrt microbenchmark in this run"}},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "cpu_baseline": cpu,
            "gpu_launches": args.steps * sweep32.kernel_launches_per_call,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
