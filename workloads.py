"""The five benchmark workloads, run through the public API; one JSON line per result.

    python workloads.py {config1,config2,config3,config4,config5,stepkernels} [opts]

config1  ring N=8192 (64 x 128 torus lattice), FP64, one DNS+PSE RK4 step at dt=0.01,
         compared with the CPU oracle's restatement of the reference step.
config2  leapfrogging rings N=131072, FP32-compensated DNS+PSE, RK4 dt=0.005, nu=1e-4;
         velocity/stretching error vs FP64 at steps 1, 50, 200; FP64 circulation and
         linear-impulse drift.
config3  random-cloud throughput sweep N = 2^14 .. 2^21: fused velocity + stretching,
         FP32c vs FP64 Gpairs/s and error.
config4  differentiation: perturbed ring N=65536, FP32c, loss = FP64-summed kinetic energy
         after 50 RK4 steps at dt=0.01, checkpoint every 10 steps; gradients w.r.t. initial
         positions, strengths and cores vs the FP64 adjoint and vs FP64 central differences
         (h=1e-6) on 64 random coordinates.
config5  dynamic-LES ring N=2^20, FP32c, PSE, RK4 dt=0.002: time per step, Gpairs/s, error vs
         FP64 at the last step.
stepkernels  GB/s of the element-wise step kernels (RK stage, RK4 combine, BDF) at N=2^22.
reference    the reference's own Numba-CUDA kernels (GPU) and Numba CPU module (host cores),
             from baseline/_ref, on the random cloud (default N=131072).
sweeps       time of each FP32c sweep of an LES step (fused LES sums vs the sweeps they replace).
peaks        FP32 FFMA / FFMA2 / mixed / MUFU rsqrt throughput microbenchmarks.

All inputs are the seeded synthetic fields of :mod:`openonda_b200.configs`.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import tempfile
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

from openonda_b200 import configs, kernels  # noqa: E402


def _emit(d):
    print(json.dumps(d), flush=True)


def _rel(a, b):
    a = a if isinstance(a, torch.Tensor) else torch.as_tensor(a)
    b = b if isinstance(b, torch.Tensor) else torch.as_tensor(b)
    return float((a - b).abs().max() / b.abs().max())


class _Timer:
    def __init__(self):
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)

    def __enter__(self):
        torch.cuda.synchronize()
        self.e0.record()
        return self

    def __exit__(self, *exc):
        self.e1.record()
        self.e1.synchronize()
        self.ms = self.e0.elapsed_time(self.e1)


def _system(field, precision, **kw):
    from openonda_b200.vpm.vpmModule import ParticleSystem

    # the reference backs up at time step 0 (0 % frequency == 0): keep that file out of cwd
    ps = ParticleSystem(monitor_variables=[], backup_frequency=10 ** 9, precision=precision,
                        backup_filename=os.path.join(tempfile.gettempdir(), "vpm_workload"),
                        **kw)
    ps.add_particle_field(field.positions, np.zeros_like(field.positions), field.strengths,
                          field.radii, field.viscosities)
    return ps


def _step(ps):
    ps.update_velocities()
    ps.update_strengths()
    ps.update_state()


def config1(args):
    import oracle
    from oracle.vpm_step import StepOracle

    f = configs.ring_8192()
    kw = dict(flow_model="DNS", viscous_scheme="PSE", time_integration_method="RK4",
              time_step_size=0.01)
    warm = _system(f, "fp64", **kw)
    _step(warm)
    ps = _system(f, "fp64", **kw)
    with _Timer() as t:
        _step(ps)
    t0 = time.perf_counter()
    so = StepOracle(oracle.gpu, f.positions, f.strengths, f.radii, f.viscosities, **kw)
    so.step()
    t_cpu = time.perf_counter() - t0
    # steady state (time step >= 3): the eager loop against advance() with the CUDA graph
    steady = {}
    for mode in ("eager", "graph"):
        sp = _system(f, "fp64", **kw)
        sp.advance(4, use_graph=(mode == "graph"))  # BDF start-up (+ capture)
        k = args.steps or 50
        with _Timer() as tt:
            sp.advance(k, use_graph=(mode == "graph"))
        steady[mode] = round(tt.ms / k, 3)
    n = f.n
    _emit({"config": "config1", "workload": f.description, "n": n,
           "b200_ms_per_step": round(t.ms, 3), "sweeps_per_step": 5,
           "steady_ms_per_step_eager": steady["eager"],
           "steady_ms_per_step_cuda_graph": steady["graph"],
           "oracle_cpu_s_per_step": round(t_cpu, 2), "oracle_threads": oracle.num_threads(),
           "rel_err_positions": _rel(torch.from_numpy(ps.get_particle_positions()),
                                     torch.from_numpy(so.x)),
           "rel_err_strengths": _rel(torch.from_numpy(ps.get_particle_strengths()),
                                     torch.from_numpy(so.a)),
           "rel_err_velocities": _rel(torch.from_numpy(ps.get_particle_velocities()),
                                      torch.from_numpy(so.u))})


def _errors_vs_fp64(ps):
    x, a, s = ps.positions, ps.strengths, ps.radii
    x32 = x.float().double()
    a32 = a.float().double()
    s32 = s.float().double()
    u64, g64 = kernels.velocity_and_strength_gradients(x32, a32, s32, precision="fp64")
    u32, g32 = kernels.velocity_and_strength_gradients(x32, a32, s32, precision="fp32c")
    return _rel(u32, u64), _rel(g32, g64)


def config2(args):
    f = configs.leapfrog_rings()
    ps = _system(f, "fp32c", flow_model="DNS", viscous_scheme="PSE",
                 time_integration_method="RK4", time_step_size=0.005)
    d0 = ps._diagnostics()
    steps = args.steps or 200
    report = {1, 50, steps}
    rows = []
    t_total = 0.0
    for k in range(1, steps + 1):
        with _Timer() as t:
            _step(ps)
        t_total += t.ms
        if k in report:
            eu, eg = _errors_vs_fp64(ps)
            d = ps._diagnostics()
            imp0 = np.linalg.norm(d0[4:7])
            rows.append({"step": k, "rel_err_velocity": eu, "rel_err_stretching": eg,
                         "circulation_drift": float((d[0] - d0[0]) / d0[0]),
                         "linear_impulse_drift": float(np.linalg.norm(d[4:7] - d0[4:7]) / imp0)})
    n = f.n
    pairs = 5.0 * n * n  # fused + PSE + 3 RK stages
    _emit({"config": "config2", "workload": f.description, "n": n, "steps": steps,
           "precision": "fp32c", "ms_per_step": round(t_total / steps, 3),
           "gpairs_per_s": round(pairs / (t_total / steps / 1e3) / 1e9, 1), "checkpoints": rows})


def _pipe_peaks():
    """In-run microbenchmark peaks (lane-ops/s): scalar FFMA, packed FFMA2, MUFU rsqrt, FP64
    DFMA; 8 blocks of 256 threads per SM, best of 5."""
    dev = torch.device("cuda")
    props = torch.cuda.get_device_properties(dev)
    out = {}
    for kind, name, lanes, dt in ((0, "ffma", 16, torch.float32), (3, "ffma2", 32, torch.float32),
                                  (2, "mufu", 16, torch.float32), (1, "dfma", 16, torch.float64)):
        blocks, threads, iters = props.multi_processor_count * 8, 256, 1 << 13
        sink = torch.empty(blocks * threads, dtype=dt, device=dev)
        kernels.launch_fma_peak(kind, blocks, threads, 64, sink)
        best = float("inf")
        for _ in range(5):
            with _Timer() as t:
                kernels.launch_fma_peak(kind, blocks, threads, iters, sink)
            best = min(best, t.ms / 1e3)
        out[name] = blocks * threads * iters * lanes / best
    return out


# FP32 lane-ops and MUFU rsqrt per ordered pair of the fused velocity + stretching sum
# (general cores): one-sided OpVelStretch 38 / 1, both-sides OpVelStretchBoth 26.5 / 0.5;
# FP64 one-sided: 38 FP64 ops (DFMA pipe) and one rsqrt() per pair.
_FUSED_OPS = {"one-sided": (38.0, 1.0), "both-sides": (26.5, 0.5)}


def config3(args):
    sizes = args.sizes or [1 << k for k in range(14, 22)]
    peaks = _pipe_peaks()
    _emit({"config": "config3", "peaks_lane_ops_per_s": {k: round(v / 1e12, 3) for k, v in
                                                          peaks.items()}})
    for n in sizes:
        f = configs.random_cloud(n, seed=0)
        r = lambda z: torch.from_numpy(np.asarray(z, np.float32).astype(np.float64)).cuda()
        x, a, s = r(f.positions), r(f.strengths), r(f.radii)
        out = {}
        res = {}
        for prec in ("fp32c", "fp64"):
            # plan set-up, and at least ~100 ms of work so the clocks leave any idle state
            t_end = time.perf_counter() + 0.1
            while True:
                kernels.velocity_and_strength_gradients(x, a, s, precision=prec)
                torch.cuda.synchronize()
                if time.perf_counter() > t_end:
                    break
            reps = (20 if n <= (1 << 16) else 5) if (prec == "fp32c" or n <= (1 << 18)) else 1
            best = float("inf")
            for _ in range(3 if reps > 1 else 1):  # best of three timing windows
                with _Timer() as t:
                    for _ in range(reps):
                        out[prec] = kernels.velocity_and_strength_gradients(x, a, s,
                                                                            precision=prec)
                best = min(best, t.ms / reps)
            res[prec] = n * n / (best / 1e3) / 1e9
        path = ("both-sides" if kernels.sweep_launches("velocity_and_strength_gradients",
                                                        "fp32c", n, n) > 2 else "one-sided")
        path64 = ("both-sides" if kernels.sweep_launches("velocity_and_strength_gradients",
                                                          "fp64", n, n) > 2 else "one-sided")
        ops, rsq = _FUSED_OPS[path]
        ops64 = _FUSED_OPS[path64][0]  # the FP64 kernels execute the same pair terms
        r32 = res["fp32c"] * 1e9
        _emit({"config": "config3", "n": n, "fp32c_gpairs_s": round(res["fp32c"], 1),
               "fp64_gpairs_s": round(res["fp64"], 1),
               "speedup": round(res["fp32c"] / res["fp64"], 2), "fp32c_path": path,
               "fp64_path": path64,
               "fp32_pipe_frac": round(r32 * ops / peaks["ffma"], 3),
               "fp32_pipe_frac_of_packed": round(r32 * ops / peaks["ffma2"], 3),
               "sfu_frac": round(r32 * rsq / peaks["mufu"], 3),
               "fp64_pipe_frac_excl_rsqrt": round(res["fp64"] * 1e9 * ops64 / peaks["dfma"], 3),
               "rel_err_velocity": _rel(out["fp32c"][0], out["fp64"][0]),
               "rel_err_stretching": _rel(out["fp32c"][1], out["fp64"][1])})


def config4(args):
    from openonda_b200 import autodiff

    f = configs.perturbed_ring()
    r = lambda z: torch.from_numpy(np.asarray(z, np.float32).astype(np.float64)).cuda()
    x0, a0, s0 = r(f.positions), r(f.strengths), r(f.radii)
    steps, dt, every = args.steps or 50, 0.01, 10

    def grad(prec):
        x, a, s = (z.clone().requires_grad_() for z in (x0, a0, s0))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xT, aT = autodiff.trajectory(x, a, s, None, dt, steps, prec, checkpoint_every=every)
        e = autodiff.kinetic_energy(xT, aT, s, prec)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        g = torch.autograd.grad(e, (x, a, s))
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        return float(e), g, t1 - t0, t2 - t1

    e32, g32, f32, b32 = grad("fp32c")
    e64, g64, f64, b64 = grad("fp64")

    def loss64(x, a, s):
        with torch.no_grad():
            xT, aT = autodiff.trajectory(x, a, s, None, dt, steps, "fp64")
            return float(kernels.total_kinetic_energy(xT, aT, s, precision="fp64"))

    rng = np.random.default_rng(2024)
    n_fd = args.fd or 64
    h = 1e-6
    fd_err32, fd_err64 = [], []
    bases = (x0, a0, s0)
    for q in range(n_fd):
        which = q % 3
        base = bases[which]
        idx = tuple(int(rng.integers(0, d)) for d in base.shape)
        step = h * (float(a0.abs().max()) if which == 1 else 1.0)
        bp, bm = base.clone(), base.clone()
        bp[idx] += step
        bm[idx] -= step
        args_p, args_m = list(bases), list(bases)
        args_p[which], args_m[which] = bp, bm
        fd = (loss64(*args_p) - loss64(*args_m)) / (2 * step)
        scale = float(g64[which].abs().max())
        fd_err64.append(abs(float(g64[which][idx]) - fd) / scale)
        fd_err32.append(abs(float(g32[which][idx]) - fd) / scale)
    _emit({"config": "config4", "workload": f.description, "n": f.n, "steps": steps,
           "dt": dt, "checkpoint_every": every, "loss_fp32c": e32, "loss_fp64": e64,
           "grad_rel_err_fp32c_vs_fp64": {k: _rel(g32[i], g64[i])
                                           for i, k in enumerate(("x", "alpha", "sigma"))},
           "fd_coordinates": n_fd, "fd_h": h,
           "fd_max_err_fp64_adjoint": max(fd_err64), "fd_max_err_fp32c_adjoint": max(fd_err32),
           "fp32c_forward_s": round(f32, 2), "fp32c_backward_s": round(b32, 2),
           "fp64_forward_s": round(f64, 2), "fp64_backward_s": round(b64, 2)})


def config5(args):
    f = configs.les_ring()
    steps = args.steps or 100
    ps = _system(f, "fp32c", flow_model="LES", viscous_scheme="PSE",
                 time_integration_method="RK4", time_step_size=0.002,
                 les_coefficient=args.les_coefficient)
    assert ps._uc  # one core for the whole ring: the uniform-core sweeps
    t_total = 0.0
    for k in range(steps):
        with _Timer() as t:
            _step(ps)
        t_total += t.ms
    eu, eg = _errors_vs_fp64(ps)
    # the LES filter sums of the final state, FP32c against FP64 (same FP32-rounded state)
    x32, a32, s32 = (t.float().double() for t in (ps.positions, ps.strengths, ps.radii))
    les64 = kernels.les_step_sums(x32, a32, s32, precision="fp64")
    les32 = kernels.les_step_sums(x32, a32, s32, precision="fp32c", uniform_core=ps._uc)
    ew = _rel(les32[2], les64[2])
    ee = abs(float(les32[3]) - float(les64[3])) / abs(float(les64[3]))
    # both coefficient schemes on the final state: the one the run used, and the other
    cnu_run = ps.Cnu
    with _Timer() as tl:
        sums = ps._les_least_squares(ps._vorticity())
    cnu_lsq = ps.Cnu
    ps.Cnu = cnu_run
    lm, mm = (float(v) for v in sums.cpu())
    n = f.n
    # 7 N^2 pair sums per step as the reference counts them (velocity + stretching counted
    # once), run here as 5 sweeps: LES step sums (velocity, stretching, vorticity,
    # enstrophy), PSE and 3 RK-stage velocities.  Gpairs/s counts the 7 sums.
    sums = 7.0
    _emit({"config": "config5", "workload": f.description, "n": n, "steps": steps,
           "precision": "fp32c", "uniform_core": ps._uc,
           "ms_per_step": round(t_total / steps, 1),
           "pair_sums_per_step": int(sums), "sweeps_per_step": 5,
           "gpairs_per_s": round(sums * n * n / (t_total / steps / 1e3) / 1e9, 1),
           "rel_err_velocity_last_step": eu, "rel_err_stretching_last_step": eg,
           "rel_err_vorticity_last_step": ew, "rel_err_enstrophy_last_step": ee,
           "les_coefficient": args.les_coefficient, "cnu": cnu_run,
           "cnu_least_squares_final_state": cnu_lsq,
           "least_squares_sums": {"LM": lm, "MM": mm,
                                  "C_unclipped": math.sqrt(lm / mm) if lm > 0 and mm > 0
                                  else None},
           "least_squares_ms": round(tl.ms, 1)})


def sweeps(args):
    """Time of each FP32c sweep of an LES step on the dynamic-LES ring (default N = 2^20):
    the fused LES step sums against the separate sweeps they replace, plus PSE and the
    velocity-only RK-stage sweep.  With --precision fp64: the FP64 self sums that take the
    both-sides schedule, each also timed one-sided (general cores, or --uniform-core)."""
    if args.precision == "fp64":
        return _sweeps_fp64(args)
    n = args.n or (1 << 20)
    k = 1 << (int(np.log2(n)) // 2)
    f = configs.les_ring(n_azimuthal=k, n_section=n // k)
    n = f.n
    r = lambda z: torch.from_numpy(np.asarray(z, np.float64)).cuda()
    x, a, s, nu = r(f.positions), r(f.strengths), r(f.radii), r(f.viscosities)
    p = "fp32c"
    cases = {
        "les_step_sums": lambda uc: kernels.les_step_sums(x, a, s, precision=p,
                                                          uniform_core=uc),
        "velocity_and_strength_gradients":
            lambda uc: kernels.velocity_and_strength_gradients(x, a, s, precision=p,
                                                               uniform_core=uc),
        "vorticity_field_at": lambda uc: kernels.vorticity_field_at(x, x, a, s, precision=p),
        "les_test_filter": lambda uc: kernels.les_test_filter(x, a, 2.0 * s, a, precision=p),
        "total_enstrophy": lambda uc: kernels.total_enstrophy(x, a, s, precision=p,
                                                              uniform_core=uc),
        "strength_gradients_pse":
            lambda uc: kernels.strength_gradients_pse(x, a, s, nu, precision=p,
                                                      uniform_core=uc),
        "selfinduced_velocity": lambda uc: kernels.selfinduced_velocity(x, a, s, precision=p,
                                                                        uniform_core=uc),
    }
    reps = args.steps or 3
    for name, fn in cases.items():
        for uc in (False, True):
            if uc and name in ("vorticity_field_at", "les_test_filter"):
                continue  # probe-style sums have no uniform-core form
            fn(uc)
            with _Timer() as t:
                for _ in range(reps):
                    fn(uc)
            ms = t.ms / reps
            _emit({"sweep": name, "uniform_core": uc, "n": n, "precision": p,
                   "ms": round(ms, 2),
                   "gpairs_per_s": round(float(n) * n / (ms / 1e3) / 1e9, 1)})


def _sweeps_fp64(args):
    n = args.n or (1 << 20)
    k = 1 << (int(np.log2(n)) // 2)
    f = configs.les_ring(n_azimuthal=k, n_section=n // k)
    n = f.n
    r = lambda z: torch.from_numpy(np.asarray(z, np.float64)).cuda()
    x, a, s, nu = r(f.positions), r(f.strengths), r(f.radii), r(f.viscosities)
    p = "fp64"
    uc = bool(args.uniform_core)  # the ring has one core
    cases = {
        "les_step_sums": lambda: kernels.les_step_sums(x, a, s, precision=p, uniform_core=uc),
        "velocity_and_strength_gradients":
            lambda: kernels.velocity_and_strength_gradients(x, a, s, precision=p,
                                                            uniform_core=uc),
        "strength_gradients_pse": lambda: kernels.strength_gradients_pse(x, a, s, nu,
                                                                         precision=p,
                                                                         uniform_core=uc),
        "selfinduced_velocity": lambda: kernels.selfinduced_velocity(x, a, s, precision=p,
                                                                     uniform_core=uc),
    }
    reps = args.steps or 1
    for name, fn in cases.items():
        row = {"sweep": name, "n": n, "precision": p, "uniform_core": uc}
        for sched, thr in (("both_sides", None), ("one_sided", 1 << 40)):
            old = kernels.set_symmetric_min_n(thr) if thr is not None else None
            try:
                fn()
                with _Timer() as t:
                    for _ in range(reps):
                        fn()
            finally:
                if old is not None:
                    kernels.set_symmetric_min_n(old)
            ms = t.ms / reps
            row[sched] = {"ms": round(ms, 1),
                          "gpairs_per_s": round(float(n) * n / (ms / 1e3) / 1e9, 1)}
        _emit(row)


def pairshards(args):
    """Each rank's share of a multi-GPU sweep of the fused sum, timed on this one GPU (the
    ranks run in turn; the collectives are not part of it): pair shards (the both-sides
    schedule split by tiles and diagonal pairs, vpm_sweep_pairs_partial + the FP64 rows)
    against target shards (vpm_sweep_records, one-sided, N / world targets).  The slowest
    rank sets the step, so the projected rate is N^2 over the slowest rank's time; the
    exchanges it leaves out move 64 MB (records) and, for pair shards, 72 MB (rows) at
    N = 2^20."""
    from openonda_b200 import _lib
    from openonda_b200.distributed import (pair_shard_ranges, pairs_layout, shard_range,
                                           sweep_pairs_partial)

    n = args.n or (1 << 20)
    f = configs.random_cloud(n, seed=0)
    r32 = lambda z: torch.from_numpy(np.asarray(z, np.float32).astype(np.float64)).cuda()
    x, a, s = r32(f.positions), r32(f.strengths), r32(f.radii)
    lib = _lib.load()
    code = _lib.precision_code("fp32c")
    rec = torch.empty((n, int(lib.vpm_record_bytes(code)) // 4), dtype=torch.float32,
                      device=x.device)
    _lib.check(lib.vpm_pack_records(x.data_ptr(), a.data_ptr(), s.data_ptr(), None, n, code,
                                    rec.data_ptr(), torch.cuda.current_stream().cuda_stream))
    nt, npairs, per, nv, wsb = pairs_layout(n, "fp32c")
    ws = torch.empty(max(wsb, 256), dtype=torch.uint8, device=x.device)
    rows = torch.empty((n, nv), dtype=torch.float64, device=x.device)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=x.device)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1)

    t1 = timed(lambda: kernels.velocity_and_strength_gradients(x, a, s, precision="fp32c"))
    _emit({"workload": "pairshards", "n": n, "world": 1, "ms": round(t1, 2),
           "gpairs_per_s": round(float(n) * n / t1 / 1e6, 1)})
    for world in args.sizes or (2, 4, 8):
        pair_ms, tgt_ms = [], []
        for r in range(world):
            t0_, t1_, p0, p1 = pair_shard_ranges(nt, npairs, r, world)
            pair_ms.append(timed(lambda: sweep_pairs_partial(rec, n, (t0_, t1_), (p0, p1),
                                                             rows, ws, "fp32c")))
            lo, hi = shard_range(n, r, world)
            m = hi - lo
            nb = kernels.workspace_bytes("velocity_and_strength_gradients", "fp32c", m, n)
            wst = torch.empty(max(nb, 256), dtype=torch.uint8, device=x.device)
            u = torch.empty((m, 3), dtype=torch.float64, device=x.device)
            g = torch.empty_like(u)
            tgt_ms.append(timed(lambda: _lib.check(lib.vpm_sweep_records(
                _lib.OPS["velocity_and_strength_gradients"], rec.data_ptr(), n, lo, m, 0,
                u.data_ptr(), g.data_ptr(), code, wst.data_ptr(), wst.numel(),
                torch.cuda.current_stream().cuda_stream))))
            del wst
        tp, tt = max(pair_ms), max(tgt_ms)
        _emit({"workload": "pairshards", "n": n, "world": world,
               "pair_shards": {"slowest_rank_ms": round(tp, 2),
                               "fastest_rank_ms": round(min(pair_ms), 2),
                               "projected_gpairs_per_s": round(float(n) * n / tp / 1e6, 1),
                               "per_gpu_vs_one_gpu": round(t1 / (world * tp), 3)},
               "target_shards": {"slowest_rank_ms": round(tt, 2),
                                 "projected_gpairs_per_s": round(float(n) * n / tt / 1e6, 1),
                                 "per_gpu_vs_one_gpu": round(t1 / (world * tt), 3)}})


def peaks(args):
    """Throughput of the FP32 pipes by microbenchmark (vpm_launch_fma_peak), at three
    occupancies: scalar FFMA, packed FFMA2, a 1:1 mix of the two, and MUFU rsqrt; in lane
    operations per clock per SM at the nominal 1965 MHz."""
    dev = torch.device("cuda")
    props = torch.cuda.get_device_properties(dev)
    for kind, name, lanes in ((0, "ffma", 16), (3, "ffma2", 32), (4, "ffma2+ffma", 32),
                              (2, "mufu_rsqrt", 16)):
        for per_sm, threads in ((8, 256), (4, 128), (2, 128)):
            blocks = props.multi_processor_count * per_sm
            sink = torch.empty(blocks * threads, dtype=torch.float32, device=dev)
            iters = 1 << 13
            kernels.launch_fma_peak(kind, blocks, threads, 64, sink)
            best = float("inf")
            for _ in range(5):
                with _Timer() as t:
                    kernels.launch_fma_peak(kind, blocks, threads, iters, sink)
                best = min(best, t.ms / 1e3)
            ops = blocks * threads * iters * lanes
            _emit({"pipe": name, "warps_per_sm": per_sm * threads // 32,
                   "t_lane_ops_per_s": round(ops / best / 1e12, 2),
                   "lane_ops_per_clk_per_sm": round(ops / best / props.multi_processor_count
                                                    / 1.965e9, 1)})


def stepkernels(args):
    from openonda_b200 import _lib

    lib = _lib.load()
    n = args.n or (1 << 22)
    dev = torch.device("cuda")
    st = torch.cuda.current_stream().cuda_stream
    x, k1, k2, k3, k4 = (torch.rand((n, 3), dtype=torch.float64, device=dev) for _ in range(5))
    out = torch.empty_like(x)
    h1, h2, h3 = (torch.rand_like(x) for _ in range(3))
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    cases = {
        "axpy (RK stage)": (lambda: lib.vpm_axpy(x.data_ptr(), k1.data_ptr(), 0.005, x.numel(),
                                                 out.data_ptr(), st), 72),
        "rk4_combine": (lambda: lib.vpm_rk4_combine(x.data_ptr(), k1.data_ptr(), k2.data_ptr(),
                                                    k3.data_ptr(), k4.data_ptr(), 0.01,
                                                    x.numel(), out.data_ptr(), st), 144),
        "bdf (BDF4 step)": (lambda: lib.vpm_bdf_update(out.data_ptr(), h1.data_ptr(),
                                                       h2.data_ptr(), h3.data_ptr(),
                                                       k1.data_ptr(), x.numel(), 5, 0.01, st),
                            216),
    }
    for name, (fn, bytes_per) in cases.items():
        fn()
        times = []
        for _ in range(10):
            flush.fill_(0)
            with _Timer() as t:
                fn()
            times.append(t.ms)
        ms = float(np.median(times))
        _emit({"kernel": name, "n": n, "bytes": bytes_per * n, "ms": round(ms, 4),
               "gb_s": round(bytes_per * n / (ms / 1e3) / 1e9, 1)})


def _reference_module(name):
    sys.path.insert(0, os.path.join(HERE, "baseline"))
    from install_ref import load_reference_module

    return load_reference_module(name)


def reference(args):
    """The reference's own code timed on this box, on the random cloud of the throughput
    sweep: its Numba-CUDA kernels (ParticlesPhysicsCuda.py, unmodified, from baseline/_ref) on
    the GPU -- kernel time by CUDA events and end to end through its module functions, which
    copy inputs in and results out on every call -- and its Numba CPU module
    (ParticlesPhysics.py) on all host cores.  Each result is compared with this library's FP64
    drop-in on the same inputs."""
    n = args.n or 131072
    f = configs.random_cloud(n, seed=0)
    x, a, s, nu = (np.ascontiguousarray(z) for z in (f.positions, f.strengths, f.radii,
                                                     f.viscosities))
    dev = torch.device("cuda")
    tx, ta, ts, tn = (torch.from_numpy(z).to(dev) for z in (x, a, s, nu))
    ours = {
        "velocity": kernels.selfinduced_velocity(tx, ta, ts, precision="fp64"),
        "stretching": kernels.strength_gradients(tx, ta, ts, precision="fp64"),
        "pse": kernels.strength_gradients_pse(tx, ta, ts, tn, precision="fp64"),
    }
    ours = {k: v.cpu().numpy() for k, v in ours.items()}
    try:
        import numba
        from numba import cuda

        t0 = time.perf_counter()
        mod = _reference_module("ParticlesPhysicsCuda")
        jit_s = time.perf_counter() - t0
        cc = cuda.get_current_device().compute_capability
    except Exception as e:  # noqa: BLE001 -- report why, do not fail the run
        _emit({"reference_gpu": "unavailable on this box",
               "error": f"{type(e).__name__}: {str(e).splitlines()[0] if str(e) else ''}"})
        mod = None
    if mod is not None:
        xd, ad, sd, nd = (cuda.to_device(z) for z in (x, a, s, nu))
        od = cuda.device_array_like(x)
        blocks = (n + mod.threads_per_block - 1) // mod.threads_per_block
        cases = {
            "velocity": (mod.get_selfinduced_velocity_kernel, (xd, ad, sd, od),
                         lambda: mod.get_selfinduced_velocity(x, a, s)),
            "stretching": (mod.get_strength_gradients_kernel, (xd, ad, sd, od),
                           lambda: mod.get_strength_gradients(x, a, s)),
            "pse": (mod.get_strength_gradients_PSE_kernel, (xd, ad, sd, nd, od),
                    lambda: mod.get_strength_gradients_PSE(x, a, s, nu)),
        }
        for name, (kern, kargs, wrapper) in cases.items():
            kern[blocks, mod.threads_per_block](*kargs)  # first launch loads the module
            cuda.synchronize()
            e0, e1 = cuda.event(), cuda.event()
            e0.record()
            kern[blocks, mod.threads_per_block](*kargs)
            e1.record()
            e1.synchronize()
            ms = cuda.event_elapsed_time(e0, e1)
            got_kernel = od.copy_to_host()
            t0 = time.perf_counter()
            got = wrapper()
            e2e_s = time.perf_counter() - t0
            _emit({"reference_gpu": name, "n": n, "numba": numba.__version__,
                   "device_cc": list(cc), "module_import_and_jit_s": round(jit_s, 1),
                   "kernel_ms": round(ms, 2),
                   "kernel_gpairs_per_s": round(float(n) * n / (ms / 1e3) / 1e9, 3),
                   "e2e_ms": round(e2e_s * 1e3, 2),
                   "e2e_gpairs_per_s": round(float(n) * n / e2e_s / 1e9, 3),
                   "rel_diff_ours_fp64_vs_reference": _rel(ours[name], got),
                   "rel_diff_kernel_vs_wrapper": _rel(got_kernel, got)})
    # the reference's CPU module, all host cores (Numba parallel), on target subsets
    try:
        import numba

        cpu = _reference_module("ParticlesPhysics")
    except Exception as e:  # noqa: BLE001
        _emit({"reference_cpu": "unavailable on this box",
               "error": f"{type(e).__name__}: {e}"})
        return
    threads = numba.get_num_threads()
    m = 64
    cpu.get_induced_velocity_at(x[:m], x[:m], a[:m], s[:m])  # JIT
    t0 = time.perf_counter()
    cpu.get_induced_velocity_at(x[:m], x, a, s)
    rate = m * n / (time.perf_counter() - t0)
    m = int(min(n, max(64, rate * (args.cpu_seconds or 5.0) / n)))
    t0 = time.perf_counter()
    got = cpu.get_induced_velocity_at(x[:m], x, a, s)
    dt = time.perf_counter() - t0
    _emit({"reference_cpu": "velocity (get_induced_velocity_at, target rows x all sources)",
           "n_sources": n, "n_targets": m, "threads": threads, "s": round(dt, 2),
           "gpairs_per_s": round(m * n / dt / 1e9, 4)})
    ns = min(n, args.cpu_n or 16384)
    xs, as_, ss, nus = x[:ns], a[:ns], s[:ns], nu[:ns]
    for name, fn in (("stretching", lambda: cpu.get_strength_gradients(xs, as_, ss)),
                     ("pse", lambda: cpu.get_strength_gradients_PSE(xs, as_, ss, nus))):
        if name == "stretching":
            cpu.get_strength_gradients(xs[:64], as_[:64], ss[:64])  # JIT
        else:
            cpu.get_strength_gradients_PSE(xs[:64], as_[:64], ss[:64], nus[:64])
        t0 = time.perf_counter()
        fn()
        dt = time.perf_counter() - t0
        _emit({"reference_cpu": name, "n": ns, "threads": threads, "s": round(dt, 2),
               "gpairs_per_s": round(float(ns) * ns / dt / 1e9, 4)})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["config1", "config2", "config3", "config4", "config5",
                                         "stepkernels", "sweeps", "peaks", "reference",
                                         "pairshards"])
    ap.add_argument("--cpu-seconds", type=float, default=None)
    ap.add_argument("--les-coefficient", default="reference",
                    choices=["reference", "least_squares"])
    ap.add_argument("--cpu-n", type=int, default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--fd", type=int, default=None)
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--sizes", type=int, nargs="*", default=None)
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--uniform-core", action="store_true")
    args = ap.parse_args()
    globals()[args.workload](args)


if __name__ == "__main__":
    main()
