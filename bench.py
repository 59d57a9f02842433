#!/usr/bin/env python
"""Benchmark of the INC 1D hybrid time-stepper on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ks_plain|burgers_plain|burgers_batched|burgers_diff|ks_diff]

Metric: cell-steps/s (one grid point advanced by one reference step()).
Default workload: the plain KS configuration - 1024 trajectories, N=256,
L=64, dt=0.25, ETRK2, a constant seeded correction field s, 400 step() calls
per rollout, all frames stored.  A bench "step" is one such rollout.

Printed (rank 0, one JSON line):
  value      - fused rollout (one launch for the whole rollout), inputs resident
               in HBM, device-timed with CUDA events, max over ranks;
  e2e        - the same through the public API (inc_b200.rollout.ks_rollout)
               with the inputs copied from pinned host memory and the final
               state copied back inside the timed region;
  plain      - the same kernels one launch per step() (eager, and captured in
               a CUDA graph), plus forward+backward numbers of both forms;
  roofline   - the fused kernel's FP32 throughput against an FMA-loop peak
               measured in this run;
  cpu_baseline - the FP32 numpy port of the reference (oracle/) on the host
               cores, on a bounded sample;
  error      - the timed launch's own frames against the FP64 oracle on the
               same inputs (relative L2 at 1, 10 and 20 step() calls);
  configs    - (default run) the other four configurations, each measured
               the same way with fewer timed repeats: Burgers plain (32 x 128,
               200 SSP-RK3 steps), the ragged batch (4096 rows, 500 steps),
               and the two differentiable training steps (Burgers 256 x 256
               with the CNN corrector, KS 512 x 512 with the FNO corrector),
               each with its fused-over-per-step ratios, roofline, e2e and
               error against FP64.
Multi-GPU (torchrun): every rank runs the full workload on its own GPU (weak
scaling, trajectories are independent, no data-path collective).
"""
from __future__ import annotations

import argparse
import copy
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["ks_plain", "burgers_plain", "burgers_batched", "burgers_diff", "ks_diff"],
                    default="ks_plain")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="the default workload only (no compact blocks of the other configurations)")
    ap.add_argument("--extra-steps", type=int, default=3, help="timed repeats of each compact block")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--profile", nargs="?", const="ks", default=None,
                    choices=["ks", "burgers_ragged", "burgers_plain", "burgers_plain_bwd", "ks_bwd", "ks_tape",
                             "burgers_cnn", "spectral_conv", "adaptive"],
                    help="a small case of one kernel for ncu (no JSON)")
    ap.add_argument("--profile-rows", type=int, default=1024, help="rows of the KS profile case")
    ap.add_argument("--tpp", type=int, default=None,
                    help="KS threads per row pair (default: autotuned; the profile case uses 32)")
    return ap.parse_args()


# ----------------------------------------------------------------------------
# CPU baseline: the oracle's FP32 numpy port of the reference, on a process
# pool of all host cores (started with spawn before any CUDA call).
# ----------------------------------------------------------------------------
def _cpu_ks_worker(args):
    import numpy as np
    from oracle import ks as oks
    u0, s, L, dt, steps, scheme = args
    u = u0.astype(np.float32)
    s = s.astype(np.float32)
    t0 = time.perf_counter()
    for _ in range(steps):
        u = oks.step(u, [L] * u.shape[0], dt, scheme, s)
    return time.perf_counter() - t0, u.shape[0] * u.shape[1] * steps


def _cpu_burgers_worker(args):
    import numpy as np
    from oracle import burgers as ob
    u0, N, L, nu, dt, steps, scheme = args
    p = ob.BurgersParams(resolution=N, L=L, dt=dt, nu=np.float32(nu))
    u, t = u0.astype(np.float32), 0.0
    fn = ob.step_ssprk3 if scheme == "ssprk3" else ob.step_euler
    t0 = time.perf_counter()
    for _ in range(steps):
        u, t = fn(u, p, t)
    return time.perf_counter() - t0, u.shape[0] * u.shape[1] * steps


class CpuBaseline:
    def __init__(self):
        import multiprocessing as mp
        self.cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        self.pool = mp.get_context("spawn").Pool(self.cores)

    def run(self, workload, cfg, steps):
        """Wall time and cell-steps of `steps` steps of the whole batch, rows split over the pool."""
        import numpy as np
        chunks = np.array_split(np.arange(cfg["B"]), self.cores)
        if workload == "ks_plain":
            jobs = [(cfg["u0"][c], cfg["s"][c], cfg["L"], cfg["dt"], steps, cfg["scheme"]) for c in chunks if len(c)]
            fn = _cpu_ks_worker
        else:
            jobs = [(cfg["u0"][c], cfg["N"], cfg["L"], cfg["nu"], cfg["dt"], steps, cfg["scheme"])
                    for c in chunks if len(c)]
            fn = _cpu_burgers_worker
        t0 = time.perf_counter()
        res = self.pool.map(fn, jobs)
        wall = time.perf_counter() - t0
        return wall, sum(r[1] for r in res)

    def sample(self, workload, cfg, budget_s):
        """(cell-steps/s, description) of a bounded sample of about budget_s seconds."""
        self.run(workload, cfg, 1)  # worker start-up and imports
        wall1, _ = self.run(workload, cfg, 1)  # calibration
        steps = int(max(1, min(cfg["steps"], budget_s / max(wall1, 1e-3))))
        wall, cells = self.run(workload, cfg, steps)
        desc = (f"{cfg['B']} rows x {steps} of {cfg['steps']} steps, numpy FP32 port of the reference "
                f"(oracle/), rows split over {self.cores} spawned processes")
        return cells / wall, desc, steps

    def close(self):
        self.pool.terminate()


# ----------------------------------------------------------------------------
# GPU helpers
# ----------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.dev = device_index

    def __enter__(self):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            target = f"GPU-{uuid}" if not uuid.startswith("GPU-") else uuid
        except Exception:
            target = str(self.dev)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", target, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower().startswith("active")})
        loaded = [r[0] for r in rows if r[0] > 0.5 * r[1]] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def event_time(fn, iters, flush=None):
    """Per-iteration device times (ms) with CUDA events on the current stream."""
    import torch
    times = []
    for _ in range(iters):
        if flush is not None:
            flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    return times


def ks_error_vs_fp64(frames, cfg, horizons=(1, 10, 20)):
    """Relative L2 error of a KS launch's frames (all rows) against the FP64 oracle
    (oracle/ks.py) run on the same seeded inputs, at the given step() counts.  The
    chaotic dynamics amplify rounding, so the 1e-5 bar holds to a horizon of 20."""
    import numpy as np
    from oracle import ks as oks
    H = max(horizons)
    got = frames[:, :H].double().cpu().numpy()
    B, N, L, dt = cfg["B"], cfg["N"], cfg["L"], cfg["dt"]
    coeffs = oks.coefficients_fp64([L] * B, N, dt, cfg["scheme"], np.float64)
    ref, out = np.asarray(cfg["u0"], dtype=np.float64), {}
    for k in range(1, H + 1):
        ref = oks.step(ref, [L] * B, dt, cfg["scheme"], cfg["s"], None, coeffs)
        if k in horizons:
            out[str(k)] = float(np.linalg.norm(got[:, k - 1] - ref) / np.linalg.norm(ref))
    return {"rel_l2_at_step": out, "rows": B, "tol": 1e-5,
            "vs": "FP64 oracle (oracle/ks.py) on the same seeded inputs, frames of the timed launch"}


def burgers_error_vs_fp64(frames, cfg):
    """Relative L2 error over all rows and frames of a Burgers rollout against the FP64 oracle."""
    import numpy as np
    from oracle import burgers as ob
    p = ob.BurgersParams(resolution=cfg["N"], L=cfg["L"], dt=cfg["dt"], nu=cfg["nu"])
    ref = ob.rollout(np.asarray(cfg["u0"], dtype=np.float64), p, cfg["steps"], cfg["scheme"])
    got = frames.double().cpu().numpy()
    return {"rel_l2_all_frames": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)), "rows": cfg["B"],
            "steps": cfg["steps"], "tol": 1e-5,
            "vs": "FP64 oracle (oracle/burgers.py) on the same seeded inputs, frames of the timed launch"}


def ragged_error_vs_fp64(final_rows, cfg, sample=64, seed=7):
    """Relative L2 error of the ragged launch's final states on a seeded subset of rows against
    the FP64 oracle (rows of one width advanced together, per-row nu and dt)."""
    import numpy as np
    from oracle import burgers as ob
    ns = np.asarray(cfg["n"])
    sub = sorted(np.random.default_rng(seed).choice(cfg["rows"], sample, replace=False).tolist())
    num = den = 0.0
    for n in sorted(set(ns[sub].tolist())):
        idx = [r for r in sub if ns[r] == n]
        u = np.stack([cfg["u0"][r] for r in idx]).astype(np.float64)
        p = ob.BurgersParams(resolution=int(n), L=2 * np.pi, dt=0.0, nu=cfg["nu"][idx][:, None])
        dt = cfg["dt"][idx][:, None]
        for _ in range(cfg["steps"]):
            u, _ = ob.step_ssprk3(u, p, 0.0, None, dt)
        got = np.stack([final_rows[r] for r in idx]).astype(np.float64)
        num += float(np.sum((got - u) ** 2))
        den += float(np.sum(u ** 2))
    return {"rel_l2_final": (num / den) ** 0.5, "rows": sample, "steps": cfg["steps"], "tol": 1e-5,
            "vs": f"FP64 oracle (oracle/burgers.py) on {sample} seeded rows of the timed launch's final state"}


def fp32_peak_tflops(device):
    """FP32 FMA throughput of this GPU, measured with inc_bench_fma."""
    import torch
    from inc_b200 import _native as nat
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    blocks, iters = sms * 8, 4096
    out = torch.empty(blocks * 256, device=device)

    def run():
        nat.check(nat.lib().inc_bench_fma(out.data_ptr(), blocks, iters, nat.stream_of(device)), "bench_fma")

    run()
    torch.cuda.synchronize()
    best = min(event_time(run, 5))
    flops = blocks * 256 * iters * 16 * 8 * 2
    return flops / (best * 1e-3) / 1e12


# ----------------------------------------------------------------------------
# KS plain configuration
# ----------------------------------------------------------------------------
def bench_ks(args, dev, world):
    import torch
    from types import SimpleNamespace
    from inc_b200.roofline import ks_flops_per_cell_step, ks_impl_flops_per_cell_step, plain_bytes_per_cell_step
    from inc_b200.rollout import ks_rollout
    from inc_b200.solvers import KSSolverTorch
    from inc_b200.workloads import ks_plain_config

    from inc_b200 import autotune
    cfg = ks_plain_config()
    B, N, steps, L, dt = cfg["B"], cfg["N"], cfg["steps"], cfg["L"], cfg["dt"]
    cells = B * N * steps
    if args.tpp:  # pinned layout (e.g. for a profiler run, whose timings would mislead the autotuner)
        tpp = args.tpp
        cfg["layout"] = {"threads_per_pair": tpp, "autotune": "skipped (--tpp)"}
    else:
        tpp, tune_ms = autotune.tune_ks(N, B, cfg["scheme"], device=dev, L=L, dt=dt)  # outside the timed regions
        cfg["layout"] = {"threads_per_pair": tpp, "autotune_ms_per_50_steps": tune_ms}
    ds = torch.full((B,), L, device=dev)
    solver = KSSolverTorch(SimpleNamespace(resolution=N, dt=dt, device=dev, domain_size=ds,
                                           alpha=torch.zeros(B, device=dev), time_scheme=cfg["scheme"],
                                           threads_per_pair=tpp))
    u0_h = torch.tensor(cfg["u0"], dtype=torch.float32).pin_memory()
    s_h = torch.tensor(cfg["s"], dtype=torch.float32).pin_memory()
    u0 = u0_h.to(dev)
    s = s_h.to(dev)
    plan = solver.plan_for(u0, ds)
    frames = torch.empty(B, steps, N, device=dev)
    flush_buf = torch.empty(256 * 2 ** 20 // 4, device=dev)  # 256 MB > 126 MB L2

    def flush():
        flush_buf.fill_(1.0)

    # --- fused rollout (value) -------------------------------------------------
    def fused():
        plan.rollout(u0, s, steps, frames, None, 0, None)

    for _ in range(args.warmup):
        fused()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        t_fused = event_time(fused, args.steps, flush)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms_fused = sum(t_fused) / len(t_fused)
    error = ks_error_vs_fp64(frames, cfg)  # the timed launch's own frames, outside the timed region

    # --- the same rollout with the opt-in 2/3-rule truncation (the reference's "3/2 padding"
    # is a physical-space no-op, so the headline runs without it, as the reference does)
    solver_d = KSSolverTorch(SimpleNamespace(resolution=N, dt=dt, device=dev, domain_size=ds,
                                             alpha=torch.zeros(B, device=dev), time_scheme=cfg["scheme"],
                                             threads_per_pair=tpp, dealias=True))
    plan_d = solver_d.plan_for(u0, ds)

    def fused_dealias():
        plan_d.rollout(u0, s, steps, frames, None, 0, None)

    for _ in range(args.warmup):
        fused_dealias()
    t_dealias = event_time(fused_dealias, args.steps, flush)
    if world > 1:
        torch.distributed.barrier()

    # --- plain: one launch per step() (eager, and captured in a CUDA graph) -------
    bufs = [torch.empty(B, N, device=dev) for _ in range(2)]
    results = torch.empty(B, steps, N, device=dev)

    def plain():
        u = u0
        for k in range(steps):
            out = bufs[k & 1]
            plan.step(u, s, None, out)
            results[:, k] = out  # simulate_rollout's results[:, step] = u_next
            u = out

    for _ in range(args.warmup):
        plain()
    torch.cuda.synchronize()
    t_plain = event_time(plain, max(2, args.steps // 2), flush)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        plain()
    torch.cuda.current_stream(dev).wait_stream(side)
    with torch.cuda.graph(graph):
        plain()
    graph.replay()
    torch.cuda.synchronize()
    t_graph = event_time(graph.replay, max(2, args.steps // 2), flush)

    # --- forward + backward (loss = sum(w * frames)) ---------------------------
    K = 8
    nseg = (steps + K - 1) // K
    ckpts = torch.empty(B, nseg, N, device=dev)
    g_frames = torch.randn(B, steps, N, device=dev, generator=torch.Generator(dev).manual_seed(5))
    g_u0 = torch.empty(B, N, device=dev)
    g_s = torch.empty(B, N, device=dev)

    def fused_fb():
        plan.rollout(u0, s, steps, frames, None, K, ckpts)
        plan.rollout_bwd(ckpts, s, steps, K, g_frames, None, g_u0, g_s)

    states = torch.empty(steps + 1, B, N, device=dev)
    ga, gb, gsk = torch.empty(B, N, device=dev), torch.empty(B, N, device=dev), torch.empty(B, N, device=dev)

    def plain_fb():
        states[0].copy_(u0)
        for k in range(steps):
            plan.step(states[k], s, None, states[k + 1])
        g_s.zero_()
        ga.zero_()
        for k in range(steps - 1, -1, -1):
            ga.add_(g_frames[:, k])
            plan.step_bwd(states[k], s, None, ga, gb, gsk)
            g_s.add_(gsk)
            ga.copy_(gb)

    tape = torch.empty(plan.tape_size(steps), dtype=torch.uint8, device=dev)  # 1.3 GB at 1024 x 256 x 400

    def fused_fb_tape():  # the forward records every step's states; the backward replays nothing
        plan.rollout_tape(u0, s, steps, frames, None, tape)
        plan.rollout_bwd_tape(tape, s, steps, g_frames, None, g_u0, g_s)

    for _ in range(max(1, args.warmup)):
        fused_fb()
        fused_fb_tape()
        plain_fb()
    torch.cuda.synchronize()
    t_ffb = event_time(fused_fb, max(2, args.steps // 2), flush)
    t_ffbt = event_time(fused_fb_tape, max(2, args.steps // 2), flush)
    t_pfb = event_time(plain_fb, 2, flush)
    del tape

    # --- e2e through the public API with host buffers -----------------------------
    u_final_h = torch.empty(B, N).pin_memory()

    def e2e():
        u0_d = u0_h.to(dev, non_blocking=True)
        s_d = s_h.to(dev, non_blocking=True)
        fr = ks_rollout(solver, u0_d, steps, ds, s=s_d)
        u_final_h.copy_(fr[:, -1], non_blocking=True)

    with torch.no_grad():
        for _ in range(args.warmup):
            e2e()
        torch.cuda.synchronize()
        t_e2e = event_time(e2e, args.steps, flush)

    # --- roofline of the fused kernel ------------------------------------------------
    # DRAM traffic of one launch of this workload, from one ncu capture
    # (profiles/ks_rollout_fused_b1024_n256_dram.md): 3.07 MB read + 359.1 MB written.
    extra_traffic = 362.2e6 if (B, N, steps) == (1024, 256, 400) else None
    peak = fp32_peak_tflops(dev)
    flops_cell = ks_flops_per_cell_step(N, cfg["scheme"])  # the reference algorithm's frozen count
    achieved = flops_cell * cells / (ms_fused * 1e-3) / 1e12
    impl_cell = ks_impl_flops_per_cell_step(N, cfg["scheme"])  # what this kernel executes
    impl_achieved = impl_cell * cells / (ms_fused * 1e-3) / 1e12
    plain_ms_step = sum(t_plain) / len(t_plain) / steps
    times = dict(fused=ms_fused, plain=sum(t_plain) / len(t_plain), graph=sum(t_graph) / len(t_graph),
                 fused_fb=sum(t_ffb) / len(t_ffb), plain_fb=sum(t_pfb) / len(t_pfb),
                 e2e=sum(t_e2e) / len(t_e2e), dealias=sum(t_dealias) / len(t_dealias),
                 fused_fb_tape=sum(t_ffbt) / len(t_ffbt))
    cfg["dealias"] = ("as the reference: its 3/2 physical-space padding is a no-op (solver_1d.py:228-233); "
                      "the opt-in 2/3 rule is timed as plain.fused_dealias_2_3")
    extra = dict(
        flops_per_cell_step=flops_cell, peak=peak, achieved=achieved,
        implementation={"flops_per_cell_step": impl_cell, "achieved": impl_achieved, "frac": impl_achieved / peak,
                        "note": "flops this kernel executes: two rows per complex FFT, FFT(s) once per launch"},
        plain_hbm_gbs=plain_bytes_per_cell_step(True) * B * N / (plain_ms_step * 1e-3) / 1e9,
        clocks=clk.summary(), h2d=2 * B * N * 4, d2h=B * N * 4, launches=args.steps, traffic=extra_traffic,
        error=error,
    )
    return cfg, cells, times, extra


# ----------------------------------------------------------------------------
# Burgers plain configuration (N=128, B=32, SSP-RK3, 200 steps)
# ----------------------------------------------------------------------------
def bench_burgers_plain(args, dev, world):
    import torch
    from types import SimpleNamespace
    from inc_b200.roofline import BURGERS_FLOPS, plain_bytes_per_cell_step
    from inc_b200.rollout import burgers_rollout
    from inc_b200.solvers import BurgersSolverTorch
    from inc_b200.workloads import burgers_plain_config

    from inc_b200 import autotune
    cfg = burgers_plain_config()
    B, N, steps = cfg["B"], cfg["N"], cfg["steps"]
    cells = B * N * steps
    cpt, tune_ms = autotune.tune_burgers(N, B, cfg["scheme"], device=dev)  # outside the timed regions
    cfg["layout"] = {"cells_per_thread": cpt, "autotune_ms_per_50_steps": tune_ms}
    sp = SimpleNamespace(resolution=N, dt=cfg["dt"], x=None, adaptive_CFL=None, L=cfg["L"], nu=cfg["nu"], device=dev,
                         convection_term="WENO", equation_type="viscosity", batch_size=B, time_scheme=cfg["scheme"],
                         cells_per_thread=cpt)
    solver = BurgersSolverTorch(sp)
    u0_h = torch.tensor(cfg["u0"], dtype=torch.float32).pin_memory()
    u0 = u0_h.to(dev)
    launch = solver.launch_for(u0)
    frames = torch.empty(B, steps, N, device=dev)
    flush_buf = torch.empty(256 * 2 ** 20 // 4, device=dev)

    def flush():
        flush_buf.fill_(1.0)

    def fused():
        launch.rollout(u0, None, steps, frames, None, 0, None)

    for _ in range(args.warmup):
        fused()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        t_fused = event_time(fused, args.steps, flush)
    torch.cuda.synchronize()
    error = burgers_error_vs_fp64(frames, cfg)  # the timed launch's own frames
    bufs = [torch.empty(B, N, device=dev) for _ in range(2)]

    def plain():
        u = u0
        for k in range(steps):
            out = bufs[k & 1]
            launch.step(u, None, out)
            frames[:, k] = out
            u = out

    for _ in range(args.warmup):
        plain()
    t_plain = event_time(plain, max(2, args.steps // 2), flush)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        plain()
    torch.cuda.current_stream(dev).wait_stream(side)
    with torch.cuda.graph(graph):
        plain()
    graph.replay()
    torch.cuda.synchronize()
    t_graph = event_time(graph.replay, max(2, args.steps // 2), flush)
    # the same per-step loop through the drop-in class (BurgersSolverTorch.step, as the reference's
    # simulate_rollout calls it): the host cost of the public per-step API beside the raw launches
    api = BurgersSolverTorch(sp)

    def api_loop():
        api.t = 0.0
        u = u0
        for k in range(steps):
            u = api.step(u)
            frames[:, k] = u

    def api_steps():  # the drop-in step alone, without the frame copies
        api.t = 0.0
        u = u0
        for _ in range(steps):
            u = api.step(u)

    with torch.no_grad():
        api_loop()
        t_api = event_time(api_loop, max(2, args.steps // 2), flush)
        api_steps()
        t_api_only = event_time(api_steps, max(2, args.steps // 2), flush)
    K = 8
    ckpts = torch.empty(B, (steps + K - 1) // K, N, device=dev)
    g_frames = torch.randn(B, steps, N, device=dev)
    g_u0 = torch.empty(B, N, device=dev)

    def fused_fb():
        launch.rollout(u0, None, steps, frames, None, K, ckpts)
        launch.rollout_bwd(ckpts, None, steps, K, g_frames, None, g_u0, None)

    states = torch.empty(steps + 1, B, N, device=dev)
    ga, gb = torch.empty(B, N, device=dev), torch.empty(B, N, device=dev)

    def plain_fb():
        states[0].copy_(u0)
        for k in range(steps):
            launch.step(states[k], None, states[k + 1])
        ga.zero_()
        for k in range(steps - 1, -1, -1):
            ga.add_(g_frames[:, k])
            launch.step_bwd(states[k], None, ga, gb, None)
            ga.copy_(gb)

    fused_fb()
    plain_fb()
    torch.cuda.synchronize()
    t_ffb = event_time(fused_fb, max(2, args.steps // 2), flush)
    t_pfb = event_time(plain_fb, 2, flush)
    u_final_h = torch.empty(B, N).pin_memory()

    def e2e():
        u0_d = u0_h.to(dev, non_blocking=True)
        fr = burgers_rollout(solver, u0_d, steps)
        u_final_h.copy_(fr[:, -1], non_blocking=True)

    with torch.no_grad():
        for _ in range(args.warmup):
            e2e()
        t_e2e = event_time(e2e, args.steps, flush)
    peak = fp32_peak_tflops(dev)
    flops_cell = BURGERS_FLOPS[cfg["scheme"]]
    ms_fused = sum(t_fused) / len(t_fused)
    achieved = flops_cell * cells / (ms_fused * 1e-3) / 1e12
    plain_ms_step = sum(t_plain) / len(t_plain) / steps
    times = dict(fused=ms_fused, plain=sum(t_plain) / len(t_plain), graph=sum(t_graph) / len(t_graph),
                 fused_fb=sum(t_ffb) / len(t_ffb), plain_fb=sum(t_pfb) / len(t_pfb), e2e=sum(t_e2e) / len(t_e2e),
                 api=sum(t_api) / len(t_api), api_only=sum(t_api_only) / len(t_api_only))
    extra = dict(flops_per_cell_step=flops_cell, peak=peak, achieved=achieved,
                 plain_hbm_gbs=plain_bytes_per_cell_step(False) * B * N / (plain_ms_step * 1e-3) / 1e9,
                 clocks=clk.summary(), h2d=B * N * 4, d2h=B * N * 4, launches=args.steps, error=error)
    return cfg, cells, times, extra


def bench_burgers_batched(args, dev, world):
    import numpy as np
    import torch
    from inc_b200.batched import RaggedBurgers
    from inc_b200.roofline import BURGERS_FLOPS
    from inc_b200.workloads import burgers_batched_config

    from inc_b200 import autotune
    cfg = burgers_batched_config()
    rb = RaggedBurgers(cfg["u0"], cfg["nu"], cfg["dt"], cfg["dx"], scheme=cfg["scheme"], device=dev)
    grid, tune_ms = autotune.tune_ragged(rb)  # outside the timed region
    cfg["layout"] = {"grid_blocks": grid, "warps_per_block": 4, "autotune_ms_per_100_steps": tune_ms}
    steps = cfg["steps"]
    cells = rb.total * steps
    out = torch.empty_like(rb.u0)

    flush_buf = torch.empty(256 * 2 ** 20 // 4, device=dev)  # 256 MB > 126 MB L2

    def flush():
        flush_buf.fill_(1.0)

    def run():
        rb.rollout(steps, out=out)

    for _ in range(args.warmup):
        run()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        t = event_time(run, args.steps, flush)
    torch.cuda.synchronize()
    error = ragged_error_vs_fp64(rb.unpack(out.cpu().numpy()), cfg)  # the timed launch's final state
    # the same kernel one launch per step (the persistent launch with steps = 1), eager and graphed
    bufs = [torch.empty_like(rb.u0) for _ in range(2)]

    def plain():
        u = rb.u0
        for k in range(steps):
            rb.rollout(1, u0=u, out=bufs[k & 1])
            u = bufs[k & 1]

    plain()
    torch.cuda.synchronize()
    t_plain = event_time(plain, max(2, args.steps // 2), flush)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        plain()
    torch.cuda.current_stream(dev).wait_stream(side)
    with torch.cuda.graph(graph):
        plain()
    graph.replay()
    torch.cuda.synchronize()
    t_graph = event_time(graph.replay, max(2, args.steps // 2), flush)
    del graph
    u0_h = rb.u0.cpu().pin_memory()
    out_h = torch.empty_like(u0_h).pin_memory()

    def e2e():
        u = u0_h.to(dev, non_blocking=True)
        o = rb.rollout(steps, u0=u)
        out_h.copy_(o, non_blocking=True)

    for _ in range(args.warmup):
        e2e()
    t_e2e = event_time(e2e, args.steps, flush)
    peak = fp32_peak_tflops(dev)
    ms = sum(t) / len(t)
    flops_cell = BURGERS_FLOPS[cfg["scheme"]]
    times = dict(fused=ms, e2e=sum(t_e2e) / len(t_e2e), plain=sum(t_plain) / len(t_plain),
                 graph=sum(t_graph) / len(t_graph))
    extra = dict(flops_per_cell_step=flops_cell, peak=peak, achieved=flops_cell * cells / (ms * 1e-3) / 1e12,
                 clocks=clk.summary(), h2d=rb.total * 4, d2h=rb.total * 4, launches=args.steps, error=error)
    cfg = dict(name="burgers_batched", B=cfg["rows"], N="64..512", steps=steps, scheme=cfg["scheme"],
               layout=cfg["layout"])
    return cfg, cells, times, extra


def bench_adaptive(dev, reps=5):
    """One adaptive-CFL step (solver_1d.py:148-179) on 4096 x 256 rows, dt spanning about ten
    substeps, beside one fixed-dt Euler step of the same batch: the cooperative kernel's cost
    per substep against a plain step launch (both CUDA-event timed, inputs in L2)."""
    import math
    import torch
    from types import SimpleNamespace
    from inc_b200.solvers import BurgersSolverTorch
    from inc_b200.workloads import burgers_plain_config
    B, N = 4096, 256
    cfg = burgers_plain_config(B=B, N=N)
    u0 = torch.tensor(cfg["u0"], dtype=torch.float32, device=dev)
    mk = lambda cfl: BurgersSolverTorch(SimpleNamespace(  # noqa: E731
        resolution=N, dt=0.05, x=None, adaptive_CFL=cfl, L=2 * math.pi, nu=0.01, device=dev,
        convection_term="WENO", equation_type="viscosity", batch_size=B, time_scheme="euler"))
    ad, fx = mk(0.2), mk(None)
    with torch.no_grad():
        for _ in range(3):
            ad.step(u0)
            fx.step(u0)
        torch.cuda.synchronize()
        t_ad = min(event_time(lambda: ad.step(u0), reps))
        subs = ad.last_substeps
        t_fx = min(event_time(lambda: fx.step(u0), reps))
    return {"batch": B, "n": N, "dt": 0.05, "cfl": 0.2, "substeps": subs, "adaptive_step_ms": t_ad,
            "fixed_dt_step_ms": t_fx, "adaptive_ms_per_substep": t_ad / max(subs, 1),
            "per_substep_over_fixed_step": t_ad / max(subs, 1) / t_fx,
            "kernel": "k_adaptive_grid (one cooperative launch, grid barrier per substep)"}


# ----------------------------------------------------------------------------
# Differentiable rollouts with a corrector network in the loop
# (Burgers + periodic CNN, KS + FNO): one training step = rollout, MSE loss,
# backward through solver and network, Adam update.
# ----------------------------------------------------------------------------
def bench_diff(args, dev, world, which):
    import torch
    from types import SimpleNamespace
    from inc_b200.correctors import FNO1D, PeriodicCNN1D
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import BurgersSolverTorch, KSSolverTorch
    from inc_b200.sharding import average_gradients_
    from inc_b200.workloads import burgers_diff_config, ks_diff_config

    # data-parallel over ranks: every rank trains the same seeded network on its own seeded
    # trajectories and the gradients are averaged every step (one all-reduce)
    rank = torch.distributed.get_rank() if world > 1 else 0
    torch.manual_seed(0)
    # FP32 throughout, the corrector included (cuDNN would otherwise run its convolutions in TF32)
    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    if which == "burgers_diff":
        cfg = burgers_diff_config(seed=3 + 1000 * rank)
        B, N, steps = cfg["B"], cfg["N"], cfg["steps"]
        mk = lambda: BurgersSolverTorch(SimpleNamespace(  # noqa: E731
            resolution=N, dt=cfg["dt"], x=None, adaptive_CFL=None, L=cfg["L"], nu=cfg["nu"], device=dev,
            convection_term="WENO", equation_type="viscosity", batch_size=B, time_scheme=cfg["scheme"]))
        net = PeriodicCNN1D(channels=32, kernel=5, layers=4).to(dev)
        L = None
    else:
        cfg = ks_diff_config(seed=4 + 1000 * rank)
        B, N, steps = cfg["B"], cfg["N"], cfg["steps"]
        L = torch.full((B,), cfg["L"], device=dev)
        mk = lambda: KSSolverTorch(SimpleNamespace(  # noqa: E731
            resolution=N, dt=cfg["dt"], device=dev, domain_size=L, alpha=torch.zeros(B, device=dev),
            time_scheme=cfg["scheme"]))
        net = FNO1D(L=int(cfg["L"]), modes=16, width=64).to(dev)  # the reference's FNO corrector
    cells = B * N * steps
    u0 = torch.tensor(cfg["u0"], dtype=torch.float32, device=dev)
    with torch.no_grad():  # target: the uncorrected solver's trajectory
        target, _ = simulate_rollout(None, mk(), u0, steps, None, L)
        target = target + 0.01 * torch.randn_like(target)
    # the accuracy checks run on the seeded network as built: after the timed Adam steps its
    # state would depend on the signs of near-zero gradients, i.e. on FP32 rounding
    net_at_init = copy.deepcopy(net)
    opt = torch.optim.Adam(net.parameters(), lr=1e-4, capturable=True)

    solver = mk()  # built once: a KS plan uploads its pairing (a host sync) when first used

    def train_step(ckpt):
        if which == "burgers_diff":
            solver.t = 0.0
        res, _ = simulate_rollout(net, solver, u0, steps, "INC", L, checkpoint_every=ckpt)
        loss = torch.mean((res - target) ** 2)
        loss.backward()
        if world > 1:
            average_gradients_(net.parameters(), local_rows=B)
        opt.step()
        opt.zero_grad(set_to_none=False)
        return loss

    def forward_only():  # evaluation rollout; for the CNN corrector simulate_rollout runs the fused kernel
        if which == "burgers_diff":
            solver.t = 0.0
        with torch.no_grad():
            simulate_rollout(net, solver, u0, steps, "INC", L)

    def forward_loop():  # the reference's loop: one corrector call and one step() launch per step
        if which == "burgers_diff":
            solver.t = 0.0
        u = u0
        with torch.no_grad():
            for _ in range(steps):
                solver.correction_s = net(u) if L is None else net(u, L)
                u = solver.step(u) if L is None else solver.step(u, L)

    def train_loop():  # the reference's training loop: one corrector call and one step() per step, autograd
        if which == "burgers_diff":
            solver.t = 0.0
        u, frames = u0, []
        for _ in range(steps):
            solver.correction_s = net(u) if L is None else net(u, L)
            u = solver.step(u) if L is None else solver.step(u, L)
            frames.append(u)
        loss = torch.mean((torch.stack(frames, 1) - target) ** 2)
        loss.backward()
        if world > 1:
            average_gradients_(net.parameters(), local_rows=B)
        opt.step()
        opt.zero_grad(set_to_none=False)
        return loss

    for _ in range(args.warmup):
        train_step(8)
        train_step(None)
        forward_only()
        forward_loop()
        train_loop()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        t_ck = event_time(lambda: train_step(8), args.steps)
    t_plain = event_time(lambda: train_step(None), args.steps)
    t_fwd = event_time(forward_only, args.steps)
    t_loop = event_time(forward_loop, args.steps)
    t_loop_train = event_time(train_loop, args.steps)
    # the evaluation loop replayed from one CUDA graph (inc_b200.graphs)
    from inc_b200.graphs import GraphedRollout
    gsolver = mk()
    graphed = GraphedRollout(net, gsolver, u0, steps, domain_size=L)
    t_gfwd = event_time(lambda: graphed(u0), args.steps)
    # the whole training step captured in one CUDA graph.  The KS corrector (the FNO, in torch)
    # keeps its activations when HBM has room for them (about 70 GB at 512 x 512 x 64 steps):
    # recomputing them under checkpointing costs more than the solver's whole step; the
    # solver's own adjoint recomputes its states either way.  Burgers runs the fused CNN
    # kernels with their segment replay (ckpt_every 8).
    graph_ckpt = 8
    if which == "ks_diff":
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats(dev)
        base = torch.cuda.memory_allocated(dev)
        train_step(None)
        torch.cuda.synchronize()
        need = torch.cuda.max_memory_allocated(dev) - base
        torch.cuda.empty_cache()
        free, _ = torch.cuda.mem_get_info(dev)
        if free > 1.5 * need:
            graph_ckpt = None
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for _ in range(3):
            train_step(graph_ckpt)
    torch.cuda.current_stream(dev).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        train_step(graph_ckpt)
    graph.replay()
    torch.cuda.synchronize()
    t_graph = event_time(graph.replay, args.steps)
    # end to end through the public API: every step's u0 and target come from pinned host
    # memory, the loss goes back to pinned host memory; the eager step (simulate_rollout,
    # backward, Adam)
    u0_host = u0.detach().cpu().pin_memory()
    tgt_host = target.detach().cpu().pin_memory()
    loss_host = torch.empty((), dtype=torch.float32).pin_memory()

    def e2e_step():
        u0.copy_(u0_host, non_blocking=True)
        target.copy_(tgt_host, non_blocking=True)
        loss_host.copy_(train_step(graph_ckpt).detach(), non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    t_e2e = event_time(e2e_step, args.steps)
    launches = count_own_launches(lambda: train_step(graph_ckpt)) * args.steps
    ms = lambda t: sum(t) / len(t)  # noqa: E731
    times = dict(fused=ms(t_graph), e2e=ms(t_e2e), plain=ms(t_plain), fwd=ms(t_fwd), ckpt=ms(t_ck), loop=ms(t_loop),
                 gfwd=ms(t_gfwd), loop_train=ms(t_loop_train))
    extra = dict(clocks=clk.summary(), h2d=(u0.numel() + target.numel()) * 4, d2h=4, launches=launches,
                 graph_ckpt=graph_ckpt)
    extra["checks"] = diff_checks(which, net_at_init, cfg, dev)
    extra["error"] = {k: extra["checks"][k] for k in ("forward_rel_l2_vs_fp64", "grad_max_rel_err_vs_fp64_fd")}
    extra["error"].update(forward_steps=extra["checks"]["forward_steps"], rows=extra["checks"]["rows"],
                          tol={"forward": 1e-5, "grad": 1e-4},
                          vs="FP64 loop on the host (torch corrector in float64, oracle step), FP64 central FD")
    if which == "ks_diff":  # the FNO's spectral convolution layer against the HBM peak
        extra["roofline"] = spectral_layer_roofline(dev, B, N)
    if which == "burgers_diff":  # the fused corrector rollout against the FP32 FMA peak
        from inc_b200.roofline import burgers_cnn_flops_per_cell_step
        fpc = burgers_cnn_flops_per_cell_step(cfg["scheme"])
        achieved = cells * fpc / (ms(t_fwd) * 1e-3) / 1e12
        peak = fp32_peak_tflops(dev)
        extra["fused_inference_roofline"] = {
            "kernel": "inc_burgers_cnn_rollout (k_cnn_rollout<256>)", "bound": "fp32", "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None, "flops_per_cell_step": fpc,
            "peak_source": "FP32 FMA loop (inc_bench_fma) measured in this run"}
    cfg = dict(name=which, B=B, N=N, steps=steps, scheme=cfg["scheme"],
               corrector=("PeriodicCNN1D(4x32ch,k5,GELU)" if which == "burgers_diff" else "FNO1D(L=100, modes=16, width=64), the reference's corrector"))
    del graph, graphed  # a CUDA graph holding NCCL calls must be released before the process group
    torch.cuda.synchronize()
    return cfg, cells, times, extra


def count_own_launches(fn):
    """Kernels of libinc_b200 that one call of fn launches (torch profiler, outside any timed region)."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    return sum(1 for e in prof.events()
               if e.device_type.name == "CUDA" and (e.name.startswith("void inc::") or e.name.startswith("inc::")))


def hbm_peak_gbs():
    """(HBM GB/s, source): the driver-measured copy bandwidth when MEASURED_PEAKS.json holds it, else the
    pool's earlier measurement."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError, TypeError):
        return 6650.0, "fallback (6.65 TB/s, an earlier copy-bandwidth measurement on this pool)"


def spectral_layer_roofline(dev, B, N, W=64, M=16):
    """One FNO layer's spectral(x) + bias + 1x1 branch (inc_spectral_conv1d) at the workload's shape,
    timed alone, against the HBM peak.  Algorithmic bytes: x, addend and y (12 B per point), the rfft
    modes and the mixed modes each written and read (32 B per mode), the weights read, relaid and
    read (24 B per weight entry).  Inputs exceed L2 (192 MB of activations); the calls are replayed from
    a CUDA graph so that the time is the device's."""
    import torch
    from inc_b200.correctors import spectral_conv1d
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.randn(B, W, N, device=dev, generator=g)
    add = torch.randn(B, W, N, device=dev, generator=g)
    wr = torch.rand(W, W, M, device=dev, generator=g) / (W * W)
    wi = torch.rand(W, W, M, device=dev, generator=g) / (W * W)
    bias = torch.randn(W, device=dev, generator=g)
    reps = 10  # layer calls per graph replay: device time without the host's per-call work
    with torch.no_grad():
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(3):
                spectral_conv1d(x, wr, wi, M, bias=bias, addend=add)
        torch.cuda.current_stream(dev).wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(reps):
                spectral_conv1d(x, wr, wi, M, bias=bias, addend=add)
        graph.replay()
        torch.cuda.synchronize()
        t = event_time(graph.replay, 10)
    ms = sum(t) / len(t) / reps
    nbytes = 12 * B * W * N + 32 * B * W * M + 24 * W * W * M
    achieved = nbytes / (ms * 1e-3) / 1e9
    peak, src = hbm_peak_gbs()
    # ncu dram__bytes_read.sum + dram__bytes_write.sum of the four kernels at this shape
    # (profiles/fno_spectral_conv_b512_w64_n512_full.md); outputs still in L2 at the end of a
    # launch are not counted there
    traffic = 167.8e6 if (B, N, W, M) == (512, 512, 64, 16) else None
    return {"kernel": "FNO spectral conv layer forward: k_sc_modes, k_sc_weights, k_sc_mix, k_sc_inverse",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "bytes_per_launch": nbytes, "ms_per_launch": ms, "peak_source": src}


def diff_checks(which, net, cfg, dev, rows=4, fwd_steps=10, grad_steps=8, directions=4, h=1e-6):
    """Accuracy of the differentiable workloads on a subset of rows, outside the timed region:
    the forward error of `fwd_steps` corrected steps against the same loop in FP64 on the host
    (the corrector in float64 torch, the oracle's step), and the gradient of a weighted sum of
    `grad_steps` frames w.r.t. u0 and the network's parameters against FP64 central
    differences (step h) along random directions."""
    import copy
    import numpy as np
    import torch
    from types import SimpleNamespace
    from inc_b200.rollout import simulate_rollout
    from inc_b200.solvers import BurgersSolverTorch, KSSolverTorch
    from oracle import burgers as ob
    from oracle import ks as oks

    N = cfg["N"]
    u0_np = np.asarray(cfg["u0"], dtype=np.float64)[:rows]
    rng = np.random.default_rng(11)
    from inc_b200.correctors import fp64_copy
    net64 = fp64_copy(net).cpu()
    params64 = list(net64.parameters())
    if which == "burgers_diff":
        p = ob.BurgersParams(resolution=N, L=cfg["L"], dt=cfg["dt"], nu=cfg["nu"])
        step64 = ob.step_ssprk3 if cfg["scheme"] == "ssprk3" else ob.step_euler
        L_dev = None

        def mk():
            return BurgersSolverTorch(SimpleNamespace(
                resolution=N, dt=cfg["dt"], x=None, adaptive_CFL=None, L=cfg["L"], nu=cfg["nu"], device=dev,
                convection_term="WENO", equation_type="viscosity", batch_size=rows, time_scheme=cfg["scheme"]))

        def loop64(u, steps):
            t, out = 0.0, []
            for _ in range(steps):
                sv = net64(torch.from_numpy(u)).detach().numpy()
                u, t = step64(u, p, t, sv)
                out.append(u)
            return np.stack(out, 1)
    else:
        Ls = np.full(rows, float(cfg["L"]))
        L_dev = torch.tensor(Ls, dtype=torch.float32, device=dev)
        L_host = torch.tensor(Ls)

        def mk():
            return KSSolverTorch(SimpleNamespace(resolution=N, dt=cfg["dt"], device=dev, domain_size=L_dev,
                                                 alpha=torch.zeros(rows, device=dev), time_scheme=cfg["scheme"]))

        def loop64(u, steps):
            out = []
            for _ in range(steps):
                sv = net64(torch.from_numpy(u), L_host).detach().numpy()
                u = oks.step(u, Ls, cfg["dt"], cfg["scheme"], sv)
                out.append(u)
            return np.stack(out, 1)
    # forward error
    u0 = torch.tensor(u0_np, dtype=torch.float32, device=dev)
    with torch.no_grad():
        fr, _ = simulate_rollout(net, mk(), u0, fwd_steps, "INC", L_dev)
    ref = loop64(u0_np, fwd_steps)
    fwd_err = float(np.linalg.norm(fr.double().cpu().numpy() - ref) / np.linalg.norm(ref))
    # gradient vs central differences
    wgt = rng.standard_normal((rows, grad_steps, N))
    u0g = torch.tensor(u0_np, dtype=torch.float32, device=dev, requires_grad=True)
    net.zero_grad()
    fr, _ = simulate_rollout(net, mk(), u0g, grad_steps, "INC", L_dev, checkpoint_every=4)
    (fr * torch.tensor(wgt, dtype=torch.float32, device=dev)).sum().backward()
    g_u = u0g.grad.double().cpu().numpy()
    g_p = [(torch.view_as_real(q.grad) if q.is_complex() else q.grad).double().cpu().numpy()
           for q in net.parameters()]
    net.zero_grad()

    def loss64(u):
        return float((loop64(u, grad_steps) * wgt).sum())
    errs_u, errs = [], []
    with torch.no_grad():
        for _ in range(directions):  # in u0
            d = rng.standard_normal(u0_np.shape)
            fd = (loss64(u0_np + h * d) - loss64(u0_np - h * d)) / (2 * h)
            errs_u.append(abs(float((g_u * d).sum()) - fd) / max(abs(fd), 1e-12))
        for _ in range(directions):  # in the parameters
            # a complex parameter (the FNO's weights1) moves along a complex direction; its
            # directional derivative is sum(Re g Re d + Im g Im d) with torch's complex gradient
            ds = [rng.standard_normal(tuple(q.shape) + ((2,) if q.is_complex() else ())) for q in params64]
            base = [q.detach().clone() for q in params64]
            vals = []
            for sign in (1.0, -1.0):
                for q, b, d in zip(params64, base, ds):
                    dt = torch.from_numpy(d)
                    q.copy_(b + sign * h * (torch.view_as_complex(dt) if q.is_complex() else dt))
                vals.append(loss64(u0_np))
            for q, b in zip(params64, base):
                q.copy_(b)
            fd = (vals[0] - vals[1]) / (2 * h)
            an = sum(float((g * d).sum()) for g, d in zip(g_p, ds))
            errs.append(abs(an - fd) / max(abs(fd), 1e-12))
    return {"rows": rows, "forward_steps": fwd_steps, "forward_rel_l2_vs_fp64": fwd_err,
            "grad_steps": grad_steps, "fd_h": h, "fd_directions": {"u0": directions, "params": directions},
            "grad_max_rel_err_vs_fp64_fd": max(errs_u + errs),
            "grad_max_rel_err_u0": max(errs_u), "grad_max_rel_err_params": max(errs),
            "network": "the seeded network before the timed training steps",
            "reference": "the same corrected loop in FP64 on the host: torch corrector in float64, oracle step"}


# ----------------------------------------------------------------------------
def reference_arm(args, rank, world):
    """The reference's algorithm on the host cores (the oracle's numpy port)."""
    if rank != 0:
        return
    from inc_b200.workloads import burgers_plain_config, ks_plain_config
    cfg = ks_plain_config() if args.workload == "ks_plain" else burgers_plain_config()
    cpu = CpuBaseline()
    try:
        cpu.run(args.workload, cfg, 1)  # worker start-up and imports
        wall1, _ = cpu.run(args.workload, cfg, 1)
        per_step = max(1, min(cfg["steps"], int(1.0 / max(wall1, 1e-3))))  # ~1 s of CPU work per bench step
        for _ in range(args.warmup):
            cpu.run(args.workload, cfg, per_step)
        walls, cells = [], 0
        for _ in range(args.steps):
            w, c = cpu.run(args.workload, cfg, per_step)
            walls.append(w)
            cells = c
    finally:
        cpu.close()
    v = cells / (sum(walls) / len(walls))
    sample = (f"{cfg['B']} rows x {per_step} steps per bench step (of {cfg['steps']} in the workload), numpy FP32 "
              f"port of the reference (oracle/), rows split over {cpu.cores} spawned processes")
    line = {"metric": "cell-steps/s", "value": v, "unit": "cell-steps/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(walls) / len(walls), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": cfg["name"], "batch": cfg["B"], "n": cfg["N"], "steps_per_rollout": cfg["steps"],
                       "scheme": cfg["scheme"]},
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": cpu.cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


EXTRA_WORKLOADS = ("burgers_plain", "burgers_batched", "burgers_diff", "ks_diff")


def run_workload(name, args, dev, world):
    """Run one workload; device times become the max over ranks."""
    import torch
    if name in ("burgers_diff", "ks_diff"):
        cfg, cells, times, extra = bench_diff(args, dev, world, name)
    else:
        fn = {"ks_plain": bench_ks, "burgers_plain": bench_burgers_plain, "burgers_batched": bench_burgers_batched}
        cfg, cells, times, extra = fn[name](args, dev, world)
    if world > 1:
        keys = sorted(times)
        t = torch.tensor([times[k] for k in keys], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        times = dict(zip(keys, t.tolist()))
    return cfg, cells, times, extra


def diff_line(args, world, cfg, cells, times, extra):
    tot = cells * world
    rate = lambda ms: tot / (ms * 1e-3)  # noqa: E731
    return {
        "metric": "cell-steps/s (fwd+bwd training step)", "value": rate(times["fused"]),
        "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": times["fused"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": cfg["name"], "batch": cfg["B"], "n": cfg["N"], "unroll": cfg["steps"],
                   "scheme": cfg["scheme"], "corrector": cfg["corrector"],
                   "checkpoint_every": extra.get("graph_ckpt"),
                   "checkpoint_note": ("solver adjoint replays its own states; the corrector's activations "
                                       "are kept (None) or recomputed every 8 steps" if cfg["name"] == "ks_diff"
                                       else "solver adjoint replays its states from checkpoints every 8 steps; "
                                       "the fused forward records the CNN's hidden pre-activations (537 MB) "
                                       "and the fused backward reads them"),
                   "value_is": "whole training step (rollout, loss, backward, Adam) in one CUDA graph",
                   "l2": "inputs and activations exceed L2 (not flushed)" if cfg["name"] == "ks_diff"
                   else "not flushed (the recorded pre-activations, 537 MB, exceed L2)",
                   "parallelism": (f"data-parallel over {world} GPUs: per-rank trajectories, corrector "
                                   "gradients averaged by one all-reduce per step" if world > 1
                                   else "single GPU")},
        "eager": {"train_step_ckpt8": rate(times["ckpt"]),
                  "train_step_no_ckpt": rate(times["plain"]),
                  "train_step_per_step_loop": rate(times["loop_train"]),
                  "forward_only": rate(times["fwd"]),
                  "forward_per_step_loop": rate(times["loop"]),
                  "forward_graphed_loop": rate(times["gfwd"])},
        "plain": {"fwd_fused_over_per_step_loop": times["loop"] / times["fwd"],
                  "fwd_bwd_fused_over_per_step_loop": times["loop_train"] / times["ckpt"],
                  "fwd_bwd_fused_graph_over_per_step_loop": times["loop_train"] / times["fused"],
                  "per_step_loop_is": "the reference's loop: one torch corrector call and one step() per step, "
                                      "autograd through both (eager)"},
        "forward_only_is": ("fused corrector + solver kernel (inc_burgers_cnn_rollout)"
                            if cfg["name"] == "burgers_diff" else "corrector in torch, solver step launches"),
        "e2e": {"value": rate(times["e2e"]), "unit": "cell-steps/s",
                "h2d_bytes_per_step": extra["h2d"], "d2h_bytes_per_step": extra["d2h"],
                "api": "eager training step: simulate_rollout, loss.backward(), Adam"},
        "roofline": extra.get("roofline") or extra.get("fused_inference_roofline"),
        "fused_inference_roofline": extra.get("fused_inference_roofline"),
        "error": extra.get("error"),
        "checks": extra.get("checks"),
        "clocks": extra["clocks"],
        "gpu_launches": extra["launches"]}


def plain_line(args, world, cfg, cells, times, extra, cpu_b):
    tot = cells * world
    rate = lambda ms: tot / (ms * 1e-3)  # noqa: E731
    l2 = "flushed (256 MB write) before every timed iteration"
    line = {
        "metric": "cell-steps/s", "value": rate(times["fused"]), "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": times["fused"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": cfg["name"], "batch": cfg["B"], "n": cfg["N"], "steps_per_rollout": cfg["steps"],
                   "scheme": cfg["scheme"], "l2": l2,
                   "per_gpu": "full workload on every rank (trajectories are independent)",
                   "layout": cfg.get("layout"), "dealias": cfg.get("dealias")},
        "e2e": {"value": rate(times["e2e"]), "unit": "cell-steps/s", "h2d_bytes_per_step": extra["h2d"],
                "d2h_bytes_per_step": extra["d2h"],
                "api": "inc_b200.batched.RaggedBurgers.rollout" if cfg["name"] == "burgers_batched"
                else "inc_b200.rollout (fused launch)"},
        "roofline": {"bound": "fp32", "achieved": extra["achieved"], "peak": extra["peak"], "unit": "TFLOP/s",
                     "frac": extra["achieved"] / extra["peak"], "traffic": extra.get("traffic"),
                     "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one full launch, "
                                        "profiles/ks_rollout_fused_b1024_n256_dram.md")
                     if extra.get("traffic") else None,
                     "peak_source": "FP32 FMA loop (inc_bench_fma) measured in this run",
                     "flops_per_cell_step": extra["flops_per_cell_step"],
                     "flops_source": ("frozen per-cell-step count of the reference algorithm "
                                      "(inc_b200/roofline.py)"),
                     "implementation": extra.get("implementation")},
        "error": extra.get("error"),
        "cpu_baseline": cpu_b,
        "clocks": extra["clocks"],
        "gpu_launches": extra["launches"],
    }
    if "plain" in times:
        p = {"eager_per_step": rate(times["plain"]), "graph_per_step": rate(times["graph"]),
             "fused_over_eager": times["plain"] / times["fused"],
             "fused_over_graph": times["graph"] / times["fused"]}
        if "fused_fb" in times:
            p.update({"fwd_bwd_fused": rate(times["fused_fb"]), "fwd_bwd_per_step": rate(times["plain_fb"]),
                      "fwd_bwd_fused_over_per_step": times["plain_fb"] / times["fused_fb"],
                      "plain_step_hbm_gbs": extra.get("plain_hbm_gbs")})
        else:
            p["fwd_bwd"] = "no backward: the ragged batch is a forward-only workload"
        if "dealias" in times:
            p["fused_dealias_2_3"] = rate(times["dealias"])
        if "fused_fb_tape" in times:
            p["fwd_bwd_fused_tape"] = rate(times["fused_fb_tape"])
            p["fwd_bwd_fused_tape_over_per_step"] = times["plain_fb"] / times["fused_fb_tape"]
            p["fwd_bwd_fused_tape_is"] = ("the forward records every step's states in a device tape "
                                          "(inc_ks_rollout_tape) and the backward reads them instead of "
                                          "replaying checkpointed segments")
        if "api" in times:
            p["api_step_eager"] = rate(times["api"])
            p["api_step_ms"] = times["api"] / cfg["steps"]
            p["graph_step_ms"] = times["graph"] / cfg["steps"]
            p["api_over_graph_time"] = times["api"] / times["graph"]
            p["api_step_only_ms"] = times["api_only"] / cfg["steps"]
            p["api_is"] = "BurgersSolverTorch.step(u) per step, eager (the drop-in API simulate_rollout calls)"
        line["plain"] = p
    return line


def compact_block(line):
    """The figures of one workload's line that the headline line carries for it."""
    keys = ("value", "unit", "ms_per_step", "steps", "warmup", "config", "plain", "roofline", "e2e", "error",
            "clocks", "gpu_launches", "eager")
    out = {k: line[k] for k in keys if k in line}
    if isinstance(out.get("roofline"), dict):
        out["roofline"] = {k: v for k, v in out["roofline"].items()
                           if k in ("bound", "achieved", "peak", "unit", "frac", "traffic", "implementation",
                                    "kernel", "peak_source")}
    return out


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and not args.profile:
        cpu = CpuBaseline()  # spawned before any CUDA call
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=dev)
    if args.profile:
        profile_small(dev, args.profile, args.profile_rows, args.tpp or 32)
        return
    cfg, cells, times, extra = run_workload(args.workload, args, dev, world)
    line = None
    if rank == 0:
        cpu_b = None
        if cpu is not None and args.workload in ("ks_plain", "burgers_plain"):
            v, desc, _ = cpu.sample(args.workload, cfg, args.cpu_seconds)
            cpu_b = {"value": v, "unit": "cell-steps/s", "cores": cpu.cores, "kind": "port", "sample": desc}
        if cpu is not None:
            cpu.close()
        if args.workload in ("burgers_diff", "ks_diff"):
            line = diff_line(args, world, cfg, cells, times, extra)
        else:
            line = plain_line(args, world, cfg, cells, times, extra, cpu_b)
    # The default run also measures the other configurations, each as a compact block of
    # the headline line (fewer timed repeats; every rank runs every block).
    if args.workload == "ks_plain" and not args.no_extra:
        sub = copy.copy(args)
        sub.steps, sub.warmup = max(2, min(args.steps, args.extra_steps)), max(3, min(args.warmup, 3))
        blocks = {}
        for name in EXTRA_WORKLOADS:
            c, n, t, e = run_workload(name, sub, dev, world)
            if rank == 0:
                full = (diff_line(sub, world, c, n, t, e) if name in ("burgers_diff", "ks_diff")
                        else plain_line(sub, world, c, n, t, e, None))
                blocks[name] = compact_block(full)
        if rank == 0:
            blocks["burgers_adaptive"] = bench_adaptive(dev)
            line["configs"] = blocks
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def profile_small(dev, which="ks", rows=1024, tpp=32):
    """Small cases for ncu captures: the KS fused rollout (rows x 256, 64 steps, `tpp` threads
    per row pair) and its backward, the ragged Burgers batch (rows of n in {64..512}, 20 steps),
    the 32x128 Burgers rollout, the fused CNN rollout, or one FNO spectral layer (512 x 64 x 512)."""
    import torch
    from types import SimpleNamespace
    if which == "adaptive":  # one adaptive-CFL step of 4096 x 256 rows (about 20 substeps)
        bench_adaptive(dev, reps=2)
        torch.cuda.synchronize()
        return
    if which == "burgers_ragged":
        from inc_b200.batched import RaggedBurgers
        from inc_b200.workloads import burgers_batched_config
        cfg = burgers_batched_config(rows=rows, steps=20)
        rb = RaggedBurgers(cfg["u0"], cfg["nu"], cfg["dt"], cfg["dx"], scheme="ssprk3", device=dev)
        for _ in range(2):
            rb.rollout(20)
        torch.cuda.synchronize()
        return
    if which == "burgers_cnn":  # fused CNN-corrected rollout and its backward (256 x 256, 32 steps)
        import math
        from inc_b200.correctors import PeriodicCNN1D
        from inc_b200.fused import burgers_cnn_rollout
        from inc_b200.solvers import BurgersSolverTorch
        B = N = 256
        sp = SimpleNamespace(resolution=N, dt=0.01, x=None, adaptive_CFL=None, L=2 * math.pi, nu=0.01, device=dev,
                             convection_term="WENO", equation_type="viscosity", batch_size=B, time_scheme="ssprk3")
        solver = BurgersSolverTorch(sp)
        torch.manual_seed(0)
        net = PeriodicCNN1D().to(dev)
        u0 = 0.5 * torch.randn(B, N, device=dev)
        for _ in range(2):
            f, c = burgers_cnn_rollout(net, solver, u0, 32, ckpt_every=8)
            (f.square().mean() + c.square().mean()).backward()
        torch.cuda.synchronize()
        return
    if which == "spectral_conv":  # one FNO layer sum, forward and backward, at the KS FNO's shape
        from inc_b200.correctors import spectral_conv1d
        B, W, N, M = 512, 64, 512, 16
        g = torch.Generator(device=dev).manual_seed(0)
        x = torch.randn(B, W, N, device=dev, generator=g, requires_grad=True)
        add = torch.randn(B, W, N, device=dev, generator=g, requires_grad=True)
        w_re = (torch.rand(W, W, M, device=dev, generator=g) / (W * W)).requires_grad_(True)
        w_im = (torch.rand(W, W, M, device=dev, generator=g) / (W * W)).requires_grad_(True)
        bias = torch.randn(W, device=dev, generator=g, requires_grad=True)
        gy = torch.randn(B, W, N, device=dev, generator=g)
        for _ in range(2):
            spectral_conv1d(x, w_re, w_im, M, bias=bias, addend=add).backward(gy)
        torch.cuda.synchronize()
        return
    if which == "burgers_plain_bwd":  # the same rollout differentiated (checkpoints every 8 steps)
        from inc_b200.rollout import burgers_rollout
        from inc_b200.solvers import BurgersSolverTorch
        from inc_b200.workloads import burgers_plain_config
        cfg = burgers_plain_config()
        sp = SimpleNamespace(resolution=cfg["N"], dt=cfg["dt"], x=None, adaptive_CFL=None, L=cfg["L"], nu=cfg["nu"],
                             device=dev, convection_term="WENO", equation_type="viscosity", batch_size=cfg["B"],
                             time_scheme="ssprk3", cells_per_thread=1)
        u0 = torch.tensor(cfg["u0"], dtype=torch.float32, device=dev)
        for _ in range(2):
            u = u0.clone().requires_grad_(True)
            burgers_rollout(BurgersSolverTorch(sp), u, cfg["steps"], ckpt_every=8).square().mean().backward()
        torch.cuda.synchronize()
        return
    if which == "burgers_plain":
        from inc_b200.rollout import burgers_rollout
        from inc_b200.solvers import BurgersSolverTorch
        from inc_b200.workloads import burgers_plain_config
        cfg = burgers_plain_config()
        sp = SimpleNamespace(resolution=cfg["N"], dt=cfg["dt"], x=None, adaptive_CFL=None, L=cfg["L"], nu=cfg["nu"],
                             device=dev, convection_term="WENO", equation_type="viscosity", batch_size=cfg["B"],
                             time_scheme="ssprk3", cells_per_thread=1)
        u0 = torch.tensor(cfg["u0"], dtype=torch.float32, device=dev)
        with torch.no_grad():
            for _ in range(2):
                burgers_rollout(BurgersSolverTorch(sp), u0, cfg["steps"])
        torch.cuda.synchronize()
        return
    from inc_b200.solvers import KSSolverTorch
    from inc_b200.workloads import ks_plain_config
    cfg = ks_plain_config(B=rows, steps=64)
    B, N = cfg["B"], cfg["N"]
    ds = torch.full((B,), cfg["L"], device=dev)
    solver = KSSolverTorch(SimpleNamespace(resolution=N, dt=cfg["dt"], device=dev, domain_size=ds,
                                           alpha=torch.zeros(B, device=dev), time_scheme="ETRK2",
                                           threads_per_pair=tpp))
    u0 = torch.tensor(cfg["u0"], dtype=torch.float32, device=dev)
    s = torch.tensor(cfg["s"], dtype=torch.float32, device=dev)
    plan = solver.plan_for(u0, ds)
    frames = torch.empty(B, cfg["steps"], N, device=dev)
    if which == "ks_tape":  # the tape rollout and its backward (no replay)
        tape = torch.empty(plan.tape_size(cfg["steps"]), dtype=torch.uint8, device=dev)
        g = torch.randn(B, cfg["steps"], N, device=dev)
        gu, gs = torch.empty_like(u0), torch.empty_like(u0)
        for _ in range(2):
            plan.rollout_tape(u0, s, cfg["steps"], frames, None, tape)
            plan.rollout_bwd_tape(tape, s, cfg["steps"], g, None, gu, gs)
        torch.cuda.synchronize()
        return
    if which == "ks_bwd":
        K = 8
        ck = torch.empty(B, (cfg["steps"] + K - 1) // K, N, device=dev)
        g = torch.randn(B, cfg["steps"], N, device=dev)
        gu, gs = torch.empty_like(u0), torch.empty_like(u0)
        for _ in range(2):
            plan.rollout(u0, s, cfg["steps"], frames, None, K, ck)
            plan.rollout_bwd(ck, s, cfg["steps"], K, g, None, gu, gs)
        torch.cuda.synchronize()
        return
    for _ in range(2):
        plan.rollout(u0, s, cfg["steps"], frames, None, 0, None)
    u = torch.empty_like(u0)
    plan.step(u0, s, None, u)
    torch.cuda.synchronize()


if __name__ == "__main__":
    main()
