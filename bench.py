#!/usr/bin/env python3
"""Benchmark: 2D Euler cell-updates/s of WENO5-SR (FP32 closure) and WENO5-JS on B200.

Workload: unit square, nx = ny = 2000 (3 ghost cells), gamma 1.4, transmissive boundaries, HLLC, SSPRK3,
CFL 0.4. Initial data: seeded four-quadrant Riemann problem (seed 0; rho in [0.5, 2], u, v in [-1, 1],
p in [0.1, 1.5]) advanced with WENO5-JS, untimed, to t0 = 0.125 (the middle of the t = 0.25 run), so
that the timed steps see the run's typical mix of plateau and non-plateau stencils. A step is one
full SSPRK3 time step (3 stages) over the whole grid; cell-updates/s = nx*ny*steps/time.

One JSON line on rank 0. Multi-GPU (torchrun): every rank advances its own replica of the workload
(weak scaling; the step has no cross-replica exchange), timed as the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--method sr_f32|sr_f64|js]

Secondary workloads (--workload):
  adv1d   4096 independent periodic 1D advection trajectories, N ~ U{100..1000}, a = +-1, distance
          ~ {2, 8, 64, 128, 256, 512, 1024} cells at CFL 0.5, seeded profile families; WENO5-SR + SSPRK3
          (--scheme 5) or WENO7-SR + Shu RK4 (--scheme 7). A step is one pass over the whole batch;
          metric: cell-steps/s = sum_i N_i steps_i / time.
  train1d closure training: one step is one forward + adjoint over B = 1024 trajectories of N = 256 cells
          at one distance, the K timed steps walking the shuffled distance cycle; metric: trajectory
          cell-steps/s (B N steps per training step / time).
  euler3d 3D shock-bubble interaction, 224x88x88 on [0,2.545]x[0,1]^2, planar shock of seeded Mach number in
          [2,3] (seed 0) into gas at rest holding a sphere of radius 0.25 with seeded density ratio in [0.1,0.3],
          post-shock inflow at x = 0, transmissive elsewhere; WENO5-SR (FP32 closure by default), HLLC,
          SSPRK3, CFL 0.4. A step is one time step from the initial state; metric: cell-updates/s.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "2D Euler cell-updates/s, WENO5-SR vs WENO5-JS on 1 B200 at matched L1 error"
UNIT = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="sr_f32", choices=["sr_f32", "sr_f64", "sr_bf16", "sr_bf16_tc", "js", "z"],
                    help="sr_bf16_tc: the BF16 closure's MLP on the tensor cores (2D step only); z: WENO5-Z "
                         "(3D step only)")
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--t0", type=float, default=0.125)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--skip-extras", action="store_true", help="no JS arm, e2e, CPU baseline (profiling runs)")
    ap.add_argument("--workload", default="euler2d", choices=["euler2d", "adv1d", "train1d", "euler3d", "euler2d_w7"],
                    help="euler2d: the headline 2D step; adv1d: 4096 ragged 1D trajectories; train1d: closure "
                         "training steps (B=1024, N=256); euler3d: the 224x88x88 shock-bubble step")
    ap.add_argument("--scheme", type=int, default=5, choices=[5, 7], help="adv1d: WENO5/SSPRK3 or WENO7/Shu RK4")
    ap.add_argument("--decomp", default="auto", choices=["auto", "slabs", "replicas"],
                    help="euler2d on N ranks: slabs = the one n x n grid cut into y-slabs with a 3-row halo "
                         "exchange per stage and a MAX all-reduce per step (strong scaling); replicas = N "
                         "independent copies (weak scaling); auto = slabs when N > 1")
    ap.add_argument("--w7-method", default="js", choices=["js", "z", "sr_f64"],
                    help="euler2d_w7: WENO7-JS, WENO7-Z or WENO7-SR (FP64 closure)")
    return ap.parse_args()


def workload_config(args, n_gpus):
    return {"workload": f"2D Euler quadrant Riemann problem {args.n}x{args.n}, seed 0, state at t0={args.t0}",
            "grid": [args.n, args.n], "ghost": 3, "gamma": 1.4, "cfl": 0.4, "boundary": "transmissive",
            "flux": "hllc", "time_integrator": "SSPRK3", "method": args.method,
            "closure_precision": {"sr_f32": "fp32", "sr_f64": "fp64", "sr_bf16": "bf16", "sr_bf16_tc": "bf16",
                                  "js": None}[args.method],
            "state_precision": "fp64", "l2_policy": "inputs larger than L2 (state 4 x 129 MB + 0.8 GB workspace)",
            "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU"}


def initial_state(n):
    from weno_sr_publishing_b200 import problems
    # the quadrant interfaces at x = y = 0.5 fall on cell edges for even n, so every cell average is a
    # single state and the midpoint rule is exact
    return problems.make_quadrant_state(n, n, problems.seeded_quadrant_states(0), quadrature=1)


CPU_SAMPLE_N = 256


def cpu_sample_state(t0):
    """The CPU-feasible sample of the benchmark workload: the same seeded quadrant problem on a 256 x 256 grid
    of the whole unit square, advanced (untimed) to t0 with the oracle's WENO5-JS, so that it holds the same
    waves as the 2000^2 state at t0 (a 2000^2 state at t0 takes thousands of 2000^2 steps, out of reach of
    the CPU)."""
    from oracle import oracle as O
    from weno_sr_publishing_b200 import problems
    m = CPU_SAMPLE_N
    init = problems.make_quadrant_state(m, m, problems.seeded_quadrant_states(0), quadrature=1)
    state, _, _, _ = O.euler2d_run(init, m, m, 1.0 / m, 1.0 / m, 0.4, t0, "js", "transmissive", fast=True)
    return state


def cpu_steps(state, method, mlp, steps):
    """Wall time of `steps` full SSPRK3 steps of the C oracle (OpenMP, all host threads) on the sample state."""
    from oracle import oracle as O
    m = CPU_SAMPLE_N
    t0 = time.perf_counter()
    for _ in range(steps):
        O.euler2d_run(state, m, m, 1.0 / m, 1.0 / m, 0.4, 1.0, method, "transmissive", params=mlp, fixed_steps=1,
                      fast=True)
    return time.perf_counter() - t0


def cpu_sample(method, mlp, t0, budget_s):
    """The repo arm's CPU baseline: the reference arm's sample and timing, for as many steps as fit the budget."""
    from oracle import oracle as O
    m = CPU_SAMPLE_N
    state = cpu_sample_state(t0)
    cpu_steps(state, method, mlp, 1)
    steps, el = 0, 0.0
    while el < budget_s and steps < 200:
        el += cpu_steps(state, method, mlp, 1)
        steps += 1
    return {"value": m * m * steps / el, "unit": UNIT, "cores": O.num_threads(True), "kind": "port",
            "sample": f"{steps} step(s) of the same seeded problem on a {m}x{m} grid of the whole unit square at "
                      f"t0={t0} (C oracle, OpenMP, -O3), {el:.1f} s; the sample bench.py --impl reference times"}


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference(args, rank):
    """The reference's CPU counterpart of the 2D step: the reference has no CPU path for 2D Euler (its Warp
    GPU kernels only, and warp-lang is not installed), so its algorithm runs as the C restatement in oracle/
    (a port), timed on all host threads. A step is one full SSPRK3 step of the CPU-feasible sample of the
    benchmark workload (cpu_sample_state: the same problem on a 256^2 grid at t0), W untimed and K timed; the
    line's config names that grid, and ms_per_step is the measured time of one sample step."""
    if rank != 0:
        return
    from oracle import oracle as O
    from weno_sr_publishing_b200.checkpoint import MODELS_DIR
    mlp = None
    if args.method != "js":
        name = "weno5_sr_fp64_step012250.npz" if args.method == "sr_f64" else "weno5_sr_fp32_step016500.npz"
        mlp = {k: v for k, v in np.load(MODELS_DIR / name).items() if k != "meta_json"}
    m = CPU_SAMPLE_N
    state = cpu_sample_state(args.t0)
    cpu_steps(state, args.method, mlp, max(args.warmup, 0))
    el = cpu_steps(state, args.method, mlp, args.steps)
    v = m * m * args.steps / el
    cfg = workload_config(args, args.gpus)
    cfg["workload"] = (f"2D Euler quadrant Riemann problem, seed 0, on a {m}x{m} grid of the unit square at "
                       f"t0={args.t0}: the CPU-feasible sample of the {args.n}x{args.n} workload")
    cfg["grid"] = [m, m]
    cfg["sample_of"] = workload_config(args, args.gpus)["workload"]
    cfg["l2_policy"] = "CPU run: state 4 x 2.1 MB"
    base = {"value": v, "unit": UNIT, "cores": O.num_threads(True), "kind": "port",
            "sample": f"{args.steps} steps (after {args.warmup} untimed) of the same problem on a {m}x{m} grid at "
                      f"t0={args.t0} (C oracle, OpenMP, -O3), {el:.1f} s"}
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg, "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.method == "z" and args.workload != "euler3d":
        raise SystemExit("--method z is for --workload euler3d")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "euler3d":
        bench_3d(args, world, rank, local)
        return
    if args.workload == "euler2d_w7":
        bench_w7(args, world, rank, local)
        return
    if args.workload != "euler2d":
        bench_1d(args, world, rank, local)
        return
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist

    from weno_sr_publishing_b200 import _native as N
    from weno_sr_publishing_b200 import euler2d as E
    from weno_sr_publishing_b200 import roofline as R
    from weno_sr_publishing_b200.checkpoint import MODELS_DIR
    from weno_sr_publishing_b200.params import Params

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    slabs = args.decomp == "slabs" or (args.decomp == "auto" and world > 1)
    if world > 1 or slabs:
        import datetime
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev, rank=rank,
                                world_size=world)
    n, K, W = args.n, args.steps, max(args.warmup, 0)
    p = Params(nx=n, ny=n, x_length=1.0, y_length=1.0, cfl=0.4)
    mlp = None
    if args.method != "js":
        name = "weno5_sr_fp64_step012250.npz" if args.method == "sr_f64" else "weno5_sr_fp32_step016500.npz"
        mlp = {k: v for k, v in np.load(MODELS_DIR / name).items() if k != "meta_json"}
    ws = E.workspace(n, n, dev)
    bufs = [torch.zeros(p.padded_shape, dtype=torch.float64, device=dev) for _ in range(4)]
    bufs[0].copy_(torch.from_numpy(initial_state(n)))
    res = E.run(bufs, p, args.t0, "js", "transmissive", ws=ws)  # untimed: advance to t0
    start = bufs[res.final_slot].clone()
    ctx = N.context(local)
    stream = torch.cuda.current_stream(dev)

    def timed(method, prm, steps, warm):
        bufs[0].copy_(start)
        if warm:
            r = E.run(bufs, p, 1.0, method, "transmissive", mlp_params=prm, fixed_steps=warm, ws=ws)
            if r.final_slot == 3:
                bufs[0].copy_(bufs[3])
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = E.run(bufs, p, 1.0, method, "transmissive", mlp_params=prm, fixed_steps=steps, ws=ws)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, r

    if slabs:
        from weno_sr_publishing_b200 import slabs as S
        sp = S.slab_params(p, world, rank)
        comm = S.DistSlabs()

        def timed_slabs(method, prm, steps, warm):
            stages = S.CudaStages(method, prm)
            slab = S.split(start, p, world, rank)
            if warm:
                slab = S.run([slab], [sp], 1.0e30, "transmissive", comm, stages, max_steps=warm).slabs[0]
            dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = S.run([slab], [sp], 1.0e30, "transmissive", comm, stages, max_steps=steps)
            e1.record(stream)
            torch.cuda.synchronize()
            t = torch.tensor([e0.elapsed_time(e1)], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item()), r

    with ClockSampler(local) as clk:
        ms, r = timed_slabs(args.method, mlp, K, W) if slabs else timed(args.method, mlp, K, W)
    clocks = clk.summary()
    units = n * n if slabs else world * n * n  # slabs: the one grid's cell updates (strong scaling)
    value = units * K / (ms * 1e-3)
    cfg = workload_config(args, world)
    if slabs:
        cfg["parallelism"] = (f"y-slabs x{world}: rank r owns rows of the one {n}x{n} grid, 3-row halo exchange "
                              f"per stage (NCCL send/recv), MAX all-reduce of the wave speed per step")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong" if slabs else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg, "clocks": clocks}
    # device loop, per step: dt kernels (2), 3 stages x 5 kernels, t/steps update (1); plus init and max speed.
    # slabs, per step: max speed (1), 3 stages x (control init + 5 kernels)
    line["gpu_launches"] = K * (1 + 3 * 6) if slabs else 2 + K * (3 + 3 * 5)

    if not args.skip_extras:
        # WENO5-JS on the same state and steps: the cost ratio of the learned closure
        ms_js, _ = timed_slabs("js", None, K, W) if slabs else timed("js", None, K, W)
        line["js"] = {"value": units * K / (ms_js * 1e-3), "ms_per_step": ms_js / K,
                      "sr_over_js_cost": (ms / K) / (ms_js / K)}

    # per-kernel device time (CUDA events around each launch) and closure tallies for the roofline
    bufs[0].copy_(start)
    E.run(bufs, p, 1.0, args.method, "transmissive", mlp_params=mlp, fixed_steps=1, opts=N.OPT_COUNT, ws=ws)
    tallies = E.counters(ws)
    ctx.profile_enable(True)
    bufs[0].copy_(start)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()  # ncu --profile-from-start off captures these launches only
    E.run(bufs, p, 1.0, args.method, "transmissive", mlp_params=mlp, fixed_steps=K, ws=ws)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    prof = ctx.profile_read()
    ctx.profile_enable(False)
    peak32 = ctx.peak_tflops(32, C_stream(stream))
    peak64 = ctx.peak_tflops(64, C_stream(stream))
    hbm = hbm_peak()
    kinds = ["normal_x", "normal_y", "flux_x", "flux_y", "update"]
    per_kernel = {}
    for k in kinds:
        tot_ms, cnt = prof[k]
        if cnt == 0:
            continue
        mlp_n, plat_n = tallies.get(k, (0, 0))
        # tallies cover one step = 3 launches of each reconstruction kernel
        work = R.kernel_work(k, args.method, n, n, mlp_n / 3.0, plat_n / 3.0)
        per_kernel[k] = {"ms_per_launch": tot_ms / cnt, "launches": cnt, "share": None,
                         **R.bound(work, tot_ms / cnt * 1e-3, peak32, peak64, hbm["gbs"])}
    tot = sum(v["ms_per_launch"] * v["launches"] for v in per_kernel.values())
    for v in per_kernel.values():
        v["share"] = v["ms_per_launch"] * v["launches"] / tot
    dom = max(per_kernel, key=lambda k: per_kernel[k]["share"])
    d = per_kernel[dom]
    traffic = NCU_TRAFFIC.get((dom, args.method, n))
    line["roofline"] = {"kernel": dom, "bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"],
                        "unit": d["unit"], "frac": d["frac"], "traffic": traffic,
                        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                          "profiles/k_normal_k_flux_sr_f32_2000.md" if traffic else None,
                        "peak_source": {"fp32_tflops": f"measured FMA probe {peak32:.1f}",
                                        "fp64_tflops": f"measured FMA probe {peak64:.1f}",
                                        "hbm_gbs": hbm["source"]}}
    step_work = {"w32": 0.0, "w64": 0.0, "bytes": 0.0}
    for k in kinds:
        if k in per_kernel:
            mlp_n, plat_n = tallies.get(k, (0, 0))
            wk = R.kernel_work(k, args.method, n, n, mlp_n / 3.0, plat_n / 3.0)
            for key in step_work:
                step_work[key] += 3 * wk[key]
    if slabs:  # each rank does its slab's share of the grid's work in the job's step time
        step_work = {k: v / world for k, v in step_work.items()}
    line["roofline_step"] = R.bound(step_work, ms / K * 1e-3, peak32, peak64, hbm["gbs"])
    line["kernels"] = {k: {kk: v[kk] for kk in ("ms_per_launch", "launches", "share", "bound", "frac")}
                       for k, v in per_kernel.items()}
    line["closure_tally_per_step"] = {k: {"mlp": v[0], "plateau": v[1]} for k, v in tallies.items()}
    if not args.skip_extras and not slabs and args.method != "js":
        line["precision_l1"] = precision_block(bufs, start, p, mlp, K, ws)

    if not args.skip_extras and slabs:
        # end to end per rank: pinned host slab -> device, one step of the decomposed grid, device -> host
        stages = S.CudaStages(args.method, mlp)
        host = torch.empty(sp.padded_shape, dtype=torch.float64, pin_memory=True)
        host.copy_(S.split(start, p, world, rank).cpu())
        slab = torch.empty(sp.padded_shape, dtype=torch.float64, device=dev)

        def e2e_step():
            slab.copy_(host, non_blocking=True)
            out = S.run([slab], [sp], 1.0e30, "transmissive", comm, stages, max_steps=1).slabs[0]
            host.copy_(out, non_blocking=True)

        for _ in range(max(W, 1)):
            e2e_step()
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        nbytes = int(np.prod(sp.padded_shape)) * 8
        line["e2e"] = {"value": units * K / (float(t.item()) * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes,
                       "api": "weno_sr_publishing_b200.slabs.run (pinned host slab per rank, 1 step per call)"}
        if rank == 0:
            line["matched_l1"] = matched_l1_block(args.method, mlp, dev)
    elif not args.skip_extras:
        # end to end: pinned host state -> device, one step, device -> pinned host, K times
        host = torch.empty(p.padded_shape, dtype=torch.float64, pin_memory=True)
        host.copy_(start.cpu())
        for _ in range(max(W, 1)):
            E.advance_host(host, p, 1, args.method, "transmissive", mlp_params=mlp, bufs=bufs, ws=ws, device=dev,
                           async_readback=True)
        E.host_wait(dev)  # the warm-up calls' read-backs are done and their steps counted out
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            E.advance_host(host, p, 1, args.method, "transmissive", mlp_params=mlp, bufs=bufs, ws=ws, device=dev,
                           async_readback=True)
        E.host_copies_done(dev)  # the last read-back is inside the timed region
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms_e2e], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e2e = float(t.item())
        host_status = E.host_wait(dev)  # after the timed region: every timed call took its step
        if host_status["steps"] != K:
            raise RuntimeError(f"advance_host took {host_status['steps']} steps in {K} calls")
        nbytes = n * n * 4 * 8  # the interior rows go in and come back; ghost cells are not copied
        line["e2e"] = {"value": world * n * n * K / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes,
                       "api": "weno_sr_publishing_b200.euler2d.advance_host -> wsr_euler2d_advance_host (pinned host "
                              "buffer, 1 step per call, async_readback=True: uploads and read-backs in row bands "
                              "overlapped with the first and last stages; the last read-back completes inside the "
                              "timed region)"}
        if rank == 0 and world == 1:
            line["cpu_baseline"] = cpu_sample(args.method, mlp, args.t0, args.cpu_seconds)
        if rank == 0:
            line["matched_l1"] = matched_l1_block(args.method, mlp, dev)
    if world > 1 or slabs:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def precision_block(bufs, start, p, mlp, steps, ws):
    """Density L1 distance (sum |rho_a - rho_b| dx dy) after the timed steps from the benchmark state between
    the closure evaluated in FP64 and in FP32 / BF16, with the same checkpoint's weights."""
    from weno_sr_publishing_b200 import euler2d as E
    rho = {}
    for m in ("sr_f64", "sr_f32", "sr_bf16"):
        bufs[0].copy_(start)
        r = E.run(bufs, p, 1.0, m, "transmissive", mlp_params=mlp, fixed_steps=steps, ws=ws)
        rho[m] = bufs[r.final_slot][3:3 + p.ny, 3:3 + p.nx, 0].double().cpu().numpy()
    l1 = {m: float(np.abs(rho[m] - rho["sr_f64"]).sum() * p.dx * p.dy) for m in ("sr_f32", "sr_bf16")}
    return {"against": "the same steps with the closure in FP64 (same checkpoint)", "steps": steps,
            "rho_l1": l1, "bound": {"sr_f32": 1e-8, "sr_bf16": 5e-4},
            "within_bound": {"sr_f32": l1["sr_f32"] <= 1e-8, "sr_bf16": l1["sr_bf16"] <= 5e-4}}


def matched_l1_block(method, mlp, dev):
    """The metric's "at matched L1 error", on a smooth and a discontinuous problem: the periodic isentropic
    vortex (the reference's exp 05 setup, [-10,10]^2, t = 2, CFL 0.4) at N = 100..800 against the exact
    solution, and the seeded quadrant problem at N = 100..400 against a 2000^2 WENO5-JS solution; for each
    SR point the JS resolution with the same L1 (log-log interpolation) and both device times to it."""
    from weno_sr_publishing_b200 import accuracy as AC
    ns = (100, 200, 400, 800)
    sr = [AC.vortex_run(n, method, mlp, dev) for n in ns]
    js = [AC.vortex_run(n, "js", None, dev) for n in ns]
    pts = lambda rs: [{"n": r.n, "l1": r.l1, "ms": r.device_ms, "steps": r.steps} for r in rs]  # noqa: E731
    vortex = {"problem": "isentropic vortex [-10,10]^2 periodic, t=2, CFL 0.4, L1(rho) vs exact cell averages",
              "sr": pts(sr), "js": pts(js), "matched": AC.matched_l1(sr[:-1], js)}
    study, ref_ms = AC.quadrant_study(method, mlp, dev)
    quadrant = {"problem": "seeded quadrant Riemann problem (seed 0), t=0.25, CFL 0.4, L1(rho) vs the 2000^2 "
                           "WENO5-JS solution block-averaged", "reference_ms": ref_ms,
                "sr": pts(study[method]), "js": pts(study["js"]),
                "matched": AC.matched_l1(study[method], study["js"])}
    return {"vortex": vortex, "quadrant": quadrant}


DIST_CYCLE = (2, 8, 64, 128, 256, 512, 1024)


def adv1d_batch(seed=0, B=4096):
    """Ragged batch of the 1D inference workload: (initial states, velocities, N, steps)."""
    from weno_sr_publishing_b200 import profiles as P
    rng = np.random.default_rng(seed)
    ns = rng.integers(100, 1001, B)
    dist = rng.choice(np.asarray(DIST_CYCLE), B)
    vel = np.where(rng.random(B) < 0.5, -1.0, 1.0)
    states = [None] * B
    for n in np.unique(ns):
        idx = np.flatnonzero(ns == n)
        desc, _ = P.make_profiles(rng, idx.size, int(n))
        u = P.cell_averages(desc, int(n), 0.0)
        for j, b in enumerate(idx):
            states[b] = u[j]
    return states, vel, ns, 2 * dist


def _closure(scheme, method):
    from weno_sr_publishing_b200 import adv1d as A1
    from weno_sr_publishing_b200.checkpoint import MODELS_DIR
    from weno_sr_publishing_b200._native import pack_params
    if method == "js":
        return "classical"
    name = {5: {"sr_f64": "weno5_sr_fp64_step012250.npz"}, 7: {}}.get(scheme, {}).get(
        method, "weno5_sr_fp32_step016500.npz" if scheme == 5 else "weno7_sr_fp64_step016750.npz")
    data = np.load(MODELS_DIR / name)
    if scheme == 5:
        packed = pack_params({k: data[k] for k in ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")})
    else:
        packed = np.concatenate([data[k].reshape(-1).astype(np.float64) for k in ("w1", "b1", "w2", "b2", "w3", "b3",
                                                                                 "w4", "b4")])
    return A1.Closure(scheme, packed, {"sr_f64": "f64", "sr_f32": "f32", "sr_bf16": "bf16"}[method])


def _adv1d_cpu(states, vel, ns, steps, scheme, closure, budget_s):
    """The oracle (numpy port of the reference's torch stepper) on a bounded sample of trajectories."""
    from oracle import adv1d_oracle as AO
    cl = None if closure == "classical" else (closure.kind, closure.precision, closure.packed)
    integ = "ssprk3" if scheme == 5 else "shu_rk4"
    work, t0, count = 0, time.perf_counter(), 0
    for b in range(len(states)):
        k = 4
        AO.run(states[b], vel[b], 1.0 / ns[b], [0.5 / ns[b]] * k, scheme, cl, integ)
        work += int(ns[b]) * k
        count += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    el = time.perf_counter() - t0
    return {"value": work / el, "unit": "cell-steps/s", "cores": 1, "kind": "port",
            "sample": f"4 steps of each of the first {count} trajectories ({work} cell-steps), numpy oracle, {el:.1f} s"}


def _train_cpu(budget_s):
    """The torch autograd oracle (forward + backward on the CPU) on B = 8 trajectories of N = 256."""
    import torch
    from oracle import train1d_oracle as TO
    from weno_sr_publishing_b200 import profiles as P
    from weno_sr_publishing_b200 import train1d as T1
    rng = np.random.default_rng(5)
    n, B, steps = 256, 8, 8
    desc, _ = P.make_profiles(rng, B, n)
    vel = T1.balanced_velocities(B)
    u0 = P.cell_averages(desc, n, 0.0)
    tg = np.stack([P.cell_averages(desc, n, vel * (k * 0.5 / n)) for k in range(1, steps + 1)], axis=1)
    packed = T1.ClosureMLP(seed=83, dtype=torch.float32).packed().detach().double().numpy()
    reps, t0 = 0, time.perf_counter()
    while True:
        TO.loss_and_grads(packed, u0, tg, vel, 0.5 / n, float(n), "f32")
        reps += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    el = time.perf_counter() - t0
    return {"value": reps * B * n * steps / el, "unit": "cell-steps/s", "cores": torch.get_num_threads(),
            "kind": "port", "sample": f"{reps} forward+backward of B={B}, N={n}, {steps} steps (torch autograd "
                                      f"oracle, FP32 closure), {el:.1f} s"}


def bench_1d(args, world, rank, local):
    import ctypes as C

    import torch
    import torch.distributed as dist
    if args.workload == "adv1d":
        method = args.method
        metric = f"1D batched advection cell-steps/s, WENO{args.scheme}-SR ({method}), 4096 ragged trajectories"
        cfg = {"workload": "4096 periodic 1D advection trajectories, N~U{100..1000}, a=+-1, distance~"
                           "{2,8,64,128,256,512,1024} cells, CFL 0.5, seeded profile families (seed 0)",
               "scheme": f"WENO{args.scheme}", "integrator": "SSPRK3" if args.scheme == 5 else "Shu RK4",
               "method": method, "l2_policy": "the 4096 trajectories stay in shared memory; HBM traffic is the "
                                              "initial and final states only"}
    else:
        method = "sr_f32" if args.method not in ("sr_f32", "sr_f64") else args.method
        metric = f"closure training cell-steps/s (forward + adjoint), WENO5-SR {method}, B=1024, N=256"
        cfg = {"workload": "closure training, B=1024 trajectories of N=256 cells, distances cycling through "
                           "{2,8,64,128,256,512,1024} cells at CFL 0.5, checkpoint every 32 steps",
               "method": method, "loss": "mean L1 to exact cell averages at every completed step",
               "l2_policy": "inputs larger than L2 for the long distances (checkpoints + stage scratch)"}
    cfg["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
    if args.workload == "adv1d" and world > 1:
        cfg["parallelism"] = (f"sharded x{world}: 4096 x {world} seeded trajectories, each rank its cost-balanced "
                              f"share (cells x steps, longest first), no data-path collective")
    if args.workload == "train1d" and world > 1:
        cfg["parallelism"] = f"data parallel x{world}: each rank its own 1024 trajectories, gradient all-reduce"
    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload == "adv1d":
            st, vel, ns, steps = adv1d_batch()
            base = _adv1d_cpu(st, vel, ns, steps, args.scheme, _closure(args.scheme, method), args.cpu_seconds)
        else:
            base = _train_cpu(args.cpu_seconds)
        line = {"metric": metric, "value": base["value"], "unit": base["unit"], "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "impl": "reference", "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": base["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    from weno_sr_publishing_b200 import _native as N
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    stream = torch.cuda.current_stream(dev)
    K, W = args.steps, max(args.warmup, 0)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def max_over_ranks(ms):
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return ms

    line = {"metric": metric, "unit": "cell-steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg}
    if args.workload == "adv1d":
        from weno_sr_publishing_b200 import adv1d as A1
        states, vel, ns, steps = adv1d_batch(B=4096 * world)
        if world > 1:  # this rank's cost-balanced share of the 4096 x world trajectories
            mine = A1.shard_by_cost(ns * steps, world, rank)
            states, vel, ns, steps = [states[b] for b in mine], vel[mine], ns[mine], steps[mine]
        closure = _closure(args.scheme, method)
        cl = A1.as_closure(closure)
        ctx = N.context(local)
        if cl is not None:
            ctx.upload_closure_kind(cl.kind, cl.packed)
        B = len(states)
        flat0 = torch.as_tensor(np.concatenate(states), device=dev)
        flat = flat0.clone()
        offs = torch.as_tensor(np.concatenate([[0], np.cumsum(ns)]), dtype=torch.int64, device=dev)
        cost = ns * steps
        order = torch.as_tensor(np.argsort(-cost, kind="stable").astype(np.int32), device=dev)
        velt = torch.as_tensor(vel, device=dev)
        dxs = torch.as_tensor(1.0 / ns, device=dev)
        nf = torch.as_tensor(steps.astype(np.int32), device=dev)
        dtf = torch.as_tensor(0.5 / ns, device=dev)
        dtl = torch.zeros(B, dtype=torch.float64, device=dev)
        wsb = int(N.lib().wsr_adv1d_workspace_bytes())
        ws = torch.zeros(wsb + 256, dtype=torch.uint8, device=dev)
        wp = (ws.data_ptr() + 255) // 256 * 256
        P_ = C.c_void_p
        meth = N.METHOD[method]
        integ = 0 if args.scheme == 5 else 1
        cnt = (C.c_ulonglong * 2)()

        def launch(opts=0, counters=None):
            ctx.check(N.lib().wsr_adv1d_run(ctx.handle, P_(flat.data_ptr()), P_(offs.data_ptr()),
                                            P_(order.data_ptr()), P_(velt.data_ptr()), P_(dxs.data_ptr()),
                                            P_(nf.data_ptr()), P_(dtf.data_ptr()), P_(dtl.data_ptr()), B,
                                            int(ns.max()), args.scheme, meth, integ, opts, None, None, counters,
                                            P_(wp), wsb, P_(stream.cuda_stream)))
        for _ in range(W):
            flat.copy_(flat0)
            launch()
        ms = 0.0
        with ClockSampler(local) as clk:
            for _ in range(K):
                flat.copy_(flat0)
                if world > 1:
                    dist.barrier()
                torch.cuda.synchronize()
                e0, e1 = ev(), ev()
                e0.record(stream)
                launch()
                e1.record(stream)
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
        ms = max_over_ranks(ms)
        work = float(np.sum(ns * steps))
        total = work
        if world > 1:  # the cell-steps of all shards
            t = torch.tensor([work], dtype=torch.float64, device=dev)
            dist.all_reduce(t)
            total = float(t.item())
        line.update({"value": total * K / (ms * 1e-3), "ms_per_step": ms / K, "clocks": clk.summary(),
                     "gpu_launches": K})
        flat.copy_(flat0)
        launch(N.OPT_COUNT, cnt)
        mlp_n, plat_n = int(cnt[0]), int(cnt[1])
        line["closure_tally_per_step"] = {"mlp": mlp_n, "plateau": plat_n}
        # end to end through the public API: host arrays in, host arrays out, every step
        integ_name = "ssprk3" if args.scheme == 5 else "shu_rk4"
        A1.run_batched(states, vel, 1.0 / ns, steps, 0.5 / ns, scheme=args.scheme, model=closure,
                       integrator=integ_name, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            outs, _ = A1.run_batched(states, vel, 1.0 / ns, steps, 0.5 / ns, scheme=args.scheme, model=closure,
                                     integrator=integ_name, device=dev, to_host=True)
        el = time.perf_counter() - t0
        nbytes = int(np.sum(ns)) * 8
        el = max_over_ranks(el * 1e3) * 1e-3
        line["e2e"] = {"value": total * K / el, "unit": "cell-steps/s", "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes,
                       "api": "weno_sr_publishing_b200.adv1d.run_batched (host arrays in, to_host=True: one upload and "
                              "one read-back of the whole batch)"}
        peak = ctx.peak_tflops(32 if method in ("sr_f32", "sr_bf16") else 64, C_stream(stream))
        line["roofline"] = _roofline_1d(args.scheme, method, work, mlp_n, plat_n, ms / K, peak, ctx, stream)
        if rank == 0 and world == 1:
            line["cpu_baseline"] = _adv1d_cpu(states, vel, ns, steps, args.scheme, closure, args.cpu_seconds)
    else:
        from weno_sr_publishing_b200 import profiles as P1
        from weno_sr_publishing_b200 import train1d as T1
        rng = np.random.default_rng(83)
        prec = "f32" if method == "sr_f32" else "f64"
        model = T1.ClosureMLP(seed=83, dtype=torch.float32 if prec == "f32" else torch.float64)
        with torch.no_grad():
            g = torch.Generator().manual_seed(1)
            for k in T1.PARAM_NAMES:
                getattr(model, k).add_((0.2 * torch.randn(getattr(model, k).shape, generator=g,
                                                          dtype=torch.float64)).to(getattr(model, k).dtype))
        packed = model.packed().detach().double().numpy()
        order = [DIST_CYCLE[T1.distance_index_for_step(s, 7, 83)] for s in range(1, K + W + 1)]
        batches = [T1.TrajectoryBatch.sample(rng, 1024, 256, d, 0.5, dev, 32) for d in order]
        ms, work, fwd_ms, bwd_ms = 0.0, 0.0, 0.0, 0.0
        for b in batches[:W]:
            r = T1._Run(b, packed, prec)
            r.forward()
            r.backward()
        with ClockSampler(local) as clk:
            for b in batches[W:]:
                r = T1._Run(b, packed, prec)
                if world > 1:
                    dist.barrier()
                torch.cuda.synchronize()
                e0, e1, e2 = ev(), ev(), ev()
                e0.record(stream)
                r.forward()
                e1.record(stream)
                g, _ = r.backward()
                if world > 1:
                    dist.all_reduce(g)  # data parallelism: the 189 gradient values summed over ranks
                e2.record(stream)
                torch.cuda.synchronize()
                fwd_ms += e0.elapsed_time(e1)
                bwd_ms += e1.elapsed_time(e2)
                work += b.B * b.n * b.steps
        ms = max_over_ranks(fwd_ms + bwd_ms)
        line.update({"value": world * work / (ms * 1e-3), "ms_per_step": ms / K, "clocks": clk.summary(),
                     "gpu_launches": 4 * K, "forward_ms": fwd_ms, "backward_ms": bwd_ms,
                     "distances": [int(d) for d in order[W:]]})
        # closure tallies of the timed forwards: the training forward equals the 1D batch path bit for bit, so
        # the batch path with its counters on the same initial states and steps counts its closure evaluations
        from weno_sr_publishing_b200 import adv1d as A1
        cl = A1.Closure(5, packed, prec)
        mlp_n = plat_n = 0
        for b in batches[W:]:
            u0 = P1.cell_averages(b.desc.cpu().numpy(), b.n, 0.0)
            _, info = A1.run_batched(list(u0), b.velocity.cpu().numpy(), 1.0 / b.n, b.steps, b.dt, scheme=5,
                                     model=cl, device=dev, count=True)
            mlp_n += info["mlp"]
            plat_n += info["plateau"]
        # forward, its recomputation from the checkpoints, and a reverse pass of twice the forward's work
        line["roofline"] = _closure_roofline(
            "k_train_fwd + k_train_bwd (4 x the counted forward closure work)", method,
            [(4.0 * mlp_n / K, 4.0 * plat_n / K, 1)], ms / K, local, stream)
        # end to end through the autograd API: host profile descriptors in, host loss and gradient out
        t0 = time.perf_counter()
        for d in order[W:]:
            desc, _ = P1.make_profiles(rng, 1024, 256)
            b = T1.TrajectoryBatch(torch.as_tensor(desc).to(dev, non_blocking=True),
                                   torch.as_tensor(T1.balanced_velocities(1024)).to(dev), 256,
                                   T1.steps_for_distance(d, 0.5), 0.5 / 256)
            model.zero_grad(set_to_none=True)
            loss = T1.trajectory_loss(model.to(dev), b)
            loss.backward()
            _ = float(loss.detach()), model.w1.grad.cpu()
        el = time.perf_counter() - t0
        line["e2e"] = {"value": world * work / el, "unit": "cell-steps/s", "h2d_bytes_per_step": 1024 * 34 * 8 + 8192,
                       "d2h_bytes_per_step": 8 + 189 * 8,
                       "api": "weno_sr_publishing_b200.train1d.trajectory_loss(...).backward() with host profiles"}
        if rank == 0 and world == 1:
            line["cpu_baseline"] = _train_cpu(args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _oracle3d_sample(sb_seed, method, params, budget_s):
    """The 3D C oracle (OpenMP, all host threads) on the same problem at a quarter of the resolution."""
    from oracle import oracle as O
    from weno_sr_publishing_b200 import problems as PR
    sb = PR.ShockBubble.seeded(sb_seed, 56, 22, 22)
    q0 = sb.state()
    dx, dy, dz = sb.spacing
    steps, t0, q = 0, time.perf_counter(), q0
    while True:
        q, _ = O.euler3d_run(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, 1, method, "hllc", params, inflow=sb.inflow(),
                             fast=True)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or steps >= 20:
            break
    cells = sb.nx * sb.ny * sb.nz
    return {"value": cells * steps / el, "unit": UNIT, "cores": O.num_threads(True), "kind": "port",
            "sample": f"{steps} step(s) of the same problem on 56x22x22 from t=0 (C oracle, OpenMP), {el:.1f} s"}


def bench_w7(args, world, rank, local):
    """WENO7 2D (JS, Z or SR-FP64 weights, --w7-method) with Shu RK4 on the periodic isentropic vortex (the
    reference's point_rk4 / point_rk4_z / point_rk4_mlp paths) at args.n^2 (default 1024 when the 2D default
    2000 is given), K steps from t = 0."""
    import torch
    import torch.distributed as dist

    from oracle import oracle as O
    from weno_sr_publishing_b200 import euler2d_w7 as E7
    from weno_sr_publishing_b200 import problems as PR
    n = 1024 if args.n == 2000 else args.n
    method = args.w7_method
    label = {"js": "WENO7-JS", "z": "WENO7-Z", "sr_f64": "WENO7-SR (FP64 closure)"}[method]
    closure = params = None
    if method == "sr_f64":
        from weno_sr_publishing_b200.checkpoint import MODELS_DIR
        params = {k: v for k, v in np.load(MODELS_DIR / "weno7_sr_fp64_step016750.npz").items() if k != "meta_json"}
        closure = params
    metric = f"2D Euler cell-updates/s, {label} Shu RK4, {n}x{n} isentropic vortex"
    cfg = {"workload": f"2D periodic isentropic vortex {n}x{n} on [-10,10]^2 (2x2 Gauss averages), from t=0",
           "scheme": f"{label} characteristic + two-point Gauss transverse", "flux": "hllc",
           "time_integrator": "Shu RK4 (L and L~)", "cfl": 0.4, "state_precision": "fp64",
           "l2_policy": f"state {(n + 8) ** 2 * 32 / 1e6:.0f} MB, workspace {(n * n * 32 * 14) / 1e6:.0f} MB",
           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
    init = PR.vortex_point_rk4(n, n, 0.0, 2)
    K, W = args.steps, max(args.warmup, 0)

    def cpu_sample():
        m = 64
        small = PR.vortex_point_rk4(m, m, 0.0, 2)
        pm = E7.Params(nx=m, ny=m)
        steps, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < args.cpu_seconds:
            _, _, k, _ = O.w7_run(small, m, m, pm.dx, pm.dy, 0.4, 100.0, "periodic", max_steps=1, fast=True,
                                  method=method, params=params)
            steps += k
        el = time.perf_counter() - t0
        return {"value": m * m * steps / el, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                "sample": f"{steps} step(s) of the same problem on {m}x{m} (C oracle, OpenMP), {el:.1f} s"}

    if args.impl == "reference":
        if rank != 0:
            return
        base = cpu_sample()
        print(json.dumps({"metric": metric, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                          "impl": "reference", "cpu_baseline": base,
                          "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    p = E7.Params(nx=n, ny=n, cfl=0.4, t_end=1.0e30)
    u0 = torch.as_tensor(init, device=dev).contiguous()
    ws = E7.workspace(n, n, dev)
    u = u0.clone()
    if W:
        E7.run(u, p, "periodic", max_steps=W, ws=ws, method=method, closure=closure)
    u.copy_(u0)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        res = E7.run(u, p, "periodic", max_steps=K, ws=ws, method=method, closure=closure)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    counts = E7.closure_counts(ws, p) if method == "sr_f64" else None
    if counts is not None:
        counts.pop("fallbacks")
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    line = {"metric": metric, "value": world * n * n * res.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": res.steps, "warmup": W, "ms_per_step": ms / max(res.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "clocks": clk.summary(), "gpu_launches": 1 + res.steps * (3 + 6 * 5 + 4),
            "state_finite": bool(torch.isfinite(u).all())}
    if counts is not None:
        line["closures_per_step"] = {k: v / max(res.steps, 1) for k, v in counts.items()}
        # the closure kernels are FP64-bound: algorithmic work = the MLP pair's multiply-adds per closure
        # evaluation (2 passes x (6x24 + 24x16 + 16x16 + 16x4) FMA = 3392 flop), device-counted evaluations
        from weno_sr_publishing_b200 import _native as N
        ctx = N.context(local)
        peak64 = ctx.peak_tflops(64, C_stream(stream))
        flop = 3392.0 * sum(counts.values())
        achieved = flop / (ms * 1e-3) / 1e12
        line["roofline"] = {"kernel": "k7s_normal + k7s_flux (the step's closure kernels)", "bound": "fp64",
                            "achieved": achieved, "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                            "traffic": None, "work": "MLP multiply-adds only (exp, rcp, features not counted)",
                            "peak_source": f"measured FMA probe {peak64:.1f}"}
    if not args.skip_extras:
        host = torch.empty(u0.shape, dtype=torch.float64, pin_memory=True)
        host.copy_(u0.cpu())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):  # each step: pinned state in, one step, state out
            u.copy_(host, non_blocking=True)
            E7.run(u, p, "periodic", max_steps=1, ws=ws, method=method, closure=closure)
            host.copy_(u, non_blocking=True)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        line["e2e"] = {"value": n * n * K / el, "unit": UNIT, "h2d_bytes_per_step": u.numel() * 8,
                       "d2h_bytes_per_step": u.numel() * 8,
                       "api": "weno_sr_publishing_b200.euler2d_w7.run (pinned host buffer, 1 step per call)"}
        if rank == 0:
            line["cpu_baseline"] = cpu_sample()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def bench_3d(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from weno_sr_publishing_b200 import euler3d as E3
    from weno_sr_publishing_b200 import problems as PR
    from weno_sr_publishing_b200.checkpoint import MODELS_DIR
    method = args.method
    params = None
    if method not in ("js", "z"):
        name = "weno5_sr_fp64_step012250.npz" if method == "sr_f64" else "weno5_sr_fp32_step016500.npz"
        params = {k: v for k, v in np.load(MODELS_DIR / name).items() if k != "meta_json"}
    scheme = {"js": "WENO5-JS", "z": "WENO5-Z"}.get(method, f"WENO5-SR ({method})")
    metric = f"3D Euler cell-updates/s, {scheme} HLLC, 224x88x88 shock-bubble"
    cfg = {"workload": "3D shock-bubble, 224x88x88 on [0,2.545]x[0,1]^2, seed 0 (Mach and density ratio), "
                       "post-shock inflow, from t=0", "method": method, "flux": "hllc", "cfl": 0.4,
           "time_integrator": "SSPRK3", "state_precision": "fp64",
           "l2_policy": "state 81 MB, workspace 0.8 GB per step: larger than L2",
           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}
    slabs = args.decomp == "slabs" or (args.decomp == "auto" and world > 1)
    if slabs:
        cfg["parallelism"] = (f"z-slabs x{world}: rank r owns planes of the one 224x88x88 grid, 3-plane halo "
                              f"exchange per stage (NCCL send/recv), MAX all-reduce of the wave speed per step")
    sb = PR.ShockBubble.seeded(0)
    if args.impl == "reference":
        if rank != 0:
            return
        base = _oracle3d_sample(0, method, params, args.cpu_seconds)
        line = {"metric": metric, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg, "impl": "reference",
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1 or slabs:
        import datetime
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29534")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev, rank=rank,
                                world_size=world)
    stream = torch.cuda.current_stream(dev)
    q0 = torch.as_tensor(sb.state(), device=dev).contiguous()
    dx, dy, dz = sb.spacing
    ws = E3.workspace(sb.nx, sb.ny, sb.nz, dev)
    K, W = args.steps, max(args.warmup, 0)
    if slabs:
        _bench_3d_slabs(args, world, rank, local, sb, q0, method, params, metric, cfg, K, W)
        return
    q = q0.clone()
    if W:
        E3.run(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, method, "hllc", params, inflow=sb.inflow(), steps=W, ws=ws)
    q.copy_(q0)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        res = E3.run(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, method, "hllc", params, inflow=sb.inflow(), steps=K,
                     ws=ws)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    cells = sb.nx * sb.ny * sb.nz
    finite = bool(torch.isfinite(q).all())
    line = {"metric": metric, "value": world * cells * K / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": cfg, "clocks": clk.summary(),
            "gpu_launches": 2 + K * (2 + 3 * 13), "t_reached": res.t, "state_finite": finite,
            "shock": {"mach": sb.mach, "density_ratio": sb.density_ratio}}
    # closure tallies over the same run
    q.copy_(q0)
    E3.run(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, method, "hllc", params, inflow=sb.inflow(), steps=K, ws=ws,
           opts=4)
    line["closure_tally_per_step"] = {k: {"mlp": v[0] / K, "plateau": v[1] / K} for k, v in E3.counters(ws).items()
                                      if k != "fallbacks"}
    # one more step from the state the tally run reached: ncu --profile-from-start off captures these launches only
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    E3.run(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, method, "hllc", params, inflow=sb.inflow(), steps=1, ws=ws)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    if method not in ("js", "z"):
        line["roofline"] = _closure_roofline(
            "k3_normal + k3_trans + k3_flux (closure work only)", method,
            [(v[0] / K, v[1] / K, 1 if k == "normal" else 2) for k, v in E3.counters(ws).items() if k != "fallbacks"],
            ms / K, local, stream)
    if not args.skip_extras:
        # end to end: every step the padded state from pinned host memory, one step, and back
        host = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True)
        host.copy_(q0.cpu())
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(K):
            q.copy_(host, non_blocking=True)
            E3.run(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, method, "hllc", params, inflow=sb.inflow(), steps=1,
                   ws=ws)
            host.copy_(q, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1)
        nbytes = int(q0.numel()) * 8
        line["e2e"] = {"value": world * cells * K / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes,
                       "api": "weno_sr_publishing_b200.euler3d.run (pinned host state copied in and out every step, "
                              "1 step per call)"}
        if rank == 0 and world == 1:
            line["cpu_baseline"] = _oracle3d_sample(0, method, params, args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _bench_3d_slabs(args, world, rank, local, sb, q0, method, params, metric, cfg, K, W):
    """The 3D step on z-slabs of the one shock-bubble grid (strong scaling), timed as the max over ranks."""
    import torch
    import torch.distributed as dist

    from weno_sr_publishing_b200 import slabs as S
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    dx, dy, dz = sb.spacing
    grid = S.slab_grid3(sb.nx, sb.ny, sb.nz, dx, dy, dz, world, rank)
    comm = S.DistSlabs()
    stages = S.CudaStages3(method, "hllc", params, sb.inflow())
    if W:
        S.run3([S.split3(q0, sb.nz, world, rank)], [grid], 0.4, comm, stages, steps=W)
    slab = S.split3(q0, sb.nz, world, rank)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        res = S.run3([slab], [grid], 0.4, comm, stages, steps=K)
        e1.record(stream)
        torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    cells = sb.nx * sb.ny * sb.nz
    ok = torch.tensor([float(torch.isfinite(slab).all())], device=dev)
    dist.all_reduce(ok, op=dist.ReduceOp.MIN)
    line = {"metric": metric, "value": cells * K / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": cfg, "clocks": clk.summary(),
            # per step: max speed (1), 3 stages x (control init + 2 boundary passes + 3 sweeps x 3 + update)
            "gpu_launches": K * (1 + 3 * 13), "t_reached": res.t, "state_finite": bool(ok.item()),
            "shock": {"mach": sb.mach, "density_ratio": sb.density_ratio}}
    if not args.skip_extras:
        # end to end: this rank's padded slab from pinned host memory, K steps, and back
        host = torch.empty(grid.padded_shape, dtype=torch.float64, pin_memory=True)
        host.copy_(S.split3(q0, sb.nz, world, rank).cpu())
        dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(K):
            slab.copy_(host, non_blocking=True)
            S.run3([slab], [grid], 0.4, comm, stages, steps=1)
            host.copy_(slab, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        nbytes = int(np.prod(grid.padded_shape)) * 8
        line["e2e"] = {"value": cells * K / (float(t.item()) * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes,
                       "api": "weno_sr_publishing_b200.slabs.run3 (this rank's pinned host slab copied in and out every "
                              "step, 1 step per call)"}
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _roofline_1d(scheme, method, work_cellsteps, mlp_n, plat_n, ms, peak, ctx, stream):
    """Closure-bound roofline of the 1D step from the device tallies (3 stages per step; SSPRK3 for
    WENO5): per MLP stencil the MLP pair in the closure precision plus the FP64 features and head, per
    plateau stencil the sensors and linear head. Shu RK4 (WENO7) evaluates 4 right-hand sides with both
    heads; its MLP is 6->24->16->16->4."""
    from weno_sr_publishing_b200 import roofline as R
    mlp_flops = R.MLP_PAIR_FLOPS if scheme == 5 else 2 * (2 * (6 * 24 + 24 * 16 + 16 * 16 + 16 * 4) + 56 * 3 + 25)
    w_mlp = mlp_n * mlp_flops
    w64 = mlp_n * (R.SENSORS64 + R.FEATURES64 + R.HEAD64) + plat_n * (R.SENSORS64 + R.HEAD64_PLATEAU)
    w64 += work_cellsteps * 3 * 6
    w32 = 0.0
    if method == "sr_f64":
        w64 += w_mlp
    else:
        w32 += w_mlp
    peak64 = ctx.peak_tflops(64, C_stream(stream))
    peak32 = ctx.peak_tflops(32, C_stream(stream))
    b = R.bound({"w32": w32, "w64": w64, "bytes": 0.0}, ms * 1e-3, peak32, peak64, 6541.0)
    return {"kernel": "k_adv1d", "bound": b["bound"], "achieved": b["achieved"], "peak": b["peak"], "unit": b["unit"],
            "frac": b["frac"], "traffic": None,
            "peak_source": {"fp32_tflops": f"measured FMA probe {peak32:.1f}",
                            "fp64_tflops": f"measured FMA probe {peak64:.1f}"}}


def _closure_roofline(kernels, method, classes, ms, local, stream):
    """Roofline of the closure work alone (a lower bound on the kernels' work, so `frac` is a lower bound): per
    evaluation the MLP pair in the closure precision plus the FP64 sensors, features and weights; per plateau
    stencil the sensors and the linear head. classes: (MLP evaluations, plateau stencils, heads per stencil) per
    step."""
    from weno_sr_publishing_b200 import _native as N
    from weno_sr_publishing_b200 import roofline as R
    ctx = N.context(local)
    peak32 = ctx.peak_tflops(32, C_stream(stream))
    peak64 = ctx.peak_tflops(64, C_stream(stream))
    w32 = w64 = 0.0
    for mlp_n, plat_n, heads in classes:
        if method == "sr_f64":
            w64 += mlp_n * R.MLP_PAIR_FLOPS
        else:
            w32 += mlp_n * R.MLP_PAIR_FLOPS
        w64 += mlp_n * (R.SENSORS64 + R.FEATURES64 + heads * R.HEAD64) + plat_n * (R.SENSORS64 +
                                                                                   heads * R.HEAD64_PLATEAU)
    b = R.bound({"w32": w32, "w64": w64, "bytes": 0.0}, ms * 1e-3, peak32, peak64, hbm_peak()["gbs"])
    return {"kernel": kernels, "bound": b["bound"], "achieved": b["achieved"], "peak": b["peak"], "unit": b["unit"],
            "frac": b["frac"], "traffic": None, "work": "closure work only (lower bound)",
            "peak_source": {"fp32_tflops": f"measured FMA probe {peak32:.1f}",
                            "fp64_tflops": f"measured FMA probe {peak64:.1f}"}}


# DRAM bytes (read + write) of one launch of the dominant kernel, from the ncu capture of the same workload
# (kernel class, method, grid): the headline configuration only.
NCU_TRAFFIC = {("flux_x", "sr_f32", 2000): 361.8e6, ("flux_x", "js", 2000): 360.6e6}


def C_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def hbm_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return {"gbs": float(json.loads(path.read_text())["hbm_gbs"]), "source": "MEASURED_PEAKS.json (measured)"}
        except (KeyError, ValueError):
            pass
    return {"gbs": 6650.0, "source": "fallback 6.65 TB/s"}


if __name__ == "__main__":
    main()
