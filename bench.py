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
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="sr_f32", choices=["sr_f32", "sr_f64", "sr_bf16", "js"])
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--t0", type=float, default=0.125)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--skip-extras", action="store_true", help="no JS arm, e2e, CPU baseline (profiling runs)")
    return ap.parse_args()


def workload_config(args, n_gpus):
    return {"workload": f"2D Euler quadrant Riemann problem {args.n}x{args.n}, seed 0, state at t0={args.t0}",
            "grid": [args.n, args.n], "ghost": 3, "gamma": 1.4, "cfl": 0.4, "boundary": "transmissive",
            "flux": "hllc", "time_integrator": "SSPRK3", "method": args.method,
            "closure_precision": {"sr_f32": "fp32", "sr_f64": "fp64", "sr_bf16": "bf16", "js": None}[args.method],
            "state_precision": "fp64", "l2_policy": "inputs larger than L2 (state 4 x 129 MB + 0.8 GB workspace)",
            "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU"}


def initial_state(n):
    from weno_sr_publishing_b200 import problems
    # the quadrant interfaces at x = y = 0.5 fall on cell edges for even n, so every cell average is a
    # single state and the midpoint rule is exact
    return problems.make_quadrant_state(n, n, problems.seeded_quadrant_states(0), quadrature=1)


def crop(state, n_crop):
    """Centre n_crop x n_crop window of a padded state, re-padded (ghosts are refilled by the BC)."""
    n = state.shape[0] - 6
    a = (n - n_crop) // 2
    out = np.zeros((n_crop + 6, n_crop + 6, 4))
    out[3:3 + n_crop, 3:3 + n_crop] = state[3 + a:3 + a + n_crop, 3 + a:3 + a + n_crop]
    return out


def cpu_sample(state, method, params, budget_s, fast=True):
    """Time the CPU oracle (all host threads) on a centre crop of the benchmark state."""
    from oracle import oracle as O
    n_crop = 256
    sub = crop(state, n_crop)
    dx = 1.0 / params["n"]
    prm = params["mlp"]
    O.euler2d_run(sub, n_crop, n_crop, dx, dx, 0.4, 1.0, method, "transmissive", params=prm, fixed_steps=1, fast=fast)
    steps, t0 = 0, time.perf_counter()
    while True:
        O.euler2d_run(sub, n_crop, n_crop, dx, dx, 0.4, 1.0, method, "transmissive", params=prm, fixed_steps=1,
                      fast=fast)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or steps >= 50:
            break
    return {"value": n_crop * n_crop * steps / el, "unit": UNIT, "cores": O.num_threads(fast),
            "kind": "port", "sample": f"{steps} step(s) of a {n_crop}x{n_crop} centre crop of the benchmark state, "
                                      f"{el:.1f} s, C oracle (OpenMP, -O3)"}


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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
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
    """The reference has no CPU path for 2D Euler (Warp GPU kernels only); its CPU counterpart here is the
    C restatement of those kernels in oracle/ (a port), timed on all host threads. The 2000^2 state at t0
    is out of reach on the CPU, so the sample is the same problem on a 256^2 grid of the whole square,
    advanced (untimed) to the same t0 with the oracle's WENO5-JS: the same physical mix of plateau and
    wave regions per cell."""
    if rank != 0:
        return
    from oracle import oracle as O
    from weno_sr_publishing_b200 import problems
    from weno_sr_publishing_b200.checkpoint import MODELS_DIR
    mlp = None
    if args.method != "js":
        name = "weno5_sr_fp64_step012250.npz" if args.method == "sr_f64" else "weno5_sr_fp32_step016500.npz"
        mlp = {k: v for k, v in np.load(MODELS_DIR / name).items() if k != "meta_json"}
    m = 256
    init = problems.make_quadrant_state(m, m, problems.seeded_quadrant_states(0), quadrature=1)
    state, _, _, _ = O.euler2d_run(init, m, m, 1.0 / m, 1.0 / m, 0.4, args.t0, "js", "transmissive", fast=True)
    dx = 1.0 / m
    for _ in range(args.warmup):
        O.euler2d_run(state, m, m, dx, dx, 0.4, 1.0, args.method, "transmissive", params=mlp, fixed_steps=1,
                      fast=True)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.euler2d_run(state, m, m, dx, dx, 0.4, 1.0, args.method, "transmissive", params=mlp, fixed_steps=1,
                      fast=True)
    el = time.perf_counter() - t0
    v = m * m * args.steps / el
    base = {"value": v, "unit": UNIT, "cores": O.num_threads(True), "kind": "port",
            "sample": f"{args.steps} steps of the same problem on a {m}x{m} grid at t0={args.t0} "
                      f"(C oracle, OpenMP), {el:.1f} s"}
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * args.n * args.n / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, args.gpus), "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
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
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
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

    with ClockSampler(local) as clk:
        ms, r = timed(args.method, mlp, K, W)
    clocks = clk.summary()
    value = world * n * n * K / (ms * 1e-3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": workload_config(args, world), "clocks": clocks}
    # per step: dt kernels (2), 3 stages x 5 kernels, t/steps update (1); plus init and max-speed per run
    line["gpu_launches"] = 2 + K * (3 + 3 * 5)

    if not args.skip_extras:
        # WENO5-JS on the same state and steps: the cost ratio of the learned closure
        ms_js, _ = timed("js", None, K, W)
        line["js"] = {"value": world * n * n * K / (ms_js * 1e-3), "ms_per_step": ms_js / K,
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
    line["roofline"] = {"kernel": dom, "bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"],
                        "unit": d["unit"], "frac": d["frac"], "traffic": None,
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
    line["roofline_step"] = R.bound(step_work, ms / K * 1e-3, peak32, peak64, hbm["gbs"])
    line["kernels"] = {k: {kk: v[kk] for kk in ("ms_per_launch", "launches", "share", "bound", "frac")}
                       for k, v in per_kernel.items()}
    line["closure_tally_per_step"] = {k: {"mlp": v[0], "plateau": v[1]} for k, v in tallies.items()}

    if not args.skip_extras:
        # end to end: pinned host state -> device, one step, device -> pinned host, K times
        host = torch.empty(p.padded_shape, dtype=torch.float64, pin_memory=True)
        host.copy_(start.cpu())
        for _ in range(max(W, 1)):
            E.advance_host(host, p, 1, args.method, "transmissive", mlp_params=mlp, bufs=bufs, ws=ws, device=dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            E.advance_host(host, p, 1, args.method, "transmissive", mlp_params=mlp, bufs=bufs, ws=ws, device=dev)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms_e2e], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e2e = float(t.item())
        nbytes = int(np.prod(p.padded_shape)) * 8
        line["e2e"] = {"value": world * n * n * K / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes,
                       "api": "weno_sr_publishing_b200.euler2d.advance_host (pinned host buffer, 1 step per call)"}
        if rank == 0 and world == 1:
            line["cpu_baseline"] = cpu_sample(start.cpu().numpy(), args.method, {"n": n, "mlp": mlp},
                                              args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


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
