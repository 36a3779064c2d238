"""Accuracy at matched cost: the periodic isentropic-vortex convergence study and the matched-L1 comparison
of WENO5-SR against WENO5-JS.

The setup is the reference's vortex experiment (experiments/05_isentropic_vortex/config.yaml; the vortex of
weno7_point_rk4_shu/point_rk4.py:81-118): [-10, 10]^2 periodic, strength 5, mean flow (1, 1), gamma 1.4,
15 x 15 Gauss-Legendre cell averages, CFL 0.4, t_end = 2, error L1(rho) = mean |rho - rho_exact| over the
cells against the exact translated finite-volume vortex.

Matched L1: with L1_JS(N) known at a few N, the JS resolution that reaches the SR error at N_SR follows
from log-log interpolation; the time to that accuracy then compares the two methods at equal error.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import euler2d as E
from . import problems
from .params import Params

LENGTH = 20.0
T_END = 2.0
CFL = 0.4


@dataclass
class VortexResult:
    n: int
    method: str
    l1: float
    l2: float
    steps: int
    device_ms: float


def vortex_run(n: int, method: str, mlp_params=None, device="cuda", quadrature: int = 15) -> VortexResult:
    """One convergence point: N x N cells to t = 2 on the GPU, device-timed."""
    p = Params(nx=n, ny=n, x_length=LENGTH, y_length=LENGTH, cfl=CFL)
    init = problems.isentropic_vortex(n, n, 0.0, quadrature, length=LENGTH)
    exact = problems.isentropic_vortex(n, n, T_END, quadrature, length=LENGTH)
    dev = torch.device(device)
    bufs = [torch.as_tensor(init, device=dev).contiguous()] + \
        [torch.zeros(p.padded_shape, dtype=torch.float64, device=dev) for _ in range(3)]
    ws = E.workspace(n, n, dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    res = E.run(bufs, p, T_END, method, "periodic", mlp_params=mlp_params, ws=ws)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    rho = bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3, 0]
    err = rho - exact[3:-3, 3:-3, 0]
    return VortexResult(n, method, float(np.mean(np.abs(err))), float(np.sqrt(np.mean(err * err))), res.steps,
                        e0.elapsed_time(e1))


def vortex7_run(n: int, device="cuda", quadrature: int = 15, method: str = "js", closure=None) -> VortexResult:
    """WENO7 (method "js", "z" or "sr_f64" with the WENO7 closure `closure`) with Shu RK4 on the same vortex
    problem (the WENO7 rows of the reference's convergence table: weno7_point_rk4_shu/point_rk4.py,
    weno7_point_rk4_z and warp_sod/point_rk4_mlp.py, HLLC, characteristic, [-10, 10]^2, CFL 0.4, t = 2)."""
    from . import euler2d_w7 as E7  # noqa: PLC0415

    p = E7.Params(nx=n, ny=n, cfl=CFL, t_end=T_END)
    init = problems.vortex_point_rk4(n, n, 0.0, quadrature)
    exact = problems.vortex_point_rk4(n, n, T_END, quadrature)
    dev = torch.device(device)
    u = torch.as_tensor(init, device=dev).contiguous()
    ws = E7.workspace(n, n, dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    res = E7.run(u, p, "periodic", ws=ws, method=method, closure=closure)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    err = u.cpu().numpy()[4:-4, 4:-4, 0] - exact[4:-4, 4:-4, 0]
    return VortexResult(n, f"w7_{method}", float(np.mean(np.abs(err))), float(np.sqrt(np.mean(err * err))), res.steps,
                        e0.elapsed_time(e1))


def loglog_n_for_error(points: list[VortexResult], target: float) -> float:
    """Resolution N at which the method's L1 equals `target`, interpolating log L1 linearly in log N between
    the two bracketing points (extrapolating from the nearest pair outside the range)."""
    pts = sorted(points, key=lambda r: r.n)
    for a, b in zip(pts, pts[1:]):
        if a.l1 >= target >= b.l1:
            break
    else:
        a, b = (pts[0], pts[1]) if target > pts[0].l1 else (pts[-2], pts[-1])
    slope = math.log(b.l1 / a.l1) / math.log(b.n / a.n)
    return a.n * math.exp(math.log(target / a.l1) / slope)


def loglog_time_at(points: list[VortexResult], n: float) -> float:
    """Device time to t_end at resolution n, interpolating log time in log N."""
    pts = sorted(points, key=lambda r: r.n)
    for a, b in zip(pts, pts[1:]):
        if a.n <= n <= b.n:
            break
    else:
        a, b = (pts[0], pts[1]) if n < pts[0].n else (pts[-2], pts[-1])
    slope = math.log(b.device_ms / a.device_ms) / math.log(b.n / a.n)
    return a.device_ms * math.exp(slope * math.log(n / a.n))


def matched_l1(sr: list[VortexResult], js: list[VortexResult]) -> list[dict]:
    """For each SR point: the JS resolution with the same L1, and the SR / JS times to that accuracy."""
    out = []
    for r in sr:
        n_js = loglog_n_for_error(js, r.l1)
        t_js = loglog_time_at(js, n_js)
        out.append({"n_sr": r.n, "l1": r.l1, "n_js_matched": n_js, "sr_ms": r.device_ms, "js_ms_matched": t_js,
                    "speedup_at_matched_l1": t_js / r.device_ms,
                    "sr_cell_updates_per_s": r.n * r.n * r.steps / (r.device_ms * 1e-3)})
    return out


# ------------------------------------------------------------------------------------------------
# Matched L1 on the discontinuous workload: the seeded quadrant Riemann problem against a fine-grid
# WENO5-JS reference, block-averaged (for_paper_results/common.py:116-120).
# ------------------------------------------------------------------------------------------------
def conservative_block_average(state: np.ndarray, target_n: int) -> np.ndarray:
    if state.shape[0] != state.shape[1] or state.shape[0] % target_n:
        raise ValueError(f"cannot block-average shape {state.shape} to {target_n}x{target_n}")
    f = state.shape[0] // target_n
    return state.reshape(target_n, f, target_n, f, state.shape[-1]).mean(axis=(1, 3))


def quadrant_run(n: int, method: str, mlp_params=None, device="cuda", seed: int = 0, t_end: float = 0.25):
    """(interior state at t_end, device ms, steps) of the seeded quadrant problem on n x n (midpoint cell
    averages: the interfaces fall on cell edges for even n)."""
    p = Params(nx=n, ny=n, x_length=1.0, y_length=1.0, cfl=CFL)
    init = problems.make_quadrant_state(n, n, problems.seeded_quadrant_states(seed), quadrature=1)
    dev = torch.device(device)
    bufs = [torch.as_tensor(init, device=dev).contiguous()] + \
        [torch.zeros(p.padded_shape, dtype=torch.float64, device=dev) for _ in range(3)]
    ws = E.workspace(n, n, dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    res = E.run(bufs, p, t_end, method, "transmissive", mlp_params=mlp_params, ws=ws)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    return bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3], e0.elapsed_time(e1), res.steps


def quadrant_study(method: str, mlp_params, device="cuda", ns=(100, 200, 400), ref_n: int = 2000, seed: int = 0):
    """L1(rho) of the method and of WENO5-JS at each n against the block-averaged ref_n^2 WENO5-JS solution,
    and the matched-L1 comparison."""
    ref, ref_ms, _ = quadrant_run(ref_n, "js", None, device, seed)
    out = {}
    for m, prm in ((method, mlp_params), ("js", None)):
        pts = []
        for n in ns:
            st, ms, steps = quadrant_run(n, m, prm, device, seed)
            err = st[..., 0] - conservative_block_average(ref, n)[..., 0]
            pts.append(VortexResult(n, m, float(np.mean(np.abs(err))), float(np.sqrt(np.mean(err * err))), steps, ms))
        out[m] = pts
    return out, ref_ms
