"""Shared implementation of the reference's adapter protocol for the three WENO5 methods.

Protocol (for_paper_results/solvers/weno5_hllc.py:294-410; weno5_hllc_refsym.py:298-544;
weno5_hllc_mixed.py:121-212): allocate_forward, launch_stage, advance_step, run_to_time. Arrays are
torch CUDA tensors in the reference's padded layout; run_to_time takes and returns numpy arrays.
"""
from __future__ import annotations

from collections.abc import Callable

import numpy as np
import torch

from .. import euler2d as E
from ..params import Params, interior_stats

SUPPORTED_BOUNDARIES = ("transmissive", "periodic", "double-mach")


def _check_boundary(boundary: str) -> None:
    if boundary not in SUPPORTED_BOUNDARIES:
        raise ValueError(f"unsupported boundary {boundary!r}")


def allocate_forward(u0, params: Params, device: str) -> dict:
    dev = torch.device(device)
    E.device_index(dev)
    init = torch.as_tensor(np.ascontiguousarray(u0, dtype=np.float64), device=dev)
    if tuple(init.shape) != params.padded_shape:
        raise ValueError(f"initial state shape {tuple(init.shape)} != {params.padded_shape}")

    def state():
        return torch.zeros(params.padded_shape, dtype=torch.float64, device=dev)

    ws = E.workspace(params.nx, params.ny, dev)
    stage_ws = {"workspace": ws}
    return {"u0": init, "u1": state(), "u2": state(), "u3": state(), "speed": None,
            "s1": stage_ws, "s2": stage_ws, "s3": stage_ws}


def launch_stage(method: str, u_stage, u0, u_out, stage: dict, params: Params, dt: float, rk: int, device: str,
                 mlp_params, boundary: str, eno_cutoff: bool = False, js_fallback: bool = False,
                 boundary_time: float = 0.0) -> None:
    _check_boundary(boundary)
    opts = (E.N.OPT_ENO_CUTOFF if eno_cutoff else 0) | (E.N.OPT_JS_FALLBACK if js_fallback else 0)
    E.stage(u_stage, u0, u_out, params, dt, rk, method, boundary, mlp_params=mlp_params, opts=opts,
            ws=stage["workspace"], boundary_time=boundary_time)


def advance_step(method: str, arrays: dict, params: Params, dt: float, device: str, mlp_params,
                 boundary: str, t: float = 0.0) -> None:
    """One SSPRK3 step from time t (the boundary times of the stages are t, t + dt and t + dt/2)."""
    for rk, src, dst, bt in ((1, "u0", "u1", t), (2, "u1", "u2", t + dt), (3, "u2", "u3", t + 0.5 * dt)):
        launch_stage(method, arrays[src], arrays["u0"], arrays[dst], arrays[f"s{rk}"], params, dt, rk, device,
                     mlp_params, boundary, boundary_time=bt)
    arrays["u0"], arrays["u3"] = arrays["u3"], arrays["u0"]


def run_to_time(method: str, initial, params: Params, t_end: float, device: str, mlp_params, boundary: str,
                eno_cutoff: bool = False, report_interval: int = 0,
                report: Callable[[int, float, float, dict], None] | None = None, health_break: bool = False,
                js_fallback: bool = False) -> tuple[np.ndarray, list[float], int, float]:
    """Time loop with the reference's stopping rule; dt, t and the stop test stay on the device.

    health_break reproduces the FP64 SR adapter (weno5_hllc_refsym.py:529-542): the loop stops when the
    state after step 1, after every report_interval-th step, or at the end holds a NaN or p <= 0.
    """
    _check_boundary(boundary)
    arrays = allocate_forward(initial, params, device)
    ws = arrays["s1"]["workspace"]
    opts = (E.N.OPT_ENO_CUTOFF if eno_cutoff else 0) | (E.N.OPT_JS_FALLBACK if js_fallback else 0)
    if report is None:
        bufs = [arrays["u0"], arrays["u1"], arrays["u2"], arrays["u3"]]
        res = E.run(bufs, params, t_end, method, boundary, mlp_params=mlp_params, opts=opts,
                    check_health=health_break, check_interval=report_interval, ws=ws)
        final = arrays["u3"] if res.final_slot == 3 else arrays["u0"]
        return final.cpu().numpy(), res.dts, res.steps, res.t
    # With a report callback the loop pauses on the host at every reporting step.
    t, step, dts = 0.0, 0, []
    while t < t_end - 1.0e-14:
        if step == 0:
            chunk = 1
        elif report_interval > 0:
            chunk = report_interval - step % report_interval
        else:
            chunk = 1 << 20
        bufs = [arrays["u0"], arrays["u1"], arrays["u2"], arrays["u3"]]
        res = E.run(bufs, params, t_end, method, boundary, mlp_params=mlp_params, opts=opts, max_steps=chunk,
                    t_start=t, ws=ws)
        if res.final_slot == 3:
            arrays["u0"], arrays["u3"] = arrays["u3"], arrays["u0"]
        if res.steps == 0:
            break
        step += res.steps
        t = res.t
        dts.extend(res.dts)
        if step == 1 or (report_interval and step % report_interval == 0) or t >= t_end - 1.0e-14:
            stats = interior_stats(arrays["u0"].cpu().numpy(), params)
            report(step, t, dts[-1], stats)
            if health_break and (stats["nan_count"] or stats["rho_neg"] or stats["p_neg"]):
                break
    return arrays["u0"].cpu().numpy(), dts, step, t
