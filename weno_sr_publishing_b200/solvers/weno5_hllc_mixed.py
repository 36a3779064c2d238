"""WENO5-SR with an FP32 MLP (FP64 state, projections, flux and update) + HLLC + SSPRK3 adapter
(for_paper_results/solvers/weno5_hllc_mixed.py:121-212)."""
from __future__ import annotations

from . import _adapter as A

METHOD = "sr_f32"


def allocate_forward(u0, params, device):
    return A.allocate_forward(u0, params, device)


def launch_stage(u_stage, u0, u_out, stage, params, dt, rk, device, mlp_params, boundary, boundary_time=0.0):
    A.launch_stage(METHOD, u_stage, u0, u_out, stage, params, dt, rk, device, mlp_params, boundary,
                   boundary_time=boundary_time)


def advance_step(arrays, params, dt, device, mlp_params, boundary):
    A.advance_step(METHOD, arrays, params, dt, device, mlp_params, boundary)


def run_to_time(u0, params, t_end, device, mlp_params, boundary, report_interval=0, report=None):
    return A.run_to_time(METHOD, u0, params, t_end, device, mlp_params, boundary, report_interval=report_interval,
                         report=report)
