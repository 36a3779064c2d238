"""WENO5-SR (FP64 reflection-averaged MLP closure) + HLLC + SSPRK3 adapter
(teacherfree_lab_weno5_v20_distance_balanced/weno5_hllc_refsym.py:298-544)."""
from __future__ import annotations

from . import _adapter as A

METHOD = "sr_f64"


def allocate_forward(initial, params, device):
    return A.allocate_forward(initial, params, device)


def launch_stage(u_stage, u0, u_out, stage, params, dt, rk, device, mlp_params, boundary, boundary_time=0.0,
                 eno_cutoff=False):
    A.launch_stage(METHOD, u_stage, u0, u_out, stage, params, dt, rk, device, mlp_params, boundary, eno_cutoff,
                   boundary_time=boundary_time)


def advance_step(arrays, params, dt, device, mlp_params, boundary):
    A.advance_step(METHOD, arrays, params, dt, device, mlp_params, boundary)


def run_to_time(initial, params, t_end, device, mlp_params, boundary, eno_cutoff=False, report_interval=100,
                report=None):
    return A.run_to_time(METHOD, initial, params, t_end, device, mlp_params, boundary, eno_cutoff=eno_cutoff,
                         report_interval=report_interval, report=report, health_break=True)
