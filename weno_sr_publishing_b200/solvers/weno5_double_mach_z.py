"""WENO5-Z on the double-Mach reflection (weno_z_borges_p2_results/weno5_double_mach_z.py:111-217): the
WENO5-Z stage of weno5_hllc_z_min with the time-dependent double-Mach boundary, evaluated at t, t + dt and
t + dt/2 for the three SSPRK3 stages."""
from __future__ import annotations

from . import _adapter as A

METHOD = "z"
BOUNDARY = "double-mach"


def allocate_forward(u0, params, device):
    return A.allocate_forward(u0, params, device)


def _launch_stage(u_stage, u0, u_out, stage, params, dt, rk, device, boundary_time):
    A.launch_stage(METHOD, u_stage, u0, u_out, stage, params, dt, rk, device, None, BOUNDARY,
                   boundary_time=boundary_time)


def run_to_time(initial, params, t_end, device, *, report_interval=100, report=None):
    return A.run_to_time(METHOD, initial, params, t_end, device, None, BOUNDARY, report_interval=report_interval,
                         report=report)
