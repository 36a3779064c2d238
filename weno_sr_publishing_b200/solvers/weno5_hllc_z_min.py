"""WENO5-Z (Borges p = 2, eps = h^2) + HLLC + SSPRK3 adapter
(weno_z_borges_p2_results/weno5_hllc_z_min.py:287-416).

Same stage layout as the WENO5-JS adapter; the Z weights take eps = dx^2 for reconstructions along x and
dy^2 along y (the normal pass of x faces and the transverse pass of y faces use dx, and the other way
round), as the reference passes params.dx / params.dy into its kernels. The reference's signatures have
no closure argument.
"""
from __future__ import annotations

from . import _adapter as A

METHOD = "z"


def allocate_forward(u0, params, device):
    return A.allocate_forward(u0, params, device)


def _launch_stage(u_stage, u0, u_out, stage, params, dt, rk, device, boundary):
    A.launch_stage(METHOD, u_stage, u0, u_out, stage, params, dt, rk, device, None, boundary)


launch_stage = _launch_stage


def advance_step(arrays, params, dt, device, boundary):
    A.advance_step(METHOD, arrays, params, dt, device, None, boundary)


def run_to_time(u0, params, t_end, device, boundary, report_interval=0, report=None):
    return A.run_to_time(METHOD, u0, params, t_end, device, None, boundary, report_interval=report_interval,
                         report=report)
