"""WENO5-JS + HLLC + SSPRK3 adapter (for_paper_results/solvers/weno5_hllc.py:294-410).

The reference adapter also accepts mlp_params, which route to its pre-V20 closure (scale feature
(log10+16)/16, no reflection average); that legacy operator is not part of the published method and is
not provided: use weno5_hllc_refsym or weno5_hllc_mixed for WENO5-SR.
"""
from __future__ import annotations

from . import _adapter as A

METHOD = "js"


def _no_legacy(mlp_params) -> None:
    if mlp_params is not None:
        raise NotImplementedError("the pre-V20 MLP closure of weno5_hllc is not provided; use weno5_hllc_refsym "
                                  "(FP64 closure) or weno5_hllc_mixed (FP32 closure)")


def allocate_forward(u0, params, device):
    return A.allocate_forward(u0, params, device)


def launch_stage(u_stage, u0, u_out, stage, params, dt, rk, device, mlp_params, boundary, eno_cutoff=False):
    _no_legacy(mlp_params)
    A.launch_stage(METHOD, u_stage, u0, u_out, stage, params, dt, rk, device, None, boundary, eno_cutoff)


def advance_step(arrays, params, dt, device, mlp_params, boundary):
    _no_legacy(mlp_params)
    A.advance_step(METHOD, arrays, params, dt, device, None, boundary)


def run_to_time(u0, params, t_end, device, mlp_params, boundary, report_interval=0, report=None):
    _no_legacy(mlp_params)
    return A.run_to_time(METHOD, u0, params, t_end, device, None, boundary, report_interval=report_interval,
                         report=report)
