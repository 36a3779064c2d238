"""Scalar WENO-Z advection steppers of the paper's order-matched Z baselines, on the GPU (libwsr.so).

Drop-in for ``weno_z_borges_p2_results/torch_weno_z.py`` (reference project, code/snapshot/) and the
``integrate`` helper of ``weno_z_borges_p2_results/run_gste.py:20-30``:

* ``ssprk3_step(state, dt, dxinv)`` -- WENO5-Z (p = 2, eps = h^2, tau5 = |b0 - b2|) with SSPRK3
  (torch_weno_z.py:14-20, 68-72);
* ``shu_rk4_step(state, dt, dxinv)`` -- WENO7-Z (p = 3, eps = h^3, tau7 = |-b0 - 3 b1 + 3 b2 + b3|) with
  Shu's RK4 and the downwind operator (torch_weno_z.py:23-32, 75-107);
* ``integrate(initial, t_end, cfl, stepper, device)`` -- steps = ceil(t_end / (cfl dx)) on [-1, 1].

``state`` is [B, N], each row a periodic trajectory advected with velocity +1 (the only sign the
reference module has), h = 1 / dxinv. Every call is one launch of the batched 1D kernel
(``adv1d.run_batched`` with ``model="z"``); there is no CPU path.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import adv1d as A

P_Z5 = 2
P_Z7 = 3
LENGTH = 2.0  # for_paper_results/run_gste.py: the GSTE domain [-1, 1]


def _steps(state, dt: float, dxinv: float, steps: int, scheme: int, integrator: str):
    t = torch.as_tensor(state, dtype=torch.float64)
    if t.ndim != 2:
        raise ValueError("state must be [B, N]")
    dev = t.device if t.is_cuda else torch.device("cuda")
    B = t.shape[0]
    outs, _ = A.run_batched([t[b] for b in range(B)], np.ones(B), 1.0 / dxinv, steps, dt, None, scheme=scheme,
                            model="z", integrator=integrator, device=dev)
    out = torch.stack(outs)
    return out if t.is_cuda else out.cpu()


def ssprk3_step(state, dt: float, dxinv: float):
    """One SSPRK3 step of WENO5-Z (torch_weno_z.py:68-72)."""
    return _steps(state, dt, dxinv, 1, 5, "ssprk3")


def shu_rk4_step(state, dt: float, dxinv: float):
    """One Shu RK4 step of WENO7-Z with L and L~ (torch_weno_z.py:75-107)."""
    return _steps(state, dt, dxinv, 1, 7, "shu_rk4")


def integrate(initial, t_end: float, cfl: float, stepper, device="cuda"):
    """GSTE integration (weno_z_borges_p2_results/run_gste.py:20-30): all steps in one launch.

    Returns (final state, steps, dt, dt / dx) like the reference."""
    u0 = np.asarray(initial, dtype=np.float64)
    nx = u0.size
    dx = LENGTH / float(nx)
    steps = int(math.ceil(t_end / (cfl * dx)))
    dt = t_end / float(steps)
    if stepper is ssprk3_step:
        scheme, integ = 5, "ssprk3"
    elif stepper is shu_rk4_step:
        scheme, integ = 7, "shu_rk4"
    else:
        raise ValueError("stepper must be weno_z.ssprk3_step or weno_z.shu_rk4_step")
    outs, _ = A.run_batched([u0], [1.0], dx, steps, dt, None, scheme=scheme, model="z", integrator=integ,
                            device=device)
    return outs[0].cpu().numpy(), steps, dt, dt / dx
