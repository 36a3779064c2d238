"""Torch-facing driver of the 3D Euler WENO5 path (libwsr.so underneath).

Reference (code/snapshot/warp_weno5_3d_rk3/): ``Weno5Rk3Solver`` (solver.py:22-329) -- ``_rk_stage``,
``advance`` and the run loop of ``run_solver`` -- and its configuration (config.py). The state is the
reference's padded array q[nz+6, ny+6, nx+6, 5] of FP64 conserved variables (rho, rho u, rho v, rho w, E),
gamma 1.4, ghost width 3. ``method`` is "js", "z" (WENO-Z, weno_z_borges_p2_results/weno5_3d_solver_z.py),
"sr_f64", "sr_f32" or "sr_bf16"; ``flux`` "evilin" (the
reference's) or "hllc"; ``inflow`` (5 conserved values) fixes the x-low ghost cells.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .euler2d import device_index, prepare_closure

_ALIGN = 256


@dataclass
class Workspace3:
    buf: torch.Tensor
    ptr: int
    nbytes: int
    shape: tuple


def workspace(nx: int, ny: int, nz: int, device="cuda") -> Workspace3:
    """Device scratch for one 3D grid: stage copy, normal and transverse face values, fluxes, control."""
    nbytes = int(N.lib().wsr_euler3d_workspace_bytes(nx, ny, nz))
    if nbytes == 0:
        raise ValueError(f"invalid grid {nx} x {ny} x {nz}")
    buf = torch.empty(nbytes + _ALIGN, dtype=torch.uint8, device=device)
    ptr = (buf.data_ptr() + _ALIGN - 1) // _ALIGN * _ALIGN
    return Workspace3(buf, ptr, nbytes, (nx, ny, nz))


def _check(q: torch.Tensor, nx: int, ny: int, nz: int) -> None:
    if not isinstance(q, torch.Tensor) or q.dtype != torch.float64 or not q.is_cuda:
        raise TypeError("state must be a float64 CUDA tensor")
    if tuple(q.shape) != (nz + 6, ny + 6, nx + 6, 5) or not q.is_contiguous():
        raise ValueError(f"state must be contiguous with shape {(nz + 6, ny + 6, nx + 6, 5)}, got {tuple(q.shape)}")


def _inflow(inflow):
    if inflow is None:
        return None, None
    arr = (C.c_double * 5)(*[float(v) for v in np.asarray(inflow, dtype=np.float64).reshape(5)])
    return arr, C.cast(arr, C.c_void_p)


def _ws(ws, nx, ny, nz, device):
    if ws is None or ws.shape != (nx, ny, nz):
        ws = workspace(nx, ny, nz, device)
    return ws


def stage(q: torch.Tensor, nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, dt: float, stage: int,
          method: str = "js", flux: str = "evilin", mlp_params=None, inflow=None, opts: int = 0,
          ws: Workspace3 | None = None) -> Workspace3:
    """One RK stage in place (Weno5Rk3Solver._rk_stage, solver.py:285-301). Returns the workspace, which
    carries the stage-start copy that stages 2 and 3 read."""
    _check(q, nx, ny, nz)
    dev = device_index(q.device)
    ctx = prepare_closure(method, mlp_params, dev)
    ws = _ws(ws, nx, ny, nz, q.device)
    keep, inf = _inflow(inflow)
    ctx.check(N.lib().wsr_euler3d_stage(ctx.handle, C.c_void_p(q.data_ptr()), nx, ny, nz, dx, dy, dz, dt, stage,
                                        N.METHOD[method], N.FLUX3[flux], opts, inf, C.c_void_p(ws.ptr), ws.nbytes,
                                        C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    del keep
    return ws


def max_speed(q: torch.Tensor, nx: int, ny: int, nz: int, ws: Workspace3 | None = None) -> float:
    _check(q, nx, ny, nz)
    dev = device_index(q.device)
    ctx = N.context(dev)
    ws = _ws(ws, nx, ny, nz, q.device)
    out = C.c_double(0.0)
    ctx.check(N.lib().wsr_euler3d_max_speed(ctx.handle, C.c_void_p(q.data_ptr()), nx, ny, nz, C.byref(out),
                                            C.c_void_p(ws.ptr), ws.nbytes,
                                            C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    return out.value


@dataclass
class RunResult3:
    steps: int
    t: float
    dts: np.ndarray
    ws: Workspace3


def run(q: torch.Tensor, nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, cfl: float,
        method: str = "js", flux: str = "evilin", mlp_params=None, inflow=None, t_end: float | None = None,
        steps: int | None = None, t_start: float = 0.0, opts: int = 0, ws: Workspace3 | None = None) -> RunResult3:
    """Advance q in place: to t_end (run_solver, solver.py:331-360), or exactly `steps` steps when t_end is
    None. dt = cfl min(dx, dy, dz) / max speed, clipped to t_end."""
    if t_end is None and steps is None:
        raise ValueError("give t_end or steps")
    _check(q, nx, ny, nz)
    dev = device_index(q.device)
    ctx = prepare_closure(method, mlp_params, dev)
    ws = _ws(ws, nx, ny, nz, q.device)
    keep, inf = _inflow(inflow)
    cap = steps if steps is not None else 1_000_000
    dts = np.zeros(cap)
    n_out, t_out = C.c_int(0), C.c_double(0.0)
    ctx.check(N.lib().wsr_euler3d_run(ctx.handle, C.c_void_p(q.data_ptr()), nx, ny, nz, dx, dy, dz, cfl, t_start,
                                      1.0e300 if t_end is None else float(t_end), cap, N.METHOD[method],
                                      N.FLUX3[flux], opts, inf, dts.ctypes.data_as(C.c_void_p), C.byref(n_out),
                                      C.byref(t_out), C.c_void_p(ws.ptr), ws.nbytes,
                                      C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    del keep
    return RunResult3(n_out.value, t_out.value, dts[:n_out.value].copy(), ws)


def counters(ws: Workspace3) -> dict[str, tuple[int, int]]:
    """(MLP, plateau) stencils of the last stage/run made with WSR_OPT_COUNT, per kernel class, and the JS
    fallbacks of the last stage/run made with OPT_JS_FALLBACK ("fallbacks")."""
    out = (C.c_ulonglong * 7)()
    ctx = N.context(device_index(ws.buf.device))
    nx, ny, nz = ws.shape
    ctx.check(N.lib().wsr_euler3d_counters(ctx.handle, C.c_void_p(ws.ptr), ws.nbytes, nx, ny, nz, out))
    return {"normal": (int(out[0]), int(out[1])), "transverse": (int(out[2]), int(out[3])),
            "flux": (int(out[4]), int(out[5])), "fallbacks": int(out[6])}
