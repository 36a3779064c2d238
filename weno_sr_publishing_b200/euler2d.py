"""Torch-facing driver of the 2D Euler WENO5 path (libwsr.so underneath).

PyTorch provides device memory and streams; every numerical operation runs in the CUDA kernels
behind the C ABI. Arrays use the reference's padded layout [(ny+6), (nx+6), 4] FP64.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .params import Params

_ALIGN = 256


def device_index(device) -> int:
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError(f"the 2D path runs on CUDA devices only (got {device!r})")
    return torch.cuda.current_device() if d.index is None else d.index


def _stream_ptr(dev: int):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


@dataclass
class Workspace:
    buf: torch.Tensor
    ptr: int
    nbytes: int
    nx: int
    ny: int


def workspace(nx: int, ny: int, device="cuda") -> Workspace:
    """Device scratch for one 2D grid: face values, fluxes and the step-control block."""
    nbytes = int(N.lib().wsr_euler2d_workspace_bytes(nx, ny))
    if nbytes == 0:
        raise ValueError(f"invalid grid {nx} x {ny}")
    buf = torch.empty(nbytes + _ALIGN, dtype=torch.uint8, device=device)
    ptr = (buf.data_ptr() + _ALIGN - 1) // _ALIGN * _ALIGN
    return Workspace(buf, ptr, nbytes, nx, ny)


def _check_state(u: torch.Tensor, p: Params) -> None:
    if not isinstance(u, torch.Tensor) or u.dtype != torch.float64 or not u.is_cuda:
        raise TypeError("state must be a float64 CUDA tensor")
    if tuple(u.shape) != p.padded_shape or not u.is_contiguous():
        raise ValueError(f"state must be contiguous with shape {p.padded_shape}, got {tuple(u.shape)}")
    if p.ghost != 3:
        raise ValueError("the 2D path uses 3 ghost cells")


def prepare_closure(method: str, mlp_params, dev: int) -> N.Context:
    ctx = N.context(dev)
    if method not in N.METHOD:
        raise ValueError(f"unknown method {method!r}")
    if method in N.SR_METHODS:
        if mlp_params is None:
            raise ValueError(f"method {method!r} needs mlp_params")
        ctx.upload_closure(N.pack_params(mlp_params))
    return ctx


def stage(u_stage: torch.Tensor, u0: torch.Tensor, u_out: torch.Tensor, params: Params, dt: float, rk: int,
          method: str, boundary: str, mlp_params=None, flux: str = "hllc", opts: int = 0,
          ws: Workspace | None = None, boundary_time: float = 0.0, y_halo: bool = False) -> None:
    """One SSPRK3 stage into the interior of u_out (launch_stage of the reference adapters); the
    double-Mach boundary is evaluated at boundary_time. y_halo: the y ghost rows of u_stage are read as stored
    (a slab of a y-decomposed grid, WSR_BC_Y_HALO)."""
    for t in (u_stage, u0, u_out):
        _check_state(t, params)
    if boundary not in N.BC:
        raise ValueError(f"unsupported boundary {boundary!r}")
    dev = u_stage.device.index
    ctx = prepare_closure(method, mlp_params, dev)
    ws = ws or workspace(params.nx, params.ny, u_stage.device)
    ctx.check(N.lib().wsr_euler2d_stage_at(
        ctx.handle, C.c_void_p(u_stage.data_ptr()), C.c_void_p(u0.data_ptr()), C.c_void_p(u_out.data_ptr()),
        params.nx, params.ny, params.dx, params.dy, params.gamma, float(dt), int(rk), N.METHOD[method],
        N.BC[boundary] | (N.BC_Y_HALO if y_halo else 0), N.FLUX[flux], int(opts), float(boundary_time),
        C.c_void_p(ws.ptr), ws.nbytes,
        _stream_ptr(dev)))


def max_speed(u: torch.Tensor, params: Params, ws: Workspace | None = None) -> float:
    _check_state(u, params)
    dev = u.device.index
    ctx = N.context(dev)
    ws = ws or workspace(params.nx, params.ny, u.device)
    out = C.c_double(0.0)
    ctx.check(N.lib().wsr_euler2d_max_speed(ctx.handle, C.c_void_p(u.data_ptr()), params.nx, params.ny,
                                            params.gamma, C.byref(out), C.c_void_p(ws.ptr), ws.nbytes,
                                            _stream_ptr(dev)))
    return out.value


def compute_dt(u: torch.Tensor, params: Params, ws: Workspace | None = None) -> float:
    """compute_dt_from_warp_array (warp_weno5_helpers.py:189-207)."""
    m = max_speed(u, params, ws)
    if m < 1.0e-15:
        return 1.0e10
    return params.cfl * min(params.dx, params.dy) / m


def counters(ws: Workspace) -> dict[str, tuple[int, int]]:
    """Per kernel class: (MLP closure evaluations, plateau stencils) of the last call made with OPT_COUNT."""
    out = (C.c_ulonglong * 8)()
    ctx = N.context(ws.buf.device.index)
    ctx.check(N.lib().wsr_euler2d_counters(ctx.handle, C.c_void_p(ws.ptr), ws.nbytes, ws.nx, ws.ny, out))
    return {k: (int(out[2 * i]), int(out[2 * i + 1])) for i, k in enumerate(("normal_x", "normal_y", "flux_x",
                                                                              "flux_y"))}


@dataclass
class RunResult:
    final_slot: int
    dts: list
    steps: int
    t: float
    fallbacks: int


def run(bufs: list, params: Params, t_end: float, method: str, boundary: str, mlp_params=None, flux: str = "hllc",
        opts: int = 0, check_health: bool = False, check_interval: int = 0, fixed_steps: int = 0,
        max_steps: int = 1 << 20, t_start: float = 0.0, ws: Workspace | None = None) -> RunResult:
    """Device-resident time loop over four state buffers (see wsr_euler2d_run)."""
    if len(bufs) != 4:
        raise ValueError("run needs four state buffers")
    for t in bufs:
        _check_state(t, params)
    if boundary not in N.BC:
        raise ValueError(f"unsupported boundary {boundary!r}")
    dev = bufs[0].device.index
    ctx = prepare_closure(method, mlp_params, dev)
    ws = ws or workspace(params.nx, params.ny, bufs[0].device)
    cap = fixed_steps if fixed_steps > 0 else max_steps
    dts = np.zeros(max(cap, 1))
    ptrs = (C.c_void_p * 4)(*[b.data_ptr() for b in bufs])
    steps, slot, fb = C.c_int(0), C.c_int(0), C.c_int(0)
    t = C.c_double(0.0)
    ctx.check(N.lib().wsr_euler2d_run(
        ctx.handle, ptrs, params.nx, params.ny, params.dx, params.dy, params.gamma, params.cfl, float(t_start),
        float(t_end), N.METHOD[method], N.BC[boundary], N.FLUX[flux], int(opts), int(bool(check_health)),
        int(check_interval), int(fixed_steps), int(cap), dts.ctypes.data_as(C.POINTER(C.c_double)), C.byref(steps),
        C.byref(t), C.byref(slot), C.byref(fb), C.c_void_p(ws.ptr), ws.nbytes, _stream_ptr(dev)))
    return RunResult(slot.value, [float(x) for x in dts[:steps.value]], steps.value, t.value, fb.value)


def advance_host(u_host, params: Params, steps: int, method: str, boundary: str, mlp_params=None,
                 bufs: list | None = None, ws: Workspace | None = None, device="cuda",
                 async_readback: bool = False, bands: int = 0):
    """Host-buffer entry (wsr_euler2d_advance_host): copy the interior of the padded host state to the device,
    run `steps` full CFL steps (bit for bit the device loop's), copy the result's interior back into u_host (in
    place; its ghost cells are left as they are), and return u_host.

    The copies run in row bands on the library's own copy streams: the first stage's wave speed and (transmissive
    boundary) normal reconstructions follow the upload band by band, and the last stage runs band by band with
    each band's read-back starting as soon as its rows are final. By default the call returns when u_host holds
    the result. With async_readback=True (pinned host memory) it returns once queued: consecutive calls on the
    same host array and `bufs` then overlap both copy directions with the computation, and u_host is complete
    after host_copies_done() (which orders the current stream after the read-backs) and a synchronisation, or
    after host_wait(). bands: 0 picks one band per 250 rows (at most 16; the first and last are half as high)."""
    dev = torch.device(device)
    if bufs is None:
        bufs = [torch.empty(params.padded_shape, dtype=torch.float64, device=dev) for _ in range(4)]
    for b in bufs:
        _check_state(b, params)
    host = torch.from_numpy(u_host) if isinstance(u_host, np.ndarray) else u_host
    if host.dtype != torch.float64 or host.is_cuda or tuple(host.shape) != tuple(params.padded_shape) \
            or not host.is_contiguous():
        raise ValueError(f"u_host must be a contiguous float64 host array of shape {tuple(params.padded_shape)}")
    if boundary not in N.BC:
        raise ValueError(f"unsupported boundary {boundary!r}")
    ctx = prepare_closure(method, mlp_params, device_index(dev))
    ws = ws or workspace(params.nx, params.ny, dev)
    ptrs = (C.c_void_p * 4)(*[b.data_ptr() for b in bufs])
    flags = N.HOST_ASYNC if async_readback else 0
    ctx.check(N.lib().wsr_euler2d_advance_host(
        ctx.handle, C.c_void_p(host.data_ptr()), ptrs, params.nx, params.ny, params.dx, params.dy, params.gamma,
        params.cfl, int(steps), N.METHOD[method], N.BC[boundary], N.FLUX["hllc"], 0, flags, int(bands),
        C.c_void_p(ws.ptr), ws.nbytes, _stream_ptr(dev)))
    return u_host


def host_copies_done(device="cuda") -> None:
    """Make the current stream wait for every read-back advance_host(async_readback=True) has issued on
    `device` (work or events recorded on the current stream afterwards come after them)."""
    dev = torch.device(device)
    ctx = N.context(device_index(dev))
    ctx.check(N.lib().wsr_euler2d_host_order(ctx.handle, _stream_ptr(dev)))


def host_wait(device="cuda") -> dict:
    """Wait for every advance_host call on `device` and its read-back; returns the steps taken and the JS
    fallbacks summed over the calls since the previous wait, and raises an error any of them met on the device."""
    dev = torch.device(device)
    ctx = N.context(device_index(dev))
    steps, fb = C.c_int(0), C.c_int(0)
    ctx.check(N.lib().wsr_euler2d_host_wait(ctx.handle, C.byref(steps), C.byref(fb)))
    return {"steps": steps.value, "fallbacks": fb.value}
