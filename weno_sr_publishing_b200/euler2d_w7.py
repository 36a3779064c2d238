"""2D Euler WENO7 (JS, Z or SR weights) with Shu's fourth-order TVD Runge-Kutta on the GPU (libwsr.so underneath).

The reference's point-value WENO7 path (weno7_point_rk4_shu/point_rk4.py): characteristic WENO7 normal
reconstruction, conservative two-point Gauss WENO7 transverse reconstruction, HLLC, and Shu's RK4 with the
downwind operator. States use the reference's padded layout [(ny+8), (nx+8), 4] FP64 (ghost width 4).
Method "sr_f64" is the paper's WENO7-SR-RK4 (teacherfree_lab_weno7_rk4_distance_balanced_fast/warp_sod/
point_rk4_mlp.py): betas from the FP64 WENO7 closure, evaluated inside the reconstruction kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _native as N
from .adv1d import Closure

_ALIGN = 256
GHOST = 4
BC = {"transmissive": 0, "outflow": 0, "periodic": 1}
# "js": classical WENO7 weights; "z": WENO-Z (p = 3, betas / 240, eps = h^3 per direction); "sr_f64": betas of
# the FP64 WENO7 closure (needs `closure`)
METHOD = {"js": 0, "z": 4, "sr_f64": 1}


@dataclass(frozen=True)
class Params:
    """point_rk4.Params (point_rk4.py:25-57): the domain is [x_min, x_max] x [y_min, y_max]."""
    nx: int
    ny: int
    x_min: float = -10.0
    x_max: float = 10.0
    y_min: float = -10.0
    y_max: float = 10.0
    ghost: int = GHOST
    gamma: float = 1.4
    cfl: float = 0.4
    t_end: float = 2.0

    @property
    def x_length(self) -> float:
        return self.x_max - self.x_min

    @property
    def y_length(self) -> float:
        return self.y_max - self.y_min

    @property
    def dx(self) -> float:
        return self.x_length / float(self.nx)

    @property
    def dy(self) -> float:
        return self.y_length / float(self.ny)

    @property
    def padded_shape(self) -> tuple[int, int, int]:
        return (self.ny + 2 * self.ghost, self.nx + 2 * self.ghost, 4)


@dataclass
class Workspace:
    buf: torch.Tensor
    ptr: int
    nbytes: int


def workspace(nx: int, ny: int, device="cuda") -> Workspace:
    nbytes = int(N.lib().wsr_euler2d_w7_workspace_bytes(nx, ny))
    if nbytes == 0:
        raise ValueError(f"invalid grid {nx} x {ny}")
    buf = torch.empty(nbytes + _ALIGN, dtype=torch.uint8, device=device)
    return Workspace(buf, (buf.data_ptr() + _ALIGN - 1) // _ALIGN * _ALIGN, nbytes)


def _check(u: torch.Tensor, p: Params) -> None:
    if not isinstance(u, torch.Tensor) or u.dtype != torch.float64 or not u.is_cuda:
        raise TypeError("state must be a float64 CUDA tensor")
    if tuple(u.shape) != p.padded_shape or not u.is_contiguous():
        raise ValueError(f"state must be contiguous with shape {p.padded_shape}, got {tuple(u.shape)}")
    if p.ghost != GHOST:
        raise ValueError("the WENO7 path uses 4 ghost cells")


def _bc(boundary: str) -> int:
    if boundary not in BC:
        raise ValueError(f"unsupported boundary {boundary!r}")
    return BC[boundary]


def _stream(dev: int):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _method(method: str) -> int:
    if method not in METHOD:
        raise ValueError(f"unsupported WENO7 method {method!r}")
    return METHOD[method]


def as_closure7(closure) -> Closure:
    """A WENO7 closure from a Closure, a checkpoint path or a {w1..b4} dict (6 -> 24 -> 16 -> 16 -> 4)."""
    if isinstance(closure, Weno7PointBeta):
        closure = closure.closure
    elif isinstance(closure, (str, Path)):
        closure = Closure.from_checkpoint(closure, "f64")
    elif not isinstance(closure, Closure):
        closure = Closure.from_params(closure, "f64")
    if closure.kind != 7:
        raise ValueError(f"the WENO7 path needs a WENO7 closure (908 parameters), got {closure.packed.size}")
    return closure


def _prepare(ctx, method: str, closure) -> int:
    m = _method(method)
    if method == "sr_f64":
        if closure is None:
            raise ValueError("method 'sr_f64' needs a WENO7 closure")
        ctx.upload_closure_kind(7, as_closure7(closure).packed)
    return m


class Weno7PointBeta:
    """The WENO7 closure of a checkpoint, in the place of the reference's torch beta provider
    (TorchWeno7PointBeta(model_path, torch_device, gamma), point_rk4_mlp.py:30-63): here the betas are
    evaluated inside the reconstruction kernels, so the object only carries the parameters."""

    def __init__(self, model_path, torch_device: str = "cuda", gamma: float = 1.4):
        self.closure = as_closure7(Closure.from_checkpoint(Path(model_path), "f64"))
        self.device = torch.device(torch_device)
        self.gamma = float(gamma)


def _opts(method: str, js_fallback: bool) -> int:
    if js_fallback and method != "sr_f64":
        raise ValueError("js_fallback applies to method 'sr_f64' only")
    return N.OPT_JS_FALLBACK if js_fallback else 0


def rhs(u: torch.Tensor, params: Params, boundary: str = "periodic", reverse: bool = False,
        ws: Workspace | None = None, method: str = "js", closure=None, js_fallback: bool = False) -> torch.Tensor:
    """L(u) (or the downwind L~(u)) on the interior, shape [ny, nx, 4] (compute_rhs, point_rk4.py:435-511;
    compute_rhs_mlp, point_rk4_mlp.py:198-277, for method "sr_f64"). js_fallback: WENO7-JS weights where the
    closure's betas are not finite or a normal face state loses positivity (counted in closure_counts)."""
    _check(u, params)
    bc = _bc(boundary)
    dev = u.device.index
    ctx = N.context(dev)
    m = _prepare(ctx, method, closure)
    ws = ws or workspace(params.nx, params.ny, u.device)
    out = torch.empty((params.ny, params.nx, 4), dtype=torch.float64, device=u.device)
    ctx.check(N.lib().wsr_euler2d_w7_rhs(ctx.handle, C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()),
                                         params.nx, params.ny, params.dx, params.dy, params.gamma, bc,
                                         m, int(bool(reverse)), _opts(method, js_fallback), C.c_void_p(ws.ptr),
                                         ws.nbytes, _stream(dev)))
    return out


@dataclass
class RunResult:
    dts: list
    steps: int
    t: float


def run(u: torch.Tensor, params: Params, boundary: str = "periodic", t_end: float | None = None,
        max_steps: int = 10_000_000, t_start: float = 0.0, ws: Workspace | None = None,
        method: str = "js", closure=None, js_fallback: bool = False) -> RunResult:
    """Advance u in place from t_start to t_end with the device-resident Shu RK4 loop (run_from_initial's
    stopping rule). js_fallback as in rhs."""
    _check(u, params)
    bc = _bc(boundary)
    dev = u.device.index
    ctx = N.context(dev)
    m = _prepare(ctx, method, closure)
    ws = ws or workspace(params.nx, params.ny, u.device)
    t_end = params.t_end if t_end is None else float(t_end)
    cap = min(int(max_steps), 1 << 22)
    dts = np.zeros(cap)
    steps, t = C.c_int(0), C.c_double(0.0)
    ctx.check(N.lib().wsr_euler2d_w7_run(
        ctx.handle, C.c_void_p(u.data_ptr()), params.nx, params.ny, params.dx, params.dy, params.gamma, params.cfl,
        float(t_start), t_end, bc, m, _opts(method, js_fallback), cap, dts.ctypes.data_as(C.POINTER(C.c_double)),
        C.byref(steps), C.byref(t), C.c_void_p(ws.ptr), ws.nbytes, _stream(dev)))
    return RunResult([float(x) for x in dts[:steps.value]], steps.value, t.value)


def closure_counts(ws: Workspace, params: Params, device=None) -> dict[str, int]:
    """Closure evaluations (stencils that ran the MLP pair) of the last rhs / run on `ws` ("sr_f64"), per kernel
    class, and the JS fallbacks taken ("fallbacks")."""
    out = (C.c_ulonglong * 5)()
    ctx = N.context(torch.device(device).index if device is not None else ws.buf.device.index)
    ctx.check(N.lib().wsr_euler2d_w7_counters(ctx.handle, C.c_void_p(ws.ptr), ws.nbytes, params.nx, params.ny, out))
    return dict(zip(("normal_x", "normal_y", "flux_x", "flux_y", "fallbacks"), (int(v) for v in out)))


def interior_stats(u_host: np.ndarray, params: Params) -> dict[str, float]:
    """point_rk4.interior_stats (point_rk4.py:120-133)."""
    g = params.ghost
    q = u_host[g:g + params.ny, g:g + params.nx, :]
    rho = np.maximum(q[..., 0], 1.0e-15)
    u, v = q[..., 1] / rho, q[..., 2] / rho
    p = (params.gamma - 1.0) * (q[..., 3] - 0.5 * rho * (u * u + v * v))
    return {"mass": float(np.sum(q[..., 0]) * params.dx * params.dy), "rho_min": float(np.nanmin(rho)),
            "rho_max": float(np.nanmax(rho)), "p_min": float(np.nanmin(p)), "p_max": float(np.nanmax(p)),
            "nan_count": float(np.isnan(q).sum()), "rho_neg": float(np.sum(rho <= 0.0)),
            "p_neg": float(np.sum(p <= 0.0))}


def run_from_initial(u0: np.ndarray, params: Params, *, device: str = "cuda", riemann_solver: str = "hllc",
                     characteristic: bool = True, report_interval: int = 0, max_steps: int = 10_000_000,
                     boundary: str = "periodic", method: str = "js", closure=None,
                     _label: str = "") -> tuple[np.ndarray, dict]:
    """point_rk4.run_from_initial (point_rk4.py:568-616): numpy in, (final padded state, summary) out.
    method "z" is weno7_point_rk4_z.run_from_initial with weight_kind 1 (the reference's WENO7-Z runs).

    Only the characteristic HLLC configuration of the paper runs is provided; the EVILIN flux and the
    conservative-variable normal reconstruction raise NotImplementedError."""
    if riemann_solver != "hllc":
        raise NotImplementedError("the WENO7 2D path provides the HLLC flux only")
    if not characteristic:
        raise NotImplementedError("the WENO7 2D path provides characteristic normal reconstruction only")
    dev = torch.device(device)
    if method == "sr_f64":
        closure = as_closure7(closure) if closure is not None else None
    u = torch.as_tensor(np.ascontiguousarray(u0, dtype=np.float64), device=dev).clone()
    ws = workspace(params.nx, params.ny, dev)
    if report_interval > 0:
        dts, t, steps = [], 0.0, 0
        while t < params.t_end and steps < max_steps:
            chunk = 1 if steps == 0 else report_interval - steps % report_interval
            res = run(u, params, boundary, max_steps=min(chunk, max_steps - steps), t_start=t, ws=ws,
                      method=method, closure=closure)
            if res.steps == 0:
                break
            dts += res.dts
            steps += res.steps
            t = res.t
            stats = interior_stats(u.cpu().numpy(), params)
            print(f"{_label}N={params.nx} step={steps:05d} t={t:.8e} dt={dts[-1]:.8e} "
                  f"rho=[{stats['rho_min']:.6e},{stats['rho_max']:.6e}] "
                  f"p=[{stats['p_min']:.6e},{stats['p_max']:.6e}] nan={int(stats['nan_count'])}", flush=True)
            if stats["nan_count"] or stats["rho_neg"] or stats["p_neg"]:
                break
    else:
        res = run(u, params, boundary, max_steps=max_steps, ws=ws, method=method, closure=closure)
        dts, steps, t = res.dts, res.steps, res.t
    final = u.cpu().numpy()
    return final, {"steps": int(steps), "t": float(t), "dt_min": float(np.min(dts)) if dts else 0.0,
                   "dt_max": float(np.max(dts)) if dts else 0.0, "dt_mean": float(np.mean(dts)) if dts else 0.0,
                   **interior_stats(final, params)}


def run_from_initial_mlp(u0: np.ndarray, params: Params, *, device: str = "cuda", riemann_solver: str = "hllc",
                         beta_model, report_interval: int = 0, max_steps: int = 10_000_000,
                         boundary: str = "periodic", eno_cutoff: bool = False) -> tuple[np.ndarray, dict]:
    """point_rk4_mlp.run_from_initial_mlp (warp_sod/point_rk4_mlp.py:300-362): WENO7-SR with Shu RK4.
    beta_model: a Weno7PointBeta, a Closure, a checkpoint path or a {w1..b4} dict. The ENO cutoff (off in the
    paper runs) raises NotImplementedError."""
    if eno_cutoff:
        raise NotImplementedError("the WENO7-SR 2D path provides eno_cutoff=False only")
    return run_from_initial(u0, params, device=device, riemann_solver=riemann_solver, characteristic=True,
                            report_interval=report_interval, max_steps=max_steps, boundary=boundary,
                            method="sr_f64", closure=beta_model, _label="MLP-RK4 ")
