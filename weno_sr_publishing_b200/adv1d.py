"""Batched 1D periodic advection with WENO5/WENO7 (JS or SR closure) on the GPU (libwsr.so).

Reference-shaped entry points (paths inside the reference project, code/snapshot/):

* ``ssprk3_step_signed(model, state, dt, dxinv, velocities)`` and
  ``rollout_distance(model, initial, distance_cells, cfl, velocities)`` --
  teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/rk3_advection.py:118-186;
* ``shu_rk4_step_signed(model, state, dt, dxinv, velocities)`` and
  ``rollout_signed(model, initial, n_steps, cfl, velocities, domain_length=1.0)`` --
  teacherfree_lab_weno7_rk4_distance_balanced_fast/rk4_advection.py:137-220;
* ``integrate_ssprk3(model, stepper, initial, cfl_limit, t_end, device)`` -- for_paper_results/run_gste.py:103-118.

``model`` is ``"classical"`` (Jiang-Shu weights), ``"z"`` (WENO-Z: p = 2, eps = dx^2 for WENO5; p = 3,
eps = dx^3 for WENO7; weno_z_borges_p2_results/torch_weno_z.py:14-32) or a closure: a :class:`Closure`, a
checkpoint path, or any object with ``w1 .. b4`` parameters (a reference torch model; float32 parameters select
the FP32 closure). ``state`` is a [B, N] tensor (or array); every row is one periodic trajectory.

``run_batched`` takes ragged trajectories (different N, velocity, dx and step schedule per row) in one
launch: one CTA per trajectory, all steps resident in shared memory.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _native as N

PARAM_NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")
NMAX = 2048
INTEG = {"ssprk3": 0, "shu_rk4": 1}


@dataclass(frozen=True)
class Closure:
    kind: int          # 5 (WENO5, 189 parameters) or 7 (WENO7, 908 parameters)
    packed: np.ndarray  # FP64 values in the packed w1 b1 ... b4 layout
    precision: str     # "f64", "f32" or "bf16"

    @property
    def method(self) -> str:
        return {"f64": "sr_f64", "f32": "sr_f32", "bf16": "sr_bf16"}[self.precision]

    @staticmethod
    def from_params(params, precision: str | None = None) -> "Closure":
        arrs = []
        dtype = None
        for k in PARAM_NAMES:
            v = params[k] if isinstance(params, dict) else getattr(params, k)
            if hasattr(v, "detach"):
                v = v.detach().cpu().numpy()
            v = np.asarray(v)
            dtype = dtype or v.dtype
            arrs.append(v.astype(np.float64).reshape(-1))
        packed = np.concatenate(arrs)
        kind = {189: 5, 908: 7}.get(packed.size)
        if kind is None:
            raise ValueError(f"{packed.size} parameters match neither WENO5 (189) nor WENO7 (908)")
        if precision is None:
            precision = "f32" if dtype == np.float32 else "f64"
        return Closure(kind, packed, precision)

    @staticmethod
    def from_checkpoint(path, precision: str | None = None) -> "Closure":
        data = np.load(Path(path), allow_pickle=True)
        missing = [k for k in PARAM_NAMES if k not in data.files]
        if missing:
            raise ValueError(f"{path} is missing arrays: {missing}")
        return Closure.from_params({k: data[k] for k in PARAM_NAMES}, precision)


def as_closure(model) -> Closure | None:
    if isinstance(model, str):
        if model not in ("classical", "z"):
            raise ValueError(f"unknown model {model!r}")
        return None
    if model is None:
        raise NotImplementedError("linear (d-weight) reconstruction is not provided; use 'classical' or a closure")
    if isinstance(model, Closure):
        return model
    if isinstance(model, (str, Path)):
        return Closure.from_checkpoint(model)
    return Closure.from_params(model)


def _workspace(device):
    nbytes = int(N.lib().wsr_adv1d_workspace_bytes())
    buf = torch.zeros(nbytes + 256, dtype=torch.uint8, device=device)
    ptr = (buf.data_ptr() + 255) // 256 * 256
    return buf, ptr, nbytes


def run_batched(states, velocities, dx, n_full, dt_full, dt_last=None, *, scheme: int = 5, model="classical",
                integrator: str = "ssprk3", device="cuda", opts: int = 0, count: bool = False, to_host: bool = False):
    """Advance ragged periodic trajectories; returns (list of final states, info): float64 device tensors, or with
    to_host=True float64 numpy arrays (one read-back of the whole batch, each array a view of it).

    states: list of 1D arrays/tensors (n_b cells each; host arrays go up in one copy); velocities, dx, dt_full,
    dt_last: per trajectory; n_full: full steps per trajectory (then one step of dt_last[b] when it is > 0)."""
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError("the 1D path runs on CUDA devices only")
    B = len(states)
    if B == 0:
        return [], {}
    closure = as_closure(model)
    if closure is not None:
        method = closure.method
    else:
        method = "z" if isinstance(model, str) and model == "z" else "js"
    if closure is not None and closure.kind != scheme:
        raise ValueError(f"a WENO{closure.kind} closure cannot drive the WENO{scheme} scheme")
    lens = [int(len(s)) for s in states]
    width = 5 if scheme == 5 else 7
    if min(lens) < width or max(lens) > NMAX:
        raise ValueError(f"every trajectory needs {width} <= n <= {NMAX} cells")
    if any(isinstance(s, torch.Tensor) and s.is_cuda for s in states):
        flat = torch.cat([torch.as_tensor(s, dtype=torch.float64).reshape(-1).to(dev) for s in states]).contiguous()
    else:  # host rows: concatenated on the host, one upload
        host_rows = [s.detach().numpy() if isinstance(s, torch.Tensor) else s for s in states]
        flat = torch.from_numpy(np.concatenate([np.asarray(s, dtype=np.float64).reshape(-1) for s in host_rows]))
        flat = flat.to(dev)
    offsets = torch.tensor(np.concatenate([[0], np.cumsum(lens)]), dtype=torch.int64, device=dev)
    vel = torch.as_tensor(np.asarray(velocities, dtype=np.float64).reshape(B), device=dev)
    dxs = torch.as_tensor(np.broadcast_to(np.asarray(dx, dtype=np.float64), (B,)).copy(), device=dev)
    nf = np.broadcast_to(np.asarray(n_full, dtype=np.int64), (B,)).astype(np.int32)
    dtf = np.broadcast_to(np.asarray(dt_full, dtype=np.float64), (B,)).copy()
    dtl = np.zeros(B) if dt_last is None else np.broadcast_to(np.asarray(dt_last, dtype=np.float64), (B,)).copy()
    cost = np.asarray(lens) * (nf + (dtl > 0))
    order = torch.as_tensor(np.argsort(-cost, kind="stable").astype(np.int32), device=dev)
    nf_t = torch.as_tensor(nf, device=dev)
    dtf_t = torch.as_tensor(dtf, device=dev)
    dtl_t = torch.as_tensor(dtl, device=dev)
    ctx = N.context(dev.index if dev.index is not None else torch.cuda.current_device())
    if closure is not None:
        ctx.upload_closure_kind(closure.kind, closure.packed)
    buf, wptr, wbytes = _workspace(dev)
    fb, err = C.c_int(0), C.c_int(0)
    cnt = (C.c_ulonglong * 2)()
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    P = C.c_void_p
    ctx.check(N.lib().wsr_adv1d_run(
        ctx.handle, P(flat.data_ptr()), P(offsets.data_ptr()), P(order.data_ptr()), P(vel.data_ptr()),
        P(dxs.data_ptr()), P(nf_t.data_ptr()), P(dtf_t.data_ptr()), P(dtl_t.data_ptr()), B, max(lens), scheme,
        N.METHOD[method], INTEG[integrator], int(opts) | (N.OPT_COUNT if count else 0), C.byref(fb), C.byref(err),
        cnt, P(wptr), wbytes, stream))
    if to_host:
        host = flat.cpu().numpy()
        edges = np.concatenate([[0], np.cumsum(lens)])
        outs = [host[edges[k]:edges[k + 1]] for k in range(B)]
    else:
        outs = list(torch.split(flat, lens))
    return outs, {"fallbacks": fb.value, "mlp": int(cnt[0]), "plateau": int(cnt[1])}


def shard_by_cost(cost, world: int, rank: int) -> np.ndarray:
    """Trajectories of `rank` when a batch is sharded over `world` ranks by cost (cells x steps of each
    trajectory): longest first, each to the rank with the least load so far (ties to the lower rank). Every
    trajectory lands on exactly one rank, every rank ends within one trajectory's cost of the mean, and every
    rank computes the same partition without communicating. Returns sorted indices."""
    cost = np.asarray(cost, dtype=np.float64).reshape(-1)
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    load = np.zeros(world)
    owner = np.empty(cost.size, dtype=np.int64)
    for b in np.argsort(-cost, kind="stable"):
        r = int(np.argmin(load))
        owner[b] = r
        load[r] += cost[b]
    return np.flatnonzero(owner == rank)


def _rows(state):
    t = torch.as_tensor(state, dtype=torch.float64)
    if t.ndim != 2:
        raise ValueError("state must be [B, N]")
    return t


def _uniform(model, state, velocities, dt, dxinv, steps, scheme, integrator):
    t = _rows(state)
    dev = t.device if t.is_cuda else torch.device("cuda")
    vel = torch.as_tensor(velocities, dtype=torch.float64).reshape(-1).cpu().numpy()
    B, n = t.shape
    outs, _ = run_batched([t[b] for b in range(B)], vel, 1.0 / dxinv, steps, dt, None, scheme=scheme, model=model,
                          integrator=integrator, device=dev)
    out = torch.stack(outs)
    return out if t.is_cuda else out.cpu()


def ssprk3_step_signed(model, state, dt: float, dxinv: float, velocities):
    """One SSPRK3 step of WENO5 with the signed upwind flux (rk3_advection.py:118-131)."""
    return _uniform(model, state, velocities, dt, dxinv, 1, 5, "ssprk3")


def shu_rk4_step_signed(model, state, dt: float, dxinv: float, velocities):
    """One Shu RK4 step of WENO7 with L and L~ (rk4_advection.py:137-195)."""
    return _uniform(model, state, velocities, dt, dxinv, 1, 7, "shu_rk4")


def cfl_schedule(distance_cells: float, cfl: float) -> tuple[float, ...]:
    """Full CFL steps plus one shortened step (rk3_advection.py:149-168)."""
    if distance_cells <= 0.0 or cfl <= 0.0:
        raise ValueError("distance_cells and cfl must be positive")
    full = int(math.floor(distance_cells / cfl))
    rem = distance_cells - full * cfl
    tol = 2.0e-13 * max(1.0, distance_cells)
    if rem < tol:
        rem = 0.0
    elif cfl - rem < tol:
        full += 1
        rem = 0.0
    sched = [float(cfl)] * full
    if rem > 0.0:
        sched.append(float(rem))
    if not sched:
        sched.append(float(distance_cells))
    if abs(sum(sched) - distance_cells) > 5.0e-12 * max(1.0, distance_cells):
        raise RuntimeError("CFL schedule does not reach the requested distance")
    return tuple(sched)


def _schedule_arrays(distance_cells: float, cfl: float):
    sched = cfl_schedule(distance_cells, cfl)
    full = sum(1 for s in sched if s == float(cfl))
    last = sched[-1] if sched[-1] != float(cfl) else 0.0
    if full + (1 if last > 0 else 0) != len(sched):  # the lone short step of a distance below one CFL step
        return 0, 0.0, sched[0]
    return full, float(cfl), last


def rollout_distance(model, initial, distance_cells: float, cfl: float, velocities):
    """Advance exactly distance_cells cell widths (rk3_advection.py:171-186)."""
    t = _rows(initial)
    B, n = t.shape
    dx = 1.0 / float(n)
    full, c_full, c_last = _schedule_arrays(distance_cells, cfl)
    dev = t.device if t.is_cuda else torch.device("cuda")
    vel = torch.as_tensor(velocities, dtype=torch.float64).reshape(-1).cpu().numpy()
    outs, _ = run_batched([t[b] for b in range(B)], vel, dx, full, c_full * dx, c_last * dx, scheme=5, model=model,
                          integrator="ssprk3", device=dev)
    out = torch.stack(outs)
    return out if t.is_cuda else out.cpu()


def rollout_signed(model, initial, n_steps: int, cfl: float, velocities, *, domain_length: float = 1.0):
    """n_steps Shu RK4 steps of WENO7 at dt = cfl dx (rk4_advection.py:198-220)."""
    t = _rows(initial)
    dx = float(domain_length) / float(t.shape[1])
    return _uniform(model, t, velocities, float(cfl) * dx, 1.0 / dx, n_steps, 7, "shu_rk4")


def integrate_ssprk3(model, stepper, initial, cfl_limit: float, t_end: float, device="cuda", length: float = 2.0):
    """GSTE integration (run_gste.py:103-118): steps = ceil(t_end / (cfl dx)), dt = t_end / steps.

    stepper: ssprk3_step_signed (WENO5) or shu_rk4_step_signed (WENO7); velocity +1."""
    u0 = np.asarray(initial, dtype=np.float64)
    nx = u0.size
    dx = length / nx
    steps = int(math.ceil(t_end / (cfl_limit * dx)))
    dt = t_end / steps
    scheme, integ = (7, "shu_rk4") if stepper is shu_rk4_step_signed else (5, "ssprk3")
    outs, _ = run_batched([u0], [1.0], dx, steps, dt, None, scheme=scheme, model=model, integrator=integ,
                          device=device)
    return outs[0].cpu().numpy(), {"steps": steps, "dt": dt, "cfl": dt / dx, "t": t_end}
