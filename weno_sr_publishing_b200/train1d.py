"""Closure training through 1D periodic advection trajectories on the GPU (libwsr.so).

Reference (code/snapshot/teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/):

* ``ClosureMLP`` -- the WENO5 closure parameters w1..b4 with the reference's seeded initialisation
  (weno5_core.py:25-48 ``SharedBadnessMLP``: normal(0, sqrt(1/fan_in)) hidden weights drawn from a CPU
  torch generator in FP64, zero biases, zero last layer, so the initial operator is the linear-weight
  WENO5), in FP64 or, like model.py:29-42, FP32;
* ``trajectory_loss(model, batch)`` -- the training objective of fast_losses.py:412-648 restricted to its
  state term: the mean L1 distance to the exact cell averages at every completed SSPRK3 step of the
  rollout, differentiable through ``torch.autograd``; forward and backward are the CUDA kernels
  (``wsr_train1d_forward`` / ``wsr_train1d_backward``, a hand-written adjoint with checkpoints every
  ``ckpt_every`` steps);
* ``train(...)`` -- the driver of train.py:261-659: shuffled distance cycle, Adam with the cosine
  learning-rate schedule, gradient clipping and skipping, npz checkpoints in the reference format and
  resumable training state;
* ``final_state_error_signed`` -- the evaluation of rk3_advection.py:533-560 (rollout to a distance,
  error against the exact averages with the reference's per-sample L4 + 0.05 relative-L2 measure).
"""
from __future__ import annotations

import csv
import ctypes as C
import json
import math
import os
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _native as N
from . import adv1d
from . import checkpoint as ckpt
from . import profiles as prof

PARAM_SHAPES = {"w1": (5, 10), "b1": (10,), "w2": (10, 6), "b2": (6,), "w3": (6, 6), "b3": (6,), "w4": (6, 3),
                "b4": (3,)}
PARAM_NAMES = tuple(PARAM_SHAPES)
DISTANCES = (2, 8, 64, 128, 256, 512, 1024)
PRECISION_METHOD = {"f64": "sr_f64", "f32": "sr_f32"}


class ClosureMLP(torch.nn.Module):
    """WENO5 closure parameters (5 -> 10 -> 6 -> 6 -> 3), initialised like the reference.

    The weights are drawn in FP64 from ``torch.Generator().manual_seed(seed)`` in the order w1, w2, w3
    (weno5_core.py:28-48); FP32 models quantise that draw (model.py:38-42)."""

    def __init__(self, seed: int = 41, dtype: torch.dtype = torch.float64):
        super().__init__()
        gen = torch.Generator(device="cpu")
        gen.manual_seed(seed)
        fan = {"w1": 5, "w2": 10, "w3": 6}
        for name, shape in PARAM_SHAPES.items():
            if name in fan:
                v = torch.randn(shape, generator=gen, dtype=torch.float64) * np.sqrt(1.0 / fan[name])
            else:
                v = torch.zeros(shape, dtype=torch.float64)
            setattr(self, name, torch.nn.Parameter(v.to(dtype)))

    @property
    def precision(self) -> str:
        return "f32" if self.w1.dtype == torch.float32 else "f64"

    def packed(self) -> torch.Tensor:
        return torch.cat([getattr(self, k).reshape(-1) for k in PARAM_NAMES])

    def params(self) -> dict:
        return {k: getattr(self, k) for k in PARAM_NAMES}

    def closure(self, precision: str | None = None) -> adv1d.Closure:
        return adv1d.Closure.from_params(self.params(), precision or self.precision)

    @classmethod
    def from_checkpoint(cls, path, dtype: torch.dtype = torch.float64) -> "ClosureMLP":
        data = np.load(Path(path), allow_pickle=True)
        m = cls(seed=0, dtype=dtype)
        with torch.no_grad():
            for k in PARAM_NAMES:
                getattr(m, k).copy_(torch.as_tensor(np.asarray(data[k]).reshape(PARAM_SHAPES[k]), dtype=dtype))
        return m


def balanced_velocities(batch: int) -> np.ndarray:
    """+1 for the first half of the batch, -1 for the second (rk3_advection.py:27-34)."""
    if batch < 2 or batch % 2:
        raise ValueError("bidirectional batches must be positive and even")
    v = np.ones(batch)
    v[batch // 2:] = -1.0
    return v


def steps_for_distance(distance: float, cfl: float) -> int:
    """train.py:103-111: the distance must be a whole number of full SSPRK3 steps."""
    raw = float(distance) / float(cfl)
    k = int(round(raw))
    if k < 1 or abs(raw - k) > 1.0e-12:
        raise ValueError(f"distance={distance:g} must contain an integer number of full SSPRK3 steps at CFL={cfl:g}")
    return k


@dataclass
class TrajectoryBatch:
    """B trajectories of n cells: profiles (desc [B, 34]) and velocities on the device, `steps` SSPRK3
    steps of dt = cfl / n. u0 = None starts from the exact cell averages of the profiles."""
    desc: torch.Tensor
    velocity: torch.Tensor
    n: int
    steps: int
    dt: float
    u0: torch.Tensor | None = None
    ckpt_every: int = 32

    @property
    def B(self) -> int:
        return int(self.desc.shape[0])

    @property
    def dx(self) -> float:
        return 1.0 / float(self.n)

    @staticmethod
    def sample(rng: np.random.Generator, batch: int, n: int, distance_cells: float, cfl: float = 0.5,
               device="cuda", ckpt_every: int = 32, family: str | None = None) -> "TrajectoryBatch":
        desc, _ = prof.make_profiles(rng, batch, n, family)
        dev = torch.device(device)
        return TrajectoryBatch(torch.as_tensor(desc, device=dev), torch.as_tensor(balanced_velocities(batch), device=dev),
                               n, steps_for_distance(distance_cells, cfl), float(cfl) / float(n), None, ckpt_every)


_workspaces: dict = {}


def _workspace(device: torch.device, nbytes: int) -> tuple[torch.Tensor, int]:
    key = device.index if device.index is not None else torch.cuda.current_device()
    buf = _workspaces.get(key)
    if buf is None or buf.numel() < nbytes + 256:
        _workspaces[key] = None
        buf = torch.empty(nbytes + 256, dtype=torch.uint8, device=device)
        _workspaces[key] = buf
    return buf, (buf.data_ptr() + 255) // 256 * 256


def _ptr(t: torch.Tensor | None) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


class _Run:
    """Forward state kept for the backward call: the workspace holds checkpoints and loss signs."""

    def __init__(self, batch: TrajectoryBatch, packed: np.ndarray, precision: str):
        self.batch, self.packed, self.precision = batch, packed, precision
        dev = batch.desc.device
        if dev.type != "cuda":
            raise ValueError("training runs on CUDA devices only")
        self.device = dev
        self.ctx = N.context(dev.index if dev.index is not None else torch.cuda.current_device())
        self.nbytes = int(N.lib().wsr_train1d_workspace_bytes(batch.B, batch.n, batch.steps, batch.ckpt_every))
        self.buf, self.ws = _workspace(dev, self.nbytes)
        self.method = N.METHOD[PRECISION_METHOD[precision]]

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, want_final: bool = False):
        b = self.batch
        self.ctx.upload_closure_kind(5, self.packed)
        loss = torch.empty((), dtype=torch.float64, device=self.device)
        final = torch.empty((b.B, b.n), dtype=torch.float64, device=self.device) if want_final else None
        u0 = None if b.u0 is None else b.u0.to(dtype=torch.float64).contiguous()
        self.ctx.check(N.lib().wsr_train1d_forward(
            self.ctx.handle, _ptr(u0), _ptr(b.desc.contiguous()), _ptr(b.velocity.contiguous()), b.B, b.n, b.dx, b.dt,
            b.steps, b.ckpt_every, self.method, _ptr(loss), _ptr(final), C.c_void_p(self.ws), self.nbytes,
            self._stream()))
        return loss, final

    def backward(self, want_u0: bool = False):
        b = self.batch
        self.ctx.upload_closure_kind(5, self.packed)
        grad = torch.empty(N.N_PARAMS5, dtype=torch.float64, device=self.device)
        gu0 = torch.empty((b.B, b.n), dtype=torch.float64, device=self.device) if want_u0 else None
        self.ctx.check(N.lib().wsr_train1d_backward(
            self.ctx.handle, _ptr(b.velocity.contiguous()), b.B, b.n, b.dx, b.dt, b.steps, b.ckpt_every, self.method,
            _ptr(grad), _ptr(gu0), C.c_void_p(self.ws), self.nbytes, self._stream()))
        return grad, gu0


class _TrajectoryLossFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, packed: torch.Tensor, batch: TrajectoryBatch, precision: str):
        run = _Run(batch, packed.detach().to(torch.float64).cpu().numpy(), precision)
        loss, _ = run.forward()
        ctx.run = run
        ctx.param_dtype = packed.dtype
        return loss

    @staticmethod
    def backward(ctx, g):
        grad, _ = ctx.run.backward()
        ctx.run = None
        return (grad * g).to(ctx.param_dtype), None, None


def trajectory_loss(model: ClosureMLP, batch: TrajectoryBatch) -> torch.Tensor:
    """Mean |u_k - e_k| over trajectories, completed steps k = 1..steps and cells, as a 0-d tensor on the
    device whose backward runs the CUDA adjoint into the model's parameter gradients."""
    packed = model.packed()
    flat = _TrajectoryLossFn.apply(packed, batch, model.precision)
    return flat


def loss_and_grads(packed: np.ndarray, batch: TrajectoryBatch, precision: str = "f64", want_u0: bool = False):
    """One forward + backward without autograd: (loss, dL/dtheta [189], dL/du0 or None, final states)."""
    run = _Run(batch, np.ascontiguousarray(packed, dtype=np.float64), precision)
    loss, final = run.forward(want_final=True)
    grad, gu0 = run.backward(want_u0=want_u0)
    return loss, grad, gu0, final


# ------------------------------------------------------------------------------------------------
# Evaluation (rk3_advection.py:134-146, 533-560)
# ------------------------------------------------------------------------------------------------
def state_error_per_sample(prediction, exact, qscale, value_range):
    absolute = (prediction - exact) / qscale[:, None]
    relative = (prediction - exact) / value_range[:, None]
    l4 = np.sqrt(np.mean(np.abs(absolute) ** 4, axis=1) + 1.0e-30)
    return l4 + 0.05 * np.mean(relative ** 2, axis=1)


def final_state_error_signed(model, desc: np.ndarray, n: int, distance_cells: float, cfl: float,
                             velocities: np.ndarray, device="cuda") -> tuple[float, float, float]:
    """(mean, mean over a > 0, mean over a < 0) of the per-sample error after advecting distance_cells."""
    initial = prof.cell_averages(desc, n, 0.0)
    vel = np.asarray(velocities, dtype=np.float64)
    t = torch.as_tensor(initial, device=device)
    final = adv1d.rollout_distance(model, t, distance_cells, cfl, torch.as_tensor(vel)).cpu().numpy()
    exact = prof.cell_averages(desc, n, np.where(vel > 0, 1.0, -1.0) * (distance_cells / float(n)))
    qscale = np.maximum(np.abs(initial).max(axis=1), 1.0)
    vrange = np.maximum(initial.max(axis=1) - initial.min(axis=1), 1.0e-6 * qscale)
    err = state_error_per_sample(final, exact, qscale, vrange)
    return float(err.mean()), float(err[vel > 0].mean()), float(err[vel < 0].mean())


# ------------------------------------------------------------------------------------------------
# Training driver (train.py:80-111, 261-659)
# ------------------------------------------------------------------------------------------------
def make_scheduler(optimizer, start_lr: float, final_lr: float, steps: int):
    ratio = final_lr / start_lr

    def factor(index: int) -> float:
        progress = min(max(index / float(max(1, steps)), 0.0), 1.0)
        return ratio + 0.5 * (1.0 - ratio) * (1.0 + math.cos(math.pi * progress))

    return torch.optim.lr_scheduler.LambdaLR(optimizer, factor)


def distance_index_for_step(step: int, count: int, seed: int) -> int:
    """Every distance once per cycle, in a reproducible shuffled order (train.py:114-123)."""
    if step < 1 or count < 1:
        raise ValueError("step and distance count must be positive")
    cycle, offset = divmod(step - 1, count)
    gen = torch.Generator(device="cpu")
    gen.manual_seed(seed + 1_000_003 * cycle)
    return int(torch.randperm(count, generator=gen).tolist()[offset])


def _atomic_torch_save(payload, path: Path) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    fd, tmp = tempfile.mkstemp(prefix=path.name + ".", suffix=".tmp", dir=path.parent)
    os.close(fd)
    try:
        torch.save(payload, tmp)
        os.replace(tmp, path)
    finally:
        Path(tmp).unlink(missing_ok=True)


@dataclass
class TrainConfig:
    out_dir: Path
    steps: int = 1000
    grid: int = 256
    batch: int = 1024
    distances: tuple = DISTANCES
    cfl: float = 0.5
    precision: str = "f32"
    lr: float = 1.0e-4
    lr_final: float = 2.0e-5
    grad_clip: float = 1.0
    grad_skip: float = 10.0
    seed: int = 83
    ckpt_every: int = 32
    log_interval: int = 20
    checkpoint_interval: int = 250
    state_interval: int = 2500
    device: str = "cuda"
    # every sod_monitor_interval steps (0 = never) rank 0 evaluates that step's checkpoint on the Sod problem
    # (sod_monitor.record_checkpoint) and adds the record to circle_validation_metrics.csv/.npz of out_dir
    sod_monitor_interval: int = 0

    def signature(self) -> dict:
        return {"steps": self.steps, "grid": self.grid, "batch": self.batch, "distances": tuple(self.distances),
                "cfl": self.cfl, "precision": self.precision, "lr": self.lr, "lr_final": self.lr_final,
                "seed": self.seed, "loss": "mean_l1_exact_cell_averages_every_step", "velocities": (1.0, -1.0)}


def _world():
    """(world size, rank) of the default process group, or (1, 0) without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def allreduce_gradients(model: torch.nn.Module) -> None:
    """Data parallelism over trajectories: average the parameter gradients over the process group (one
    all-reduce of the 189 packed values; each rank's loss is the mean over its own trajectories, so the
    average is the gradient of the global mean)."""
    world, _ = _world()
    if world == 1:
        return
    import torch.distributed as dist
    params = [p for p in model.parameters() if p.grad is not None]
    flat = torch.cat([p.grad.reshape(-1).to(torch.float64) for p in params])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    flat /= world
    o = 0
    for p in params:
        k = p.grad.numel()
        p.grad.copy_(flat[o:o + k].reshape(p.grad.shape).to(p.grad.dtype))
        o += k


def _allreduce_mean(value: float, device) -> float:
    world, _ = _world()
    if world == 1:
        return value
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item()) / world


def _save_model(path: Path, model: ClosureMLP, step: int, cfg: TrainConfig) -> None:
    meta = {"raw_step": step, "recipe": "l1_exact_cell_averages_every_step", "precision": cfg.precision,
            "primary_cfl": cfg.cfl, "propagation_distances_cells": list(cfg.distances),
            "distance_sampling": "one_each_per_shuffled_cycle", "batch": cfg.batch, "grid": cfg.grid,
            "reflection_formula": "0.5*(M(x)+P*M(P*x))", "adjoint": "hand-written, checkpoint every "
            f"{cfg.ckpt_every} steps", "advection_velocities": [-1.0, 1.0]}
    ckpt.save_checkpoint(path, {k: v.detach().cpu().numpy() for k, v in model.params().items()}, meta)


def train(cfg: TrainConfig, resume: Path | None = None, max_steps: int | None = None) -> dict:
    """Train a WENO5 closure from the reference's initialisation; returns a summary dict.

    Writes checkpoints/model_step_XXXXXX.npz every checkpoint_interval steps, state/latest.pt every
    state_interval steps (and at the end), and history.csv.

    Under torch.distributed (one process per GPU) the batch of each step is split over the ranks: every rank
    draws its own cfg.batch / world trajectories from its own seeded stream, and the gradients are averaged
    with one all-reduce before the identical optimiser steps; rank 0 writes the files."""
    world, rank = _world()
    if cfg.batch % (2 * world):
        raise ValueError(f"batch {cfg.batch} must split into an even number of trajectories per rank ({world} ranks)")
    local_batch = cfg.batch // world
    out = Path(cfg.out_dir)
    if rank == 0:
        out.mkdir(parents=True, exist_ok=True)
    dtype = torch.float32 if cfg.precision == "f32" else torch.float64
    dev = torch.device(cfg.device)
    model = ClosureMLP(seed=cfg.seed, dtype=dtype).to(dev)
    opt = torch.optim.Adam(model.parameters(), lr=cfg.lr)
    sched = make_scheduler(opt, cfg.lr, cfg.lr_final, cfg.steps)
    rng = np.random.default_rng(cfg.seed if world == 1 else [cfg.seed, rank])
    start, skipped = 1, 0
    if resume is not None:
        state = torch.load(resume, map_location=dev, weights_only=False)
        if state.get("training_signature") != cfg.signature():
            raise ValueError("resume training signature mismatch")
        model.load_state_dict(state["model_state_dict"])
        opt.load_state_dict(state["optimizer_state_dict"])
        sched.load_state_dict(state["scheduler_state_dict"])
        rng.bit_generator.state = state["profile_rng_state"] if world == 1 else state["profile_rng_states"][rank]
        start, skipped = int(state["step"]) + 1, int(state.get("skipped", 0))
    elif rank == 0:
        _save_model(out / "checkpoints" / "model_step_000000.npz", model, 0, cfg)
    hist = out / "history.csv"
    fields = ["step", "loss", "distance_cells", "horizon", "batch", "lr", "grad", "skipped"]
    if rank == 0 and (start == 1 or not hist.exists()):
        with hist.open("w", newline="") as f:
            csv.DictWriter(f, fieldnames=fields).writeheader()
    end = cfg.steps if max_steps is None else min(cfg.steps, start - 1 + max_steps)
    last = {}

    def save_state(step):
        rng_states = [rng.bit_generator.state]
        if world > 1:
            import torch.distributed as dist
            rng_states = [None] * world
            dist.all_gather_object(rng_states, rng.bit_generator.state)
        if rank == 0:
            _atomic_torch_save({"step": step, "skipped": skipped, "model_state_dict": model.state_dict(),
                                "optimizer_state_dict": opt.state_dict(), "scheduler_state_dict": sched.state_dict(),
                                "profile_rng_state": rng_states[0], "profile_rng_states": rng_states,
                                "training_signature": cfg.signature()}, out / "state" / "latest.pt")

    for step in range(start, end + 1):
        dist = float(cfg.distances[distance_index_for_step(step, len(cfg.distances), cfg.seed)])
        batch = TrajectoryBatch.sample(rng, local_batch, cfg.grid, dist, cfg.cfl, dev, cfg.ckpt_every)
        loss = trajectory_loss(model, batch)
        opt.zero_grad(set_to_none=True)
        lval = _allreduce_mean(float(loss.detach()), dev)
        if not math.isfinite(lval):
            skipped += 1
            sched.step()
            continue
        loss.backward()
        allreduce_gradients(model)
        grad = float(torch.nn.utils.clip_grad_norm_(model.parameters(), cfg.grad_clip))
        if not math.isfinite(grad) or grad > cfg.grad_skip:
            skipped += 1
            opt.zero_grad(set_to_none=True)
        else:
            opt.step()
        sched.step()
        last = {"step": step, "loss": lval, "distance_cells": dist, "horizon": batch.steps, "batch": batch.B * world,
                "lr": sched.get_last_lr()[0], "grad": grad, "skipped": skipped}
        if rank == 0 and (step == 1 or step % cfg.log_interval == 0):
            with hist.open("a", newline="") as f:
                csv.DictWriter(f, fieldnames=fields).writerow(last)
        if rank == 0 and step % cfg.checkpoint_interval == 0:
            _save_model(out / "checkpoints" / f"model_step_{step:06d}.npz", model, step, cfg)
        if rank == 0 and cfg.sod_monitor_interval > 0 and step % cfg.sod_monitor_interval == 0:
            from . import sod_monitor as SM
            ck = out / "checkpoints" / f"model_step_{step:06d}.npz"
            if step % cfg.checkpoint_interval != 0:
                _save_model(ck, model, step, cfg)
            SM.record_checkpoint(out, ck, step, SM.SodMonitorConfig(
                precision="sr_f32" if cfg.precision == "f32" else "sr_f64"), dev)
        if step % cfg.state_interval == 0:
            save_state(step)
    save_state(end)
    if rank == 0:
        _save_model(out / "checkpoints" / f"model_step_{end:06d}.npz", model, end, cfg)
        (out / "summary.json").write_text(json.dumps({**last, "completed": end}, indent=1))
    return {"model": model, "last": last, "skipped": skipped, "completed": end}
