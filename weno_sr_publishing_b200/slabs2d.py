"""Y-slab decomposition of the 2D Euler WENO5 step over ranks (one process per GPU).

The global grid (nx x ny interior cells, ghost width 3) is cut into slabs of whole rows; rank r owns rows
[y0_r, y1_r) in the reference's padded layout [(ny_r + 6), (nx + 6), 4] with its own 3 ghost rows below and
above. Before every SSPRK3 stage the slabs exchange 3 interior rows with each neighbour -- one contiguous
3 x (nx + 6) x 4 block per side, sent upward in one phase and downward in the next (torch.distributed
point-to-point: NCCL between GPUs, gloo between CPU processes) -- and the outermost slabs fill their outer
ghost rows from the global boundary (transmissive: copies of the edge row; periodic: the wrap-around
neighbour). The kernels read those ghost rows as stored (WSR_BC_Y_HALO) and derive the x ghosts as usual. One
MAX all-reduce of the wave speed per step gives every rank the same dt; the loop applies the device loop's
dt and stop rules (wsr_euler2d_run, warp_weno5_helpers.py:189-207, weno5_hllc_refsym.py:462-544), so a
decomposed run equals the single-domain run bit for bit.

The double-Mach boundary (time-dependent y boundaries) is not decomposed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from . import euler2d as E
from .params import Params

GHOST = 3


def slab_rows(ny: int, world: int, rank: int) -> tuple[int, int]:
    """Rows [y0, y1) of slab `rank` when ny rows are cut into `world` slabs of ny // world or ny // world + 1
    rows (the first ny % world slabs take the extra row). Every slab needs at least 3 rows, so that a halo
    comes from one neighbour."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad slab {rank} of {world}")
    base, extra = divmod(int(ny), world)
    if base < GHOST:
        raise ValueError(f"{ny} rows over {world} slabs leaves slabs of {base} rows; every slab needs at least "
                         f"{GHOST}")
    y0 = rank * base + min(rank, extra)
    return y0, y0 + base + (1 if rank < extra else 0)


@dataclass(frozen=True)
class SlabParams(Params):
    """Params of one slab: ny is the slab's row count and dy the global grid's (not y_length / ny)."""
    slab_dy: float = 0.0
    y0: int = 0

    @property
    def dy(self) -> float:
        return self.slab_dy


def slab_params(params: Params, world: int, rank: int) -> SlabParams:
    y0, y1 = slab_rows(params.ny, world, rank)
    return SlabParams(nx=params.nx, ny=y1 - y0, ghost=params.ghost, gamma=params.gamma, x_length=params.x_length,
                      y_length=params.dy * (y1 - y0), cfl=params.cfl, t_end=params.t_end, slab_dy=params.dy, y0=y0)


def split(u_global, params: Params, world: int, rank: int):
    """The padded slab `rank` of a padded global state (numpy or torch), ghost rows included (copied)."""
    y0, y1 = slab_rows(params.ny, world, rank)
    part = u_global[y0:y1 + 2 * GHOST]
    return part.clone() if isinstance(part, torch.Tensor) else np.array(part, copy=True)


def fill_outer_rows(u, periodic: bool, lower_edge: bool, upper_edge: bool) -> None:
    """Transmissive global boundary: the outer ghost rows of an edge slab copy its edge row."""
    if periodic:
        return
    ny = u.shape[0] - 2 * GHOST
    if lower_edge:
        for k in range(GHOST):
            u[k] = u[GHOST]
    if upper_edge:
        for k in range(GHOST):
            u[ny + GHOST + k] = u[ny + GHOST - 1]


class LocalSlabs:
    """All slabs in this process (a single GPU, or the CPU): halos are copied between the slab arrays."""

    def __init__(self, world: int):
        self.world = world

    def exchange(self, slabs: list, periodic: bool) -> None:
        if len(slabs) != self.world:
            raise ValueError(f"expected {self.world} slabs, got {len(slabs)}")
        n = self.world
        for r, u in enumerate(slabs):
            ny = u.shape[0] - 2 * GHOST
            below = r - 1 if r > 0 else (n - 1 if periodic else None)
            above = r + 1 if r < n - 1 else (0 if periodic else None)
            if below is not None:
                b = slabs[below]
                nb = b.shape[0] - 2 * GHOST
                u[0:GHOST] = b[nb:nb + GHOST]
            if above is not None:
                u[ny + GHOST:ny + 2 * GHOST] = slabs[above][GHOST:2 * GHOST]
            fill_outer_rows(u, periodic, r == 0, r == n - 1)

    def max(self, value: float) -> float:
        return value


class DistSlabs:
    """One slab per rank of the default torch.distributed process group."""

    def __init__(self, group=None):
        import torch.distributed as dist  # noqa: PLC0415

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def _swap(self, send, dst, recv, src) -> None:
        d = self.dist
        ops = []
        if dst is not None:
            ops.append(d.P2POp(d.isend, send, dst, self.group))
        if src is not None:
            ops.append(d.P2POp(d.irecv, recv, src, self.group))
        if ops:
            for req in d.batch_isend_irecv(ops):
                req.wait()

    def exchange(self, slabs: list, periodic: bool) -> None:
        if len(slabs) != 1:
            raise ValueError("DistSlabs holds one slab per rank")
        u = slabs[0]
        t = u if isinstance(u, torch.Tensor) else torch.from_numpy(u)
        ny = t.shape[0] - 2 * GHOST
        r, n = self.rank, self.world
        below = r - 1 if r > 0 else (n - 1 if periodic else None)
        above = r + 1 if r < n - 1 else (0 if periodic else None)
        if n == 1 and periodic:  # own wrap-around
            t[0:GHOST] = t[ny:ny + GHOST].clone()
            t[ny + GHOST:] = t[GHOST:2 * GHOST].clone()
            return
        # phase 1: top interior rows go up, the bottom ghost rows come from below
        self._swap(t[ny:ny + GHOST], above, t[0:GHOST], below)
        # phase 2: bottom interior rows go down, the top ghost rows come from above
        self._swap(t[GHOST:2 * GHOST], below, t[ny + GHOST:ny + 2 * GHOST], above)
        fill_outer_rows(t, periodic, r == 0, r == n - 1)

    def max(self, value: float) -> float:
        d = self.dist
        backend = d.get_backend(self.group)
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        v = torch.tensor([value], dtype=torch.float64, device=dev)
        d.all_reduce(v, op=d.ReduceOp.MAX, group=self.group)
        return float(v.item())


class CudaStages:
    """The slab stages and wave speeds through libwsr.so (WSR_BC_Y_HALO)."""

    def __init__(self, method: str, mlp_params=None, flux: str = "hllc", opts: int = 0):
        self.method, self.mlp_params, self.flux, self.opts = method, mlp_params, flux, opts
        self._ws: dict = {}

    def _workspace(self, u: torch.Tensor, p: Params):
        key = (u.device.index, p.nx, p.ny)
        if key not in self._ws:
            self._ws[key] = E.workspace(p.nx, p.ny, u.device)
        return self._ws[key]

    def max_speed(self, u: torch.Tensor, p: Params) -> float:
        return E.max_speed(u, p, self._workspace(u, p))

    def stage(self, u_stage, u0, u_out, p: Params, dt: float, rk: int, boundary: str) -> None:
        E.stage(u_stage, u0, u_out, p, dt, rk, self.method, boundary, self.mlp_params, self.flux, self.opts,
                ws=self._workspace(u_stage, p), y_halo=True)

    def empty_like(self, u):
        return torch.empty_like(u)


@dataclass
class SlabRun:
    slabs: list          # final padded state of each local slab
    params: list         # SlabParams of each local slab
    dts: list = field(default_factory=list)
    steps: int = 0
    t: float = 0.0


def run(slabs: list, params: list, t_end: float, boundary: str, comm, stages,
        max_steps: int = 1 << 20, t_start: float = 0.0) -> SlabRun:
    """SSPRK3 time loop over the local slabs (`slabs[k]` padded, `params[k]` its SlabParams); `comm` is a
    LocalSlabs (all slabs here) or DistSlabs (one per rank); `stages` computes stages and wave speeds
    (CudaStages for the GPU). The slabs are advanced out of place; the returned SlabRun holds the final ones."""
    if boundary not in ("transmissive", "periodic"):
        raise NotImplementedError(f"the y-slab decomposition supports transmissive and periodic boundaries, not "
                                  f"{boundary!r}")
    if boundary not in N.BC:
        raise ValueError(f"unsupported boundary {boundary!r}")
    periodic = boundary == "periodic"
    p0 = params[0]
    hmin = min(p0.dx, p0.dy)
    bufs = [[u] + [stages.empty_like(u) for _ in range(3)] for u in slabs]
    t, steps, dts = float(t_start), 0, []
    while steps < max_steps:
        if not t < t_end - 1.0e-14:
            break
        ms = comm.max(max(stages.max_speed(b[0], p) for b, p in zip(bufs, params)))
        dt = 1.0e10 if ms < 1.0e-15 else p0.cfl * hmin / ms
        rem = t_end - t
        dt = dt if dt < rem else rem
        if not math.isfinite(dt) or dt <= 0.0:
            break
        for rk, src, dst in ((1, 0, 1), (2, 1, 2), (3, 2, 3)):
            comm.exchange([b[src] for b in bufs], periodic)
            for b, p in zip(bufs, params):
                stages.stage(b[src], b[0], b[dst], p, dt, rk, boundary)
        for b in bufs:
            b[0], b[3] = b[3], b[0]
        t = t + dt
        steps += 1
        dts.append(dt)
    return SlabRun([b[0] for b in bufs], list(params), dts, steps, t)


def gather_interior(slabs: list) -> np.ndarray:
    """Interior rows of the slabs in order, as one [ny][nx][4] host array."""
    parts = []
    for u in slabs:
        a = u.detach().cpu().numpy() if isinstance(u, torch.Tensor) else np.asarray(u)
        parts.append(a[GHOST:a.shape[0] - GHOST, GHOST:a.shape[1] - GHOST])
    return np.concatenate(parts, axis=0)
