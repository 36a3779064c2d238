"""Slab decompositions of the 2D and 3D Euler WENO5 steps over ranks (one process per GPU): y-slabs in 2D,
z-slabs in 3D -- in both layouts the leading array axis, so the halo blocks are contiguous.

2D. The global grid (nx x ny interior cells, ghost width 3) is cut into slabs of whole rows; rank r owns rows
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

3D. The grid [nz+6][ny+6][nx+6][5] is cut into z-slabs the same way; before every RK stage 3 z-planes are
exchanged with each neighbour (the global z ends copy their edge plane: the solver's outflow boundary), and
the stage fills the x and y ghosts of every plane itself, halo planes included, and leaves the z ghost
planes as given (WSR_OPT_Z_HALO). The loop applies the 3D solver's dt and stop rules (solver.py:303-329).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from . import euler2d as E
from . import euler3d as E3
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


class _DeviceWord:
    """One int64 in device memory as a torch tensor (the wave-speed slot of a slab's control block)."""

    def __init__(self, ptr: int):
        self.__cuda_array_interface__ = {"shape": (1,), "typestr": "<i8", "data": (ptr, False), "version": 3}


def _device_loop_applies(slabs, comm, stages) -> bool:
    return (isinstance(comm, DistSlabs) and isinstance(stages, CudaStages) and len(slabs) == 1
            and isinstance(slabs[0], torch.Tensor) and slabs[0].is_cuda and comm.dist.get_backend(comm.group) == "nccl")


def _run_device(u: torch.Tensor, p, t_end: float, periodic: bool, comm, stages, max_steps: int, t_start: float,
                batch: int = 16) -> SlabRun:
    """The device-resident loop of one slab per rank: dt, t and the stop test stay in the slab's control block
    (wsr_euler2d_slab_*), the halos and the wave speed's MAX all-reduce go over NCCL on the same stream, and the
    host reads the control block every `batch` steps; no host synchronisation inside a batch."""
    dev = u.device
    L = N.lib()
    ctx = E.prepare_closure(stages.method, stages.mlp_params, dev.index)
    ws = stages._workspace(u, p)
    stream = E._stream_ptr(dev.index)
    bufs = [u] + [torch.empty_like(u) for _ in range(3)]
    ctx.check(L.wsr_euler2d_slab_begin(ctx.handle, C.c_void_p(u.data_ptr()), p.nx, p.ny, p.dx, p.dy, p.gamma, p.cfl,
                                       float(t_start), float(t_end), int(max_steps), C.c_void_p(ws.ptr), ws.nbytes,
                                       stream))
    slot_ptr = C.c_void_p()
    ctx.check(L.wsr_euler2d_slab_speed_slot(ctx.handle, C.c_void_p(ws.ptr), ws.nbytes, p.nx, p.ny,
                                            C.byref(slot_ptr)))
    slot = torch.as_tensor(_DeviceWord(slot_ptr.value), device=dev)
    d = comm.dist
    d.all_reduce(slot, op=d.ReduceOp.MAX, group=comm.group)
    bc = N.BC["periodic" if periodic else "transmissive"] | N.BC_Y_HALO
    method, flux = N.METHOD[stages.method], N.FLUX[stages.flux]
    ring = (C.c_double * 64)()
    steps, t, done = C.c_int(0), C.c_double(0.0), C.c_int(0)
    launched, dts = 0, []
    while launched < max_steps and not done.value:
        for s in range(launched, min(launched + batch, max_steps)):
            a, b = (bufs[0], bufs[3]) if s % 2 == 0 else (bufs[3], bufs[0])
            ctx.check(L.wsr_euler2d_slab_step(ctx.handle, 0, p.nx, p.ny, p.dx, p.dy, C.c_void_p(ws.ptr), ws.nbytes,
                                              stream))
            for rk, src, dst in ((1, a, bufs[1]), (2, bufs[1], bufs[2]), (3, bufs[2], b)):
                comm.exchange([src], periodic)
                ctx.check(L.wsr_euler2d_slab_stage(ctx.handle, C.c_void_p(src.data_ptr()), C.c_void_p(a.data_ptr()),
                                                   C.c_void_p(dst.data_ptr()), p.nx, p.ny, p.dx, p.dy, p.gamma, rk,
                                                   method, bc, flux, int(stages.opts), C.c_void_p(ws.ptr), ws.nbytes,
                                                   stream))
            d.all_reduce(slot, op=d.ReduceOp.MAX, group=comm.group)
            ctx.check(L.wsr_euler2d_slab_step(ctx.handle, 1, p.nx, p.ny, p.dx, p.dy, C.c_void_p(ws.ptr), ws.nbytes,
                                              stream))
        launched = min(launched + batch, max_steps)
        seen = len(dts)
        ctx.check(L.wsr_euler2d_slab_status(ctx.handle, C.c_void_p(ws.ptr), ws.nbytes, p.nx, p.ny, C.byref(steps),
                                            C.byref(t), C.byref(done), ring, stream))
        dts += [float(ring[k % 64]) for k in range(seen, steps.value)]
    final = bufs[0] if steps.value % 2 == 0 else bufs[3]
    return SlabRun([final], [p], dts, steps.value, t.value)


def run(slabs: list, params: list, t_end: float, boundary: str, comm, stages,
        max_steps: int = 1 << 20, t_start: float = 0.0, host_loop: bool = False) -> SlabRun:
    """SSPRK3 time loop over the local slabs (`slabs[k]` padded, `params[k]` its SlabParams); `comm` is a
    LocalSlabs (all slabs here) or DistSlabs (one per rank); `stages` computes stages and wave speeds
    (CudaStages for the GPU). The slabs are advanced out of place; the returned SlabRun holds the final ones.
    One CUDA slab per rank over NCCL runs the device-resident loop (no host synchronisation per step) unless
    host_loop is set; the results are the same bit for bit."""
    if boundary not in ("transmissive", "periodic"):
        raise NotImplementedError(f"the y-slab decomposition supports transmissive and periodic boundaries, not "
                                  f"{boundary!r}")
    if boundary not in N.BC:
        raise ValueError(f"unsupported boundary {boundary!r}")
    periodic = boundary == "periodic"
    if not host_loop and _device_loop_applies(slabs, comm, stages):
        return _run_device(slabs[0], params[0], t_end, periodic, comm, stages, max_steps, t_start)
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


# ------------------------------------------------------------------------------------------------
# 3D z-slabs
# ------------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class Grid3:
    """One z-slab of a 3D grid: its interior size, the spacings of the global grid, its first global plane."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    z0: int = 0

    @property
    def padded_shape(self) -> tuple[int, int, int, int]:
        return (self.nz + 2 * GHOST, self.ny + 2 * GHOST, self.nx + 2 * GHOST, 5)


def slab_grid3(nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, world: int, rank: int) -> Grid3:
    z0, z1 = slab_rows(nz, world, rank)
    return Grid3(nx, ny, z1 - z0, dx, dy, dz, z0)


def split3(q_global, nz: int, world: int, rank: int):
    """The padded z-slab `rank` of a padded global 3D state, ghost planes included (copied)."""
    return split(q_global, Params(nx=1, ny=nz), world, rank)


class CudaStages3:
    """The 3D z-slab stages (in place, stage-start copy in the slab's workspace) and wave speeds through
    libwsr.so (WSR_OPT_Z_HALO)."""

    def __init__(self, method: str = "js", flux: str = "evilin", mlp_params=None, inflow=None, opts: int = 0):
        self.method, self.flux, self.mlp_params, self.inflow, self.opts = method, flux, mlp_params, inflow, opts
        self._ws: dict = {}

    def _workspace(self, q: torch.Tensor, g: Grid3):
        key = (q.data_ptr(), g.nx, g.ny, g.nz)
        if key not in self._ws:
            self._ws[key] = E3.workspace(g.nx, g.ny, g.nz, q.device)
        return self._ws[key]

    def max_speed(self, q: torch.Tensor, g: Grid3) -> float:
        return E3.max_speed(q, g.nx, g.ny, g.nz, self._workspace(q, g))

    def stage(self, q: torch.Tensor, g: Grid3, dt: float, stage: int) -> None:
        E3.stage(q, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, dt, stage, self.method, self.flux, self.mlp_params,
                 self.inflow, self.opts | N.OPT_Z_HALO, ws=self._workspace(q, g))


@dataclass
class SlabRun3:
    slabs: list
    grids: list
    dts: list = field(default_factory=list)
    steps: int = 0
    t: float = 0.0


def run3(slabs: list, grids: list, cfl: float, comm, stages, t_end: float | None = None, steps: int | None = None,
         t_start: float = 0.0) -> SlabRun3:
    """Advance the local 3D z-slabs in place: to t_end, or exactly `steps` steps when t_end is None
    (Weno5Rk3Solver.advance, solver.py:303-329: dt = cfl min(dx, dy, dz) / max speed, 1e10 below 1e-15,
    clipped to t_end; stop when t == t_end)."""
    if t_end is None and steps is None:
        raise ValueError("give t_end or steps")
    g0 = grids[0]
    hmin = min(g0.dx, g0.dy, g0.dz)
    t_stop = 1.0e300 if t_end is None else float(t_end)
    cap = steps if steps is not None else 1_000_000
    t, taken, dts = float(t_start), 0, []
    for _ in range(cap):
        if t == t_stop:
            break
        m = comm.max(max(stages.max_speed(q, g) for q, g in zip(slabs, grids)))
        dt = 1.0e10 if m < 1.0e-15 else cfl * hmin / m
        if t + dt > t_stop:
            dt = t_stop - t
        t = t + dt
        for st in (1, 2, 3):
            comm.exchange(slabs, False)
            for q, g in zip(slabs, grids):
                stages.stage(q, g, dt, st)
        taken += 1
        dts.append(dt)
    return SlabRun3(slabs, list(grids), dts, taken, t)


def gather_interior3(slabs: list) -> np.ndarray:
    """Interior cells of the 3D slabs in order, as one [nz][ny][nx][5] host array."""
    parts = []
    for q in slabs:
        a = q.detach().cpu().numpy() if isinstance(q, torch.Tensor) else np.asarray(q)
        parts.append(a[GHOST:-GHOST, GHOST:-GHOST, GHOST:-GHOST])
    return np.concatenate(parts, axis=0)
