"""CPU: the y-slab decomposition of the 2D step (partition, halo exchange, global boundary rows, time loop)
driven through the oracle's stage in y-halo mode, in one process and as two gloo ranks; every decomposed run
equals the single-domain oracle run bit for bit."""
from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200 import slabs as S
from weno_sr_publishing_b200.params import Params

NX, NY = 17, 14


class OracleStages:
    """The oracle's stage (y-halo mode) and wave speed, on numpy slabs."""

    def __init__(self, method="js", params=None):
        self.method, self.params = method, params

    def max_speed(self, u, p):
        return O.max_speed(u, p.nx, p.ny, p.gamma)

    def stage(self, u_stage, u0, u_out, p, dt, rk, boundary):
        u_out[...] = O.euler2d_stage(u_stage, u0, u_out, p.nx, p.ny, p.dx, p.dy, dt, rk, self.method, boundary,
                                     params=self.params, gamma=p.gamma, y_halo=True)

    def empty_like(self, u):
        return np.zeros_like(u)


def _initial(seed=3):
    init = problems.make_quadrant_state(NX, NY, problems.seeded_quadrant_states(seed), 3)
    rng = np.random.default_rng(seed)
    init[3:-3, 3:-3, 0] *= 1.0 + 0.05 * rng.uniform(size=(NY, NX))  # break the quadrant symmetry
    return np.ascontiguousarray(init)


def _params():
    return Params(nx=NX, ny=NY, x_length=1.0, y_length=0.8, cfl=0.4)


def test_slab_rows_partition():
    for ny, world in ((14, 1), (14, 2), (14, 3), (14, 4), (2000, 8), (9, 3)):
        rows = [S.slab_rows(ny, world, r) for r in range(world)]
        assert rows[0][0] == 0 and rows[-1][1] == ny
        assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
        sizes = [y1 - y0 for y0, y1 in rows]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        S.slab_rows(8, 3, 0)  # slabs of 2 rows
    with pytest.raises(ValueError):
        S.slab_rows(14, 2, 2)


def test_slab_params_keep_the_global_spacing():
    p = Params(nx=10, ny=7, x_length=1.0, y_length=0.7000000000000001)
    for r in range(2):
        sp = S.slab_params(p, 2, r)
        assert sp.dy == p.dy and sp.dx == p.dx and sp.padded_shape == (sp.ny + 6, 16, 4)


@pytest.mark.parametrize("boundary", ["transmissive", "periodic"])
@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_halo_exchange_matches_the_global_ghost_rows(boundary, world):
    rng = np.random.default_rng(world)
    p = _params()
    glob = rng.normal(size=p.padded_shape)
    g = 3
    if boundary == "periodic":
        glob[:g], glob[NY + g:] = glob[NY:NY + g], glob[g:2 * g]
    else:
        glob[:g], glob[NY + g:] = glob[g], glob[NY + g - 1]
    slabs = [S.split(glob, p, world, r) for r in range(world)]
    for s in slabs:
        s[:g] = np.nan
        s[-g:] = np.nan
    S.LocalSlabs(world).exchange(slabs, boundary == "periodic")
    for r, s in enumerate(slabs):
        y0, y1 = S.slab_rows(NY, world, r)
        np.testing.assert_array_equal(s, glob[y0:y1 + 2 * g])


@pytest.mark.parametrize("boundary", ["transmissive", "periodic"])
@pytest.mark.parametrize("world", [2, 3])
def test_decomposed_oracle_run_equals_single_domain(boundary, world):
    p = _params()
    init = _initial()
    t_end = 0.02
    ref, rdts, rsteps, rt = O.euler2d_run(init, NX, NY, p.dx, p.dy, p.cfl, t_end, "js", boundary)
    params = [S.slab_params(p, world, r) for r in range(world)]
    slabs = [S.split(init, p, world, r) for r in range(world)]
    res = S.run(slabs, params, t_end, boundary, S.LocalSlabs(world), OracleStages("js"))
    assert res.steps == rsteps and res.t == rt and res.dts == list(rdts)
    np.testing.assert_array_equal(S.gather_interior(res.slabs), ref[3:-3, 3:-3])


def test_decomposed_sr_run_equals_single_domain():
    from weno_sr_publishing_b200.checkpoint import MODELS_DIR

    w = dict(np.load(MODELS_DIR / "weno5_sr_fp64_step012250.npz"))
    p = _params()
    init = _initial(5)
    ref, _, rsteps, rt = O.euler2d_run(init, NX, NY, p.dx, p.dy, p.cfl, 0.01, "sr_f64", "transmissive", params=w)
    params = [S.slab_params(p, 3, r) for r in range(3)]
    slabs = [S.split(init, p, 3, r) for r in range(3)]
    res = S.run(slabs, params, 0.01, "transmissive", S.LocalSlabs(3), OracleStages("sr_f64", w))
    assert res.steps == rsteps and res.t == rt
    np.testing.assert_array_equal(S.gather_interior(res.slabs), ref[3:-3, 3:-3])


def test_double_mach_is_not_decomposed():
    p = _params()
    with pytest.raises(NotImplementedError):
        S.run([S.split(_initial(), p, 1, 0)], [S.slab_params(p, 1, 0)], 0.01, "double-mach", S.LocalSlabs(1),
              OracleStages())


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, boundary, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = _params()
        comm = S.DistSlabs()
        res = S.run([S.split(_initial(), p, world, rank)], [S.slab_params(p, world, rank)], 0.02, boundary, comm,
                    OracleStages("js"))
        out[rank] = (S.gather_interior(res.slabs), res.steps, res.t, res.dts)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("boundary", ["transmissive", "periodic"])
def test_two_gloo_ranks_equal_single_domain(boundary):
    world = 2
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, _free_port(), boundary, out), nprocs=world, join=True)
    p = _params()
    ref, rdts, rsteps, rt = O.euler2d_run(_initial(), NX, NY, p.dx, p.dy, p.cfl, 0.02, "js", boundary)
    got = np.concatenate([out[r][0] for r in range(world)], axis=0)
    for r in range(world):
        assert out[r][1] == rsteps and out[r][2] == rt and out[r][3] == list(rdts)
    np.testing.assert_array_equal(got, ref[3:-3, 3:-3])


def test_three_gloo_ranks_periodic():
    world = 3
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, _free_port(), "periodic", out), nprocs=world, join=True)
    p = _params()
    ref, _, rsteps, _ = O.euler2d_run(_initial(), NX, NY, p.dx, p.dy, p.cfl, 0.02, "js", "periodic")
    np.testing.assert_array_equal(np.concatenate([out[r][0] for r in range(world)], axis=0), ref[3:-3, 3:-3])
    assert all(out[r][1] == rsteps for r in range(world))


# ------------------------------------------------------------------------------------------------
# 3D z-slabs
# ------------------------------------------------------------------------------------------------
NX3, NY3, NZ3 = 7, 6, 13


class OracleStages3:
    """The 3D oracle's stage (z-halo mode) and wave speed, on numpy slabs; q0 per slab."""

    def __init__(self, method="js", flux="evilin", params=None, inflow=None):
        self.method, self.flux, self.params, self.inflow = method, flux, params, inflow
        self.q0 = {}

    def max_speed(self, q, g):
        return O.euler3d_max_speed(q, g.nx, g.ny, g.nz)

    def stage(self, q, g, dt, st):
        q0 = self.q0.setdefault(id(q), np.zeros_like(q))
        O.euler3d_stage(q, q0, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, dt, st, self.method, self.flux, self.params,
                        self.inflow, z_halo=True)


def _initial3(seed=1):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*[(np.arange(n) + 0.5) / n for n in (NZ3, NY3, NX3)], indexing="ij")
    rho = 1.0 + 0.4 * (x + 0.6 * y + 0.3 * z > 0.8) + 0.05 * rng.uniform(size=x.shape)
    p = 1.0 + 1.5 * (z < 0.4) + 0.05 * rng.uniform(size=x.shape)
    u, v, w = 0.3 * rng.uniform(-1, 1, x.shape), 0.2 * rng.uniform(-1, 1, x.shape), 0.25 * np.sin(6 * x)
    inner = np.stack([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)], axis=-1)
    return np.ascontiguousarray(np.pad(inner, ((3, 3), (3, 3), (3, 3), (0, 0)), mode="edge"))


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("method,flux,inflow", [("js", "evilin", None), ("js", "hllc", None),
                                                ("sr_f64", "hllc", (1.2, 0.4, 0.0, 0.0, 3.0))])
def test_decomposed_3d_oracle_run_equals_single_domain(world, method, flux, inflow):
    params = None
    if method != "js":
        from weno_sr_publishing_b200.checkpoint import MODELS_DIR
        params = dict(np.load(MODELS_DIR / "weno5_sr_fp64_step012250.npz"))
    q = _initial3()
    d = (0.1, 0.11, 0.09)
    ref, rdts = O.euler3d_run(q, NX3, NY3, NZ3, *d, 0.4, 3, method, flux, params=params, inflow=inflow)[:2]
    grids = [S.slab_grid3(NX3, NY3, NZ3, *d, world, r) for r in range(world)]
    slabs = [S.split3(q, NZ3, world, r) for r in range(world)]
    res = S.run3(slabs, grids, 0.4, S.LocalSlabs(world), OracleStages3(method, flux, params, inflow), steps=3)
    assert res.steps == 3 and res.dts == list(rdts)
    np.testing.assert_array_equal(S.gather_interior3(res.slabs), ref[3:-3, 3:-3, 3:-3])


def _worker3(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        d = (0.1, 0.11, 0.09)
        res = S.run3([S.split3(_initial3(), NZ3, world, rank)], [S.slab_grid3(NX3, NY3, NZ3, *d, world, rank)], 0.4,
                     S.DistSlabs(), OracleStages3("js", "hllc"), t_end=0.05)
        out[rank] = (S.gather_interior3(res.slabs), res.steps, res.t)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_3d_equal_single_domain():
    world = 2
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker3, args=(world, _free_port(), out), nprocs=world, join=True)
    ref, rdts = O.euler3d_run(_initial3(), NX3, NY3, NZ3, 0.1, 0.11, 0.09, 0.4, 100, "js", "hllc", t_end=0.05)[:2]
    assert out[0][1] == out[1][1] == len(rdts) and out[0][2] == out[1][2]
    np.testing.assert_array_equal(np.concatenate([out[r][0] for r in range(world)], axis=0), ref[3:-3, 3:-3, 3:-3])
