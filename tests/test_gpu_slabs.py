"""GPU: the y-slab decomposition of the 2D step through the CUDA kernels (WSR_BC_Y_HALO). The slabs of one
GPU run in one process (LocalSlabs: halos copied between the slab tensors), and a one-rank NCCL group runs the
DistSlabs path; every decomposed run equals the single-domain device loop bit for bit."""
from __future__ import annotations

import ctypes as C
import datetime
import os
import socket

import numpy as np
import pytest
import torch

from weno_sr_publishing_b200 import _native as N
from weno_sr_publishing_b200 import euler2d as E
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200 import slabs as S
from weno_sr_publishing_b200.checkpoint import MODELS_DIR
from weno_sr_publishing_b200.params import Params

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
NX, NY = 70, 53


def _initial(seed=2):
    init = problems.make_quadrant_state(NX, NY, problems.seeded_quadrant_states(seed), 3)
    rng = np.random.default_rng(seed)
    init[3:-3, 3:-3, 0] *= 1.0 + 0.05 * rng.uniform(size=(NY, NX))
    return np.ascontiguousarray(init)


def _closure(method):
    if method == "js":
        return None
    name = "weno5_sr_fp64_step012250.npz" if method == "sr_f64" else "weno5_sr_fp32_step016500.npz"
    return {k: v for k, v in np.load(MODELS_DIR / name).items() if k != "meta_json"}


def _single(init, p, t_end, method, boundary):
    bufs = [torch.as_tensor(init, device=DEV).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                      device=DEV) for _ in range(3)]
    res = E.run(bufs, p, t_end, method, boundary, mlp_params=_closure(method))
    return bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3], res


@pytest.mark.parametrize("method", ["js", "sr_f32", "sr_f64"])
@pytest.mark.parametrize("boundary", ["transmissive", "periodic"])
@pytest.mark.parametrize("world", [2, 3, 5])
def test_slabs_equal_single_domain(method, boundary, world):
    p = Params(nx=NX, ny=NY, x_length=1.0, y_length=0.75, cfl=0.4)
    init = _initial()
    t_end = 0.03
    ref, rres = _single(init, p, t_end, method, boundary)
    g = torch.as_tensor(init, device=DEV)
    slabs = [S.split(g, p, world, r) for r in range(world)]
    params = [S.slab_params(p, world, r) for r in range(world)]
    res = S.run(slabs, params, t_end, boundary, S.LocalSlabs(world), S.CudaStages(method, _closure(method)))
    assert res.steps == rres.steps and res.t == rres.t and res.dts == rres.dts
    np.testing.assert_array_equal(S.gather_interior(res.slabs), ref)


def test_run_loop_rejects_the_halo_flag():
    p = Params(nx=16, ny=16, x_length=1.0, y_length=1.0)
    bufs = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
    ws = E.workspace(16, 16, DEV)
    ctx = N.context(0)
    arr = (C.c_void_p * 4)(*[b.data_ptr() for b in bufs])
    steps, t = C.c_int(0), C.c_double(0.0)
    slot, fb = C.c_int(0), C.c_int(0)
    dts = (C.c_double * 4)()
    rc = N.lib().wsr_euler2d_run(ctx.handle, arr, 16, 16, p.dx, p.dy, 1.4, 0.4, 0.0, 0.1, 0, N.BC_Y_HALO, 0, 0, 0, 0,
                                 1, 4, dts, C.byref(steps), C.byref(t), C.byref(slot), C.byref(fb), C.c_void_p(ws.ptr),
                                 ws.nbytes, None)
    assert rc == 1 and b"WSR_BC_Y_HALO" in N.lib().wsr_last_error(ctx.handle)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("boundary", ["transmissive", "periodic"])
def test_one_rank_nccl_group(boundary):
    """DistSlabs on a one-rank NCCL group: the edge rows, the self wrap-around and the MAX all-reduce on the
    device, equal to the device loop."""
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device(DEV))
    try:
        p = Params(nx=NX, ny=NY, x_length=1.0, y_length=0.75, cfl=0.4)
        init = _initial(4)
        ref, rres = _single(init, p, 0.02, "sr_f32", boundary)
        res = S.run([torch.as_tensor(init, device=DEV).clone()], [S.slab_params(p, 1, 0)], 0.02, boundary,
                    S.DistSlabs(), S.CudaStages("sr_f32", _closure("sr_f32")))
        assert res.steps == rres.steps and res.t == rres.t
        np.testing.assert_array_equal(S.gather_interior(res.slabs), ref)
        # the device-resident loop (dt and the stop test on the device) equals the host-driven loop bit for bit,
        # also when the run stops inside a batch of launched steps (max_steps)
        host = S.run([torch.as_tensor(init, device=DEV).clone()], [S.slab_params(p, 1, 0)], 0.02, boundary,
                     S.DistSlabs(), S.CudaStages("sr_f32", _closure("sr_f32")), host_loop=True)
        assert host.dts == res.dts and host.steps == res.steps
        np.testing.assert_array_equal(S.gather_interior(host.slabs), S.gather_interior(res.slabs))
        part = S.run([torch.as_tensor(init, device=DEV).clone()], [S.slab_params(p, 1, 0)], 0.02, boundary,
                     S.DistSlabs(), S.CudaStages("sr_f32", _closure("sr_f32")), max_steps=21)
        part_h = S.run([torch.as_tensor(init, device=DEV).clone()], [S.slab_params(p, 1, 0)], 0.02, boundary,
                       S.DistSlabs(), S.CudaStages("sr_f32", _closure("sr_f32")), max_steps=21, host_loop=True)
        assert part.steps == part_h.steps == min(21, res.steps) and part.dts == part_h.dts
        np.testing.assert_array_equal(S.gather_interior(part.slabs), S.gather_interior(part_h.slabs))
    finally:
        dist.destroy_process_group()


def _initial3(nx, ny, nz, seed=1):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*[(np.arange(n) + 0.5) / n for n in (nz, ny, nx)], indexing="ij")
    rho = 1.0 + 0.4 * (x + 0.6 * y + 0.3 * z > 0.8) + 0.05 * rng.uniform(size=x.shape)
    p = 1.0 + 1.5 * (z < 0.4) + 0.05 * rng.uniform(size=x.shape)
    u, v, w = 0.3 * rng.uniform(-1, 1, x.shape), 0.2 * rng.uniform(-1, 1, x.shape), 0.25 * np.sin(6 * x)
    inner = np.stack([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)], axis=-1)
    return np.ascontiguousarray(np.pad(inner, ((3, 3), (3, 3), (3, 3), (0, 0)), mode="edge"))


@pytest.mark.parametrize("world", [2, 4])
@pytest.mark.parametrize("method,flux,inflow", [("js", "evilin", None), ("sr_f32", "hllc", None),
                                                ("sr_f64", "hllc", (1.2, 0.4, 0.0, 0.0, 3.0))])
def test_3d_slabs_equal_single_domain(world, method, flux, inflow):
    from weno_sr_publishing_b200 import euler3d as E3

    nx, ny, nz = 24, 17, 30
    d = (0.05, 0.06, 0.04)
    q0 = _initial3(nx, ny, nz)
    q = torch.as_tensor(q0, device=DEV).clone()
    rres = E3.run(q, nx, ny, nz, *d, 0.4, method, flux, mlp_params=_closure(method), inflow=inflow, steps=4)
    ref = q.cpu().numpy()[3:-3, 3:-3, 3:-3]
    g = torch.as_tensor(q0, device=DEV)
    slabs = [S.split3(g, nz, world, r) for r in range(world)]
    grids = [S.slab_grid3(nx, ny, nz, *d, world, r) for r in range(world)]
    res = S.run3(slabs, grids, 0.4, S.LocalSlabs(world), S.CudaStages3(method, flux, _closure(method), inflow),
                 steps=4)
    assert res.steps == rres.steps and res.dts == list(rres.dts)
    np.testing.assert_array_equal(S.gather_interior3(res.slabs), ref)


def test_3d_run_rejects_the_halo_option():
    from weno_sr_publishing_b200 import euler3d as E3

    q = torch.as_tensor(_initial3(8, 8, 8), device=DEV)
    with pytest.raises(ValueError, match="WSR_OPT_Z_HALO"):
        E3.run(q, 8, 8, 8, 0.1, 0.1, 0.1, 0.4, steps=1, opts=N.OPT_Z_HALO)
