"""The no-allocation stage entry point (wsr_euler2d_stage_noalloc) against wsr_euler2d_stage.

wsr_euler2d_stage_noalloc exists for callers that cannot call cudaMalloc (a host that owns all device
memory through its own pool, or a step that must not pay cudaMalloc's implicit synchronisation): its
scratch is a static device array inside libwsr.so instead of a caller workspace. This test calls it
through the C ABI, twice in a row on the same device, and checks each result against the allocating
entry point on the same inputs. It lives in its own file, collected last, so that a run stopping at the
first failure has already run every other test.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest
import torch

from weno_sr_publishing_b200 import _native as N
from weno_sr_publishing_b200 import euler2d as E
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200.params import Params

pytestmark = pytest.mark.gpu

MODELS = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")
WSR_ERR_SCRATCH_LIMIT = 4
TOL = 1e-13  # relative max-norm, the tightest stage tolerance of the GPU suite


def _lib():
    return N.lib()  # the binding declares wsr_euler2d_stage_noalloc's argument types


def _noalloc(u_stage, u0, u_out, p, dt, rk, method, packed, bc="transmissive", flux="hllc"):
    ptr = packed.ctypes.data_as(C.POINTER(C.c_double)) if packed is not None else None
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib().wsr_euler2d_stage_noalloc(
        C.c_void_p(u_stage.data_ptr()), C.c_void_p(u0.data_ptr()), C.c_void_p(u_out.data_ptr()), p.nx, p.ny, p.dx,
        p.dy, p.gamma, dt, rk, N.METHOD[method], N.BC[bc], N.FLUX[flux], 0, ptr, stream)


CHECKPOINTS = {"js": None, "z": None, "sr_f64": "weno5_sr_fp64_step012250.npz",
               "sr_f32": "weno5_sr_fp32_step016500.npz", "sr_bf16": "weno5_sr_fp32_step016500.npz"}


def _two_stages_against_workspace_stage(method, nx, ny, bc, flux="hllc"):
    torch.cuda.set_device(0)
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    init = torch.as_tensor(problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(4), 3),
                           device="cuda:0")
    model = CHECKPOINTS[method]
    params = None if model is None else {k: v for k, v in np.load(MODELS / model).items() if k in NAMES}
    packed = None if params is None else N.pack_params(params)
    dt = 0.4 * min(p.dx, p.dy) / E.max_speed(init, p)
    # two calls in a row: stage 1 from the initial state, then stage 2 from the first call's output
    ref1 = torch.zeros_like(init)
    E.stage(init, init, ref1, p, dt, 1, method, bc, mlp_params=params, flux=flux)
    ref2 = torch.zeros_like(init)
    E.stage(ref1, init, ref2, p, dt, 2, method, bc, mlp_params=params, flux=flux)
    got1 = torch.zeros_like(init)
    assert _noalloc(init, init, got1, p, dt, 1, method, packed, bc, flux) == 0
    got2 = torch.zeros_like(init)
    assert _noalloc(got1, init, got2, p, dt, 2, method, packed, bc, flux) == 0
    torch.cuda.synchronize()
    for got, ref in ((got1, ref1), (got2, ref2)):
        g, r = got.cpu().numpy(), ref.cpu().numpy()
        err = float(np.abs(g - r).max() / np.abs(r).max())
        assert err <= TOL, err


@pytest.mark.parametrize("method", ["js", "z", "sr_f64", "sr_f32", "sr_bf16"])
def test_noalloc_stage_matches_workspace_stage_twice(method):
    _two_stages_against_workspace_stage(method, 96, 80, "transmissive")


@pytest.mark.parametrize("method,flux", [("sr_f32", "hllc"), ("js", "force")])
def test_noalloc_periodic_and_force(method, flux):
    _two_stages_against_workspace_stage(method, 72, 88, "periodic", flux)


def test_noalloc_at_the_largest_grid_the_scratch_holds():
    # 400 x 400 is the largest square grid whose stage scratch fits the static array
    _two_stages_against_workspace_stage("js", 400, 400, "transmissive")
    _two_stages_against_workspace_stage("sr_f32", 400, 400, "transmissive")


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    torch.cuda.set_device(0)
    p = Params(nx=512, ny=512, x_length=1.0, y_length=1.0, cfl=0.4)
    u = torch.zeros(p.padded_shape, dtype=torch.float64, device="cuda:0")
    assert _noalloc(u, u, u, p, 1e-3, 1, "js", None) == WSR_ERR_SCRATCH_LIMIT


def test_noalloc_rejects_unsupported_boundaries():
    torch.cuda.set_device(0)
    p = Params(nx=32, ny=32, x_length=1.0, y_length=1.0, cfl=0.4)
    u = torch.zeros(p.padded_shape, dtype=torch.float64, device="cuda:0")
    assert _noalloc(u, u, u, p, 1e-3, 1, "js", None, bc="double-mach") == 1  # WSR_ERR_ARG
