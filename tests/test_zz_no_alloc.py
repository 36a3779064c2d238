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
    L = N.lib()
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.wsr_euler2d_stage_noalloc.argtypes = [vp, vp, vp, i, i, d, d, d, d, i, i, i, i, i, C.POINTER(d), vp]
    L.wsr_euler2d_stage_noalloc.restype = i
    return L


def _noalloc(u_stage, u0, u_out, p, dt, rk, method, packed):
    ptr = packed.ctypes.data_as(C.POINTER(C.c_double)) if packed is not None else None
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib().wsr_euler2d_stage_noalloc(
        C.c_void_p(u_stage.data_ptr()), C.c_void_p(u0.data_ptr()), C.c_void_p(u_out.data_ptr()), p.nx, p.ny, p.dx,
        p.dy, p.gamma, dt, rk, N.METHOD[method], N.BC["transmissive"], N.FLUX["hllc"], 0, ptr, stream)


@pytest.mark.parametrize("method,model", [("js", None), ("sr_f64", "weno5_sr_fp64_step012250.npz"),
                                          ("sr_f32", "weno5_sr_fp32_step016500.npz")])
def test_noalloc_stage_matches_workspace_stage_twice(method, model):
    torch.cuda.set_device(0)
    nx, ny = 96, 80
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    init = torch.as_tensor(problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(4), 3),
                           device="cuda:0")
    params = None if model is None else {k: v for k, v in np.load(MODELS / model).items() if k in NAMES}
    packed = None if params is None else N.pack_params(params)
    dt = 0.4 * min(p.dx, p.dy) / E.max_speed(init, p)
    # two calls in a row: stage 1 from the initial state, then stage 2 from the first call's output
    ref1 = torch.zeros_like(init)
    E.stage(init, init, ref1, p, dt, 1, method, "transmissive", mlp_params=params)
    ref2 = torch.zeros_like(init)
    E.stage(ref1, init, ref2, p, dt, 2, method, "transmissive", mlp_params=params)
    got1 = torch.zeros_like(init)
    assert _noalloc(init, init, got1, p, dt, 1, method, packed) == 0
    got2 = torch.zeros_like(init)
    assert _noalloc(got1, init, got2, p, dt, 2, method, packed) == 0
    torch.cuda.synchronize()
    for got, ref in ((got1, ref1), (got2, ref2)):
        g, r = got.cpu().numpy(), ref.cpu().numpy()
        err = float(np.abs(g - r).max() / np.abs(r).max())
        assert err <= TOL, err


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    torch.cuda.set_device(0)
    p = Params(nx=512, ny=512, x_length=1.0, y_length=1.0, cfl=0.4)
    u = torch.zeros(p.padded_shape, dtype=torch.float64, device="cuda:0")
    assert _noalloc(u, u, u, p, 1e-3, 1, "js", None) == WSR_ERR_SCRATCH_LIMIT
