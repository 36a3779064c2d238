"""GPU: the host-buffer entry (euler2d.advance_host) equals the device loop bit for bit over repeated calls, for
both result slots (1 and 2 steps per call): synchronous by default (the host buffer holds the result when the
call returns), and with the opt-in overlapped read-back once host_copies_done() and a synchronisation have run.
Two host buffers that share the same device buffers keep their results apart."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from weno_sr_publishing_b200 import euler2d as E
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200.checkpoint import MODELS_DIR
from weno_sr_publishing_b200.params import Params

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _case(seed=1):
    n = 96
    p = Params(nx=n, ny=n - 7, x_length=1.0, y_length=0.9, cfl=0.4)
    init = problems.make_quadrant_state(p.nx, p.ny, problems.seeded_quadrant_states(seed), 3)
    mlp = {k: v for k, v in np.load(MODELS_DIR / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}
    return p, init, mlp


def _device_loop(p, init, mlp, steps):
    bufs = [torch.as_tensor(init, device=DEV).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                      device=DEV) for _ in range(3)]
    res = E.run(bufs, p, 1.0e300, "sr_f32", "transmissive", mlp_params=mlp, fixed_steps=steps)
    return bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3]


@pytest.mark.parametrize("per_call", [1, 2])
@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("async_readback", [False, True])
def test_advance_host_equals_device_loop(per_call, pinned, async_readback):
    p, init, mlp = _case()
    calls = 5
    ref = _device_loop(p, init, mlp, calls * per_call)
    host = torch.as_tensor(init).clone()
    if pinned:
        host = host.pin_memory()
    work = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
    ws = E.workspace(p.nx, p.ny, DEV)
    for _ in range(calls):
        E.advance_host(host, p, per_call, "sr_f32", "transmissive", mlp_params=mlp, bufs=work, ws=ws, device=DEV,
                       async_readback=async_readback)
    if async_readback:
        E.host_copies_done(DEV)
        torch.cuda.synchronize()
    # synchronous mode: no synchronisation of any kind between the last call and this read
    np.testing.assert_array_equal(host.numpy()[3:-3, 3:-3], ref)


def test_two_host_buffers_sharing_device_buffers():
    p, init_a, mlp = _case(1)
    _, init_b, _ = _case(2)
    ref_a, ref_b = _device_loop(p, init_a, mlp, 3), _device_loop(p, init_b, mlp, 3)
    ha, hb = torch.as_tensor(init_a).clone().pin_memory(), torch.as_tensor(init_b).clone().pin_memory()
    work = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
    ws = E.workspace(p.nx, p.ny, DEV)
    for _ in range(3):  # alternate the host buffers over the same device buffers, read-backs overlapped
        E.advance_host(ha, p, 1, "sr_f32", "transmissive", mlp_params=mlp, bufs=work, ws=ws, device=DEV,
                       async_readback=True)
        E.advance_host(hb, p, 1, "sr_f32", "transmissive", mlp_params=mlp, bufs=work, ws=ws, device=DEV,
                       async_readback=True)
    E.host_copies_done(DEV)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ha.numpy()[3:-3, 3:-3], ref_a)
    np.testing.assert_array_equal(hb.numpy()[3:-3, 3:-3], ref_b)
