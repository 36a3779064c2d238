"""GPU: the host-buffer entry (euler2d.advance_host -> wsr_euler2d_advance_host) equals the device loop bit for
bit over repeated calls, for both result slots (1 and 2 steps per call), with the copies and the first and last
stages in one band or several: synchronous by default (the host buffer holds the result when the call returns),
and with the overlapped read-back once host_copies_done() and a synchronisation, or host_wait(), have run. Two
host buffers that share the same device buffers keep their results apart; ghost cells of the host array are left
as they were."""
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
MLP = {k: v for k, v in np.load(MODELS_DIR / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}


def _case(seed=1):
    n = 96
    p = Params(nx=n, ny=n - 7, x_length=1.0, y_length=0.9, cfl=0.4)
    init = problems.make_quadrant_state(p.nx, p.ny, problems.seeded_quadrant_states(seed), 3)
    return p, init


def _device_loop(p, init, steps, method="sr_f32", boundary="transmissive"):
    bufs = [torch.as_tensor(init, device=DEV).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                      device=DEV) for _ in range(3)]
    mlp = MLP if method != "js" else None
    res = E.run(bufs, p, 1.0e300, method, boundary, mlp_params=mlp, fixed_steps=steps)
    return bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3]


@pytest.mark.parametrize("bands", [0, 5])
@pytest.mark.parametrize("per_call", [1, 2])
@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("async_readback", [False, True])
def test_advance_host_equals_device_loop(bands, per_call, pinned, async_readback):
    p, init = _case()
    calls = 5
    ref = _device_loop(p, init, calls * per_call)
    host = torch.as_tensor(init).clone()
    if pinned:
        host = host.pin_memory()
    work = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
    ws = E.workspace(p.nx, p.ny, DEV)
    for _ in range(calls):
        E.advance_host(host, p, per_call, "sr_f32", "transmissive", mlp_params=MLP, bufs=work, ws=ws, device=DEV,
                       async_readback=async_readback, bands=bands)
    if async_readback:
        E.host_copies_done(DEV)
        torch.cuda.synchronize()
    # synchronous mode: no synchronisation of any kind between the last call and this read
    np.testing.assert_array_equal(host.numpy()[3:-3, 3:-3], ref)
    if async_readback:
        assert E.host_wait(DEV)["steps"] == calls * per_call


@pytest.mark.parametrize("method,boundary", [("js", "transmissive"), ("js", "periodic"), ("sr_f32", "periodic"),
                                             ("z", "transmissive")])
def test_banded_stages_equal_device_loop(method, boundary):
    """Many small bands (down to 5 rows) through the first-stage and last-stage band logic, both boundaries."""
    p, init = _case(3)
    ref = _device_loop(p, init, 3, method, boundary)
    for bands in (2, 7, 16):
        host = torch.as_tensor(init).clone().pin_memory()
        work = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
        for _ in range(3):
            E.advance_host(host, p, 1, method, boundary, mlp_params=MLP if method != "js" else None, bufs=work,
                           device=DEV, async_readback=True, bands=bands)
        assert E.host_wait(DEV)["steps"] == 3
        np.testing.assert_array_equal(host.numpy()[3:-3, 3:-3], ref)


def test_ghost_cells_of_the_host_array_are_kept():
    p, init = _case(2)
    host = torch.as_tensor(init).clone().pin_memory()
    host[:3] = 7.0
    host[:, :3] = -3.0
    before = host.clone()
    E.advance_host(host, p, 1, "js", "transmissive", device=DEV, bands=4)
    h, b = host.numpy(), before.numpy()
    np.testing.assert_array_equal(h[:3], b[:3])
    np.testing.assert_array_equal(h[-3:], b[-3:])
    np.testing.assert_array_equal(h[:, :3], b[:, :3])
    np.testing.assert_array_equal(h[:, -3:], b[:, -3:])
    assert not np.array_equal(h[3:-3, 3:-3], b[3:-3, 3:-3])


def test_two_host_buffers_sharing_device_buffers():
    p, init_a = _case(1)
    _, init_b = _case(2)
    ref_a, ref_b = _device_loop(p, init_a, 3), _device_loop(p, init_b, 3)
    ha, hb = torch.as_tensor(init_a).clone().pin_memory(), torch.as_tensor(init_b).clone().pin_memory()
    work = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
    ws = E.workspace(p.nx, p.ny, DEV)
    for _ in range(3):  # alternate the host buffers over the same device buffers, read-backs overlapped
        E.advance_host(ha, p, 1, "sr_f32", "transmissive", mlp_params=MLP, bufs=work, ws=ws, device=DEV,
                       async_readback=True, bands=3)
        E.advance_host(hb, p, 1, "sr_f32", "transmissive", mlp_params=MLP, bufs=work, ws=ws, device=DEV,
                       async_readback=True, bands=3)
    E.host_copies_done(DEV)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ha.numpy()[3:-3, 3:-3], ref_a)
    np.testing.assert_array_equal(hb.numpy()[3:-3, 3:-3], ref_b)
    assert E.host_wait(DEV)["steps"] == 6


def test_invalid_host_arguments_raise():
    p, init = _case()
    with pytest.raises(ValueError):
        E.advance_host(np.zeros((5, 5, 4)), p, 1, "js", "transmissive", device=DEV)
    with pytest.raises(ValueError):
        E.advance_host(torch.as_tensor(init).clone(), p, 0, "js", "transmissive", device=DEV)


def test_device_work_on_the_buffers_waits_for_the_read_back():
    """An overlapped read-back of bufs[3] is still in flight when a device loop on the same buffers overwrites
    bufs[3]: the loop is ordered after the read-back, so the host array holds the host-buffer call's result."""
    p, init = _case(4)
    want = _device_loop(p, init, 1)
    host = torch.as_tensor(init).clone().pin_memory()
    work = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
    E.advance_host(host, p, 1, "sr_f32", "transmissive", mlp_params=MLP, bufs=work, device=DEV, async_readback=True)
    other = problems.make_quadrant_state(p.nx, p.ny, problems.seeded_quadrant_states(5), 3)
    work[0].copy_(torch.as_tensor(other, device=DEV))
    E.run(work, p, 1.0e300, "sr_f32", "transmissive", mlp_params=MLP, fixed_steps=3)
    E.host_wait(DEV)
    np.testing.assert_array_equal(host.numpy()[3:-3, 3:-3], want)
