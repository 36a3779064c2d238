"""GPU: the host-buffer entry (euler2d.advance_host) with its banded, overlapped copies equals the device loop
bit for bit over repeated calls, for both result slots (1 and 2 steps per call)."""
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


@pytest.mark.parametrize("per_call", [1, 2])
@pytest.mark.parametrize("pinned", [True, False])
def test_advance_host_equals_device_loop(per_call, pinned):
    n = 96
    p = Params(nx=n, ny=n - 7, x_length=1.0, y_length=0.9, cfl=0.4)
    init = problems.make_quadrant_state(p.nx, p.ny, problems.seeded_quadrant_states(1), 3)
    mlp = {k: v for k, v in np.load(MODELS_DIR / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}
    calls = 5
    bufs = [torch.as_tensor(init, device=DEV).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                      device=DEV) for _ in range(3)]
    res = E.run(bufs, p, 1.0e300, "sr_f32", "transmissive", mlp_params=mlp, fixed_steps=calls * per_call)
    ref = bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3]
    host = torch.as_tensor(init).clone()
    if pinned:
        host = host.pin_memory()
    work = [torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV) for _ in range(4)]
    ws = E.workspace(p.nx, p.ny, DEV)
    for _ in range(calls):
        E.advance_host(host, p, per_call, "sr_f32", "transmissive", mlp_params=mlp, bufs=work, ws=ws, device=DEV)
    E.host_copies_done(DEV)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host.numpy()[3:-3, 3:-3], ref)
