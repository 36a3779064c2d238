"""GPU at the benchmark sizes: one stage of the 2000 x 2000 seeded quadrant and of the 224 x 88 x 88
shock-bubble against the CPU oracle, and size-independent properties of the 2000 x 2000 step (periodic
conservation, x/y transpose symmetry)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import oracle as O
from weno_sr_publishing_b200 import euler2d as E
from weno_sr_publishing_b200 import euler3d as E3
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200.checkpoint import MODELS_DIR
from weno_sr_publishing_b200.params import Params

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
N = 2000
P32 = {k: v for k, v in np.load(MODELS_DIR / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}
PARAMS = {"js": None, "sr_f32": P32}
TOL = {"js": 1e-13, "sr_f32": 2e-6}


def _params():
    return Params(nx=N, ny=N, x_length=1.0, y_length=1.0, cfl=0.4)


@pytest.fixture(scope="module")
def quadrant():
    return problems.make_quadrant_state(N, N, problems.seeded_quadrant_states(0), 2)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("method", ["js", "sr_f32"])
def test_headline_stage_against_oracle(quadrant, method):
    p = _params()
    dt = E.compute_dt(torch.as_tensor(quadrant, device=DEV), p)
    assert dt == p.cfl * min(p.dx, p.dy) / O.max_speed(quadrant, N, N)
    u = torch.as_tensor(quadrant, device=DEV)
    out = torch.zeros_like(u)
    E.stage(u, u, out, p, dt, 1, method, "transmissive", PARAMS[method])
    ref = O.euler2d_stage(quadrant, quadrant, np.zeros_like(quadrant), N, N, p.dx, p.dy, dt, 1, method,
                          "transmissive", params=PARAMS[method])
    assert _rel(out.cpu().numpy()[3:-3, 3:-3], ref[3:-3, 3:-3]) <= TOL[method]


def test_headline_periodic_conservation(quadrant):
    p = _params()
    init = quadrant.copy()
    bufs = [torch.as_tensor(init, device=DEV).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                      device=DEV) for _ in range(3)]
    res = E.run(bufs, p, 1.0, "sr_f32", "periodic", mlp_params=P32, fixed_steps=3)
    m0 = init[3:-3, 3:-3].sum(axis=(0, 1))
    m1 = bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3].sum(axis=(0, 1))
    assert np.all(np.abs(m1 - m0) <= 1e-11 * np.abs(m0).max())


def test_headline_transpose_symmetry(quadrant):
    p = _params()
    tr = np.ascontiguousarray(quadrant.transpose(1, 0, 2)[..., [0, 2, 1, 3]])
    outs = []
    for u in (quadrant, tr):
        bufs = [torch.as_tensor(u, device=DEV).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                       device=DEV) for _ in range(3)]
        res = E.run(bufs, p, 1.0, "js", "transmissive", fixed_steps=2)
        outs.append(bufs[res.final_slot].cpu().numpy()[3:-3, 3:-3])
    back = outs[1].transpose(1, 0, 2)[..., [0, 2, 1, 3]]
    assert _rel(back, outs[0]) <= 1e-12


def test_shock_bubble_stage_against_oracle():
    sb = problems.ShockBubble.seeded(0)
    q0 = sb.state()
    dx, dy, dz = sb.spacing
    q = torch.as_tensor(q0, device=DEV).contiguous()
    dt = 0.4 * min(dx, dy, dz) / E3.max_speed(q, sb.nx, sb.ny, sb.nz)
    E3.stage(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, dt, 1, "sr_f32", "hllc", P32, inflow=sb.inflow())
    ref = np.array(q0, copy=True)
    O.euler3d_stage(ref, np.zeros_like(ref), sb.nx, sb.ny, sb.nz, dx, dy, dz, dt, 1, "sr_f32", "hllc", params=P32,
                    inflow=sb.inflow())
    assert _rel(q.cpu().numpy()[3:-3, 3:-3, 3:-3], ref[3:-3, 3:-3, 3:-3]) <= 2e-6
