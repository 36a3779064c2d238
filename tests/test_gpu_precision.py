"""GPU: the precision contract of the reduced-precision closures on the 2D Euler path.

The FP32 and BF16 closures (features normalised in single precision, hardware exp/reciprocal approximations in
the MLP) stand in for the FP64 closure only within a stated bound on the density they produce. Each case runs
the seeded four-quadrant Riemann problem at 400^2 (unit square, transmissive, HLLC, SSPRK3, CFL 0.4) to
t = 0.25 three times with the SAME checkpoint's weights, the closure evaluated in FP64, FP32 and BF16, and
compares the final densities in the L1 norm (sum |rho_a - rho_b| dx dy over the interior):

  FP32 closure vs FP64 closure: <= 1e-8
  BF16 closure vs FP64 closure: <= 5e-4

and, for scale, both differences against the difference between the FP64 closure and WENO5-JS on the same
problem (the effect of the closure itself)."""
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
N = 400
T_END = 0.25
BOUND = {"sr_f32": 1.0e-8, "sr_bf16": 5.0e-4}
MLP = {k: v for k, v in np.load(MODELS_DIR / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}


def _final_density(init: np.ndarray, p: Params, method: str) -> np.ndarray:
    bufs = [torch.as_tensor(init, device=DEV).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                      device=DEV) for _ in range(3)]
    res = E.run(bufs, p, T_END, method, "transmissive", mlp_params=None if method == "js" else MLP)
    assert abs(res.t - T_END) <= 1e-14, res.t
    return bufs[res.final_slot][3:3 + p.ny, 3:3 + p.nx, 0].cpu().numpy()


@pytest.fixture(scope="module")
def runs():
    p = Params(nx=N, ny=N, x_length=1.0, y_length=1.0, cfl=0.4, t_end=T_END)
    out = {}
    for seed in range(4):
        init = problems.make_quadrant_state(N, N, problems.seeded_quadrant_states(seed), quadrature=1)
        out[seed] = {m: _final_density(init, p, m) for m in ("sr_f64", "sr_f32", "sr_bf16", "js")}
    return p, out


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("method", ["sr_f32", "sr_bf16"])
def test_closure_precision_density_l1(runs, seed, method):
    p, out = runs
    r = out[seed]
    l1 = float(np.abs(r[method] - r["sr_f64"]).sum() * p.dx * p.dy)
    closure_effect = float(np.abs(r["js"] - r["sr_f64"]).sum() * p.dx * p.dy)
    print(f"seed {seed}: {method} vs sr_f64 density L1 {l1:.3e}; js vs sr_f64 {closure_effect:.3e}")
    assert np.isfinite(r[method]).all()
    assert l1 <= BOUND[method], l1
    assert l1 < 0.1 * closure_effect  # the precision loss is small against what the closure changes
