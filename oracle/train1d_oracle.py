"""CPU oracle of the closure-training objective and its gradients (torch autograd on CPU).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA training kernels (forward loss, hand-written adjoint).
It restates, in torch, the reference's differentiable WENO5-SR step (paths inside the reference project,
code/snapshot/teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/):

  weno5_core.py    135-239  gamma, deltas, features (+16/16 scale), plateau mask, candidates, optimal
                            weights, omega_from_ratio (beta = 3 r, power 2, eps 1e-12)
  model.py          16-80   scale remap to +4/4, FP32 MLP (FP64 features cast right before the first
                            layer, ratios cast back), reflection average 0.5 (M(x) + P M(Px))
  teacherfree_lab_weno5_v9_exact_fvm/v9_model.py (FP64 MLP with the same remap)
  rk3_advection.py  71-131  upwind face state per velocity sign, signed rhs, SSPRK3
  fast_losses.py   412-648  rollout with the state in the graph, exact targets at every completed step

with the plain L1 objective  L = mean over (trajectory, completed step, cell) of |u - e|. Gradients are
torch autograd's, so their conventions at non-smooth points (|x| at 0, ties of maximum, max over a
dimension, clamp bounds) are the reference's by construction.

Pinned by tests/test_train1d_oracle.py against gradients that tests/golden/make_golden_train.py produced
by running the reference's own torch functions under autograd.
"""
from __future__ import annotations

import torch

NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")
SHAPES = {"w1": (5, 10), "b1": (10,), "w2": (10, 6), "b2": (6,), "w3": (6, 6), "b3": (6,), "w4": (6, 3), "b4": (3,)}


def unpack(packed, dtype=torch.float64, requires_grad: bool = True) -> dict:
    """189 packed values -> {w1..b4} leaf tensors."""
    flat = torch.as_tensor(packed, dtype=torch.float64)
    out, o = {}, 0
    for k in NAMES:
        size = 1
        for s in SHAPES[k]:
            size *= s
        out[k] = flat[o:o + size].reshape(SHAPES[k]).to(dtype).clone().requires_grad_(requires_grad)
        o += size
    return out


def stencils(u: torch.Tensor) -> torch.Tensor:
    """[B, n] -> [B, n, 5] periodic stencils u[i-2 .. i+2]."""
    return torch.stack([torch.roll(u, 2 - k, dims=1) for k in range(5)], dim=-1)


def features(q: torch.Tensor):
    """(MLP inputs with the +4/4 scale, plateau mask) of stencils q [..., 5]."""
    q0, q1, q2, q3, q4 = q.unbind(-1)
    dl = [(13.0 / 12.0) * torch.abs(q0 - 2.0 * q1 + q2) + 0.25 * torch.abs(q0 - 4.0 * q1 + 3.0 * q2),
          (13.0 / 12.0) * torch.abs(q1 - 2.0 * q2 + q3) + 0.25 * torch.abs(q1 - q3),
          (13.0 / 12.0) * torch.abs(q2 - 2.0 * q3 + q4) + 0.25 * torch.abs(3.0 * q2 - 4.0 * q3 + q4)]
    dmax = torch.maximum(torch.maximum(dl[0], dl[1]), dl[2])
    inv = 1.0 / torch.clamp(dmax, min=1.0e-15)
    eps = 1.0e-15
    g = [torch.abs(q0 - 2.0 * q1 + q2) / (torch.abs(q1 - q0) + torch.abs(q2 - q1) + eps),
         torch.abs(q1 - 2.0 * q2 + q3) / (torch.abs(q2 - q1) + torch.abs(q3 - q2) + eps),
         torch.abs(q2 - 2.0 * q3 + q4) / (torch.abs(q3 - q2) + torch.abs(q4 - q3) + eps)]
    gamma = torch.clamp(torch.maximum(torch.maximum(g[0], g[1]), g[2]), 0.0, 1.0)
    qscale = torch.clamp(torch.max(torch.abs(q), dim=-1).values, min=1.0)
    rel = torch.clamp(dmax / qscale, min=1.0e-30)
    old = torch.clamp((torch.log10(rel) + 16.0) / 16.0, 0.0, 1.0)
    scale = torch.clamp((16.0 * old - 16.0 + 4.0) / 4.0, 0.0, 1.0)
    x = torch.stack((dl[0] * inv, dl[1] * inv, dl[2] * inv, gamma, scale), dim=-1)
    return x, dmax <= 1.0e-13 * qscale


def mlp(x: torch.Tensor, p: dict) -> torch.Tensor:
    """softmax(6 tanh(raw/6)) of the swish MLP in the parameters' dtype; returned in x's dtype."""
    h = x.to(p["w1"].dtype)
    for layer in (1, 2, 3):
        h = h @ p[f"w{layer}"] + p[f"b{layer}"]
        h = h * torch.sigmoid(h)
    raw = h @ p["w4"] + p["b4"]
    return torch.softmax(6.0 * torch.tanh(raw / 6.0), dim=-1).to(x.dtype)


def ratios(x: torch.Tensor, p: dict) -> torch.Tensor:
    xr = torch.stack((x[..., 2], x[..., 1], x[..., 0], x[..., 3], x[..., 4]), dim=-1)
    return 0.5 * (mlp(x, p) + mlp(xr, p).flip(-1))


D = {1: (0.1, 0.6, 0.3), 2: (0.3, 0.6, 0.1)}


def candidates(q: torch.Tensor, lr: int) -> torch.Tensor:
    q0, q1, q2, q3, q4 = q.unbind(-1)
    if lr == 1:
        return torch.stack(((1.0 / 3.0) * q0 - (7.0 / 6.0) * q1 + (11.0 / 6.0) * q2,
                            -(1.0 / 6.0) * q1 + (5.0 / 6.0) * q2 + (1.0 / 3.0) * q3,
                            (1.0 / 3.0) * q2 + (5.0 / 6.0) * q3 - (1.0 / 6.0) * q4), dim=-1)
    return torch.stack((-(1.0 / 6.0) * q0 + (5.0 / 6.0) * q1 + (1.0 / 3.0) * q2,
                        (1.0 / 3.0) * q1 + (5.0 / 6.0) * q2 - (1.0 / 6.0) * q3,
                        (11.0 / 6.0) * q2 - (7.0 / 6.0) * q3 + (1.0 / 3.0) * q4), dim=-1)


def head(q, r, plateau, lr: int) -> torch.Tensor:
    d = torch.tensor(D[lr], dtype=torch.float64)
    alpha = d / torch.pow(3.0 * r + 1.0e-12, 2.0)
    omega = alpha / torch.sum(alpha, dim=-1, keepdim=True)
    omega = torch.where(plateau[..., None], d.expand_as(omega), omega)
    return torch.sum(omega * candidates(q, lr), dim=-1)


def rhs(u: torch.Tensor, vel: torch.Tensor, dxinv: float, p: dict) -> torch.Tensor:
    q = stencils(u)
    x, plat = features(q)
    r = ratios(x, p)
    pos = head(q, r, plat, 1)
    neg = torch.roll(head(q, r, plat, 2), -1, dims=1)
    face = torch.where((vel > 0.0)[:, None], pos, neg)
    flux = vel[:, None] * face
    return -(flux - torch.roll(flux, 1, dims=1)) * dxinv


def ssprk3(u, vel, dt, dxinv, p):
    u1 = u + dt * rhs(u, vel, dxinv, p)
    u2 = 0.75 * u + 0.25 * (u1 + dt * rhs(u1, vel, dxinv, p))
    return u / 3.0 + (2.0 / 3.0) * (u2 + dt * rhs(u2, vel, dxinv, p))


def trajectory_loss(p: dict, u0: torch.Tensor, targets: torch.Tensor, vel: torch.Tensor, dt: float, dxinv: float):
    """(loss, final state): targets [B, S, n] are the exact averages after steps 1..S."""
    u = u0
    total = torch.zeros((), dtype=torch.float64)
    S = targets.shape[1]
    for k in range(S):
        u = ssprk3(u, vel, dt, dxinv, p)
        total = total + torch.sum(torch.abs(u - targets[:, k]))
    return total / (u0.shape[0] * S * u0.shape[1]), u


def loss_and_grads(packed, u0, targets, vel, dt: float, dxinv: float, precision: str = "f64"):
    """(loss, dL/dtheta packed [189] FP64, dL/du0 [B, n], final state) as numpy arrays."""
    dtype = torch.float32 if precision == "f32" else torch.float64
    p = unpack(packed, dtype)
    u = torch.as_tensor(u0, dtype=torch.float64).clone().requires_grad_(True)
    loss, final = trajectory_loss(p, u, torch.as_tensor(targets, dtype=torch.float64),
                                  torch.as_tensor(vel, dtype=torch.float64), dt, dxinv)
    grads = torch.autograd.grad(loss, [p[k] for k in NAMES] + [u])
    g = torch.cat([t.reshape(-1).to(torch.float64) for t in grads[:-1]])
    return float(loss.detach()), g.numpy(), grads[-1].numpy(), final.detach().numpy()
