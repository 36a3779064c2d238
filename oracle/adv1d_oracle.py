"""CPU oracle for batched 1D periodic linear advection with WENO5/WENO7 (JS or SR closure).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA 1D path and its CPU baseline. It restates, in
numpy, the reference's PyTorch code (paths inside the reference project, code/snapshot/):

  teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/
    weno5_core.py        158-239  features (+16/16 scale), plateau, candidates, omega_from_ratio,
                                  classical_omega (eps 1e-6, p 2)
    model.py             16-80    scale remap to +4/4, FP32 MLP, reflection average
    apost_advect_fvm.py  16-19    periodic 5-point stencils
    rk3_advection.py     82-186   signed upwind interface state, rhs, SSPRK3, cfl_schedule, rollout
  teacherfree_lab_weno5_v12_reflection_sym/v12_model.py 14-50 (FP64 MLP, same reflection)
  teacherfree_lab_weno7_rk4_distance_balanced_fast(-2)/
    weno7_core.py        28-324   WENO7 candidates, optimal weights, delta forms, features, gamma,
                                  plateau, omega (beta = 4 r), classical omega, MLP 6->24->16->16->4
    rk4_advection.py     31-220   7-point stencils, face states, L and L~ (reverse upwind), Shu RK4
  for_paper_results/run_gste.py 103-118 (GSTE schedule: steps = ceil(t/(cfl dx)), dt = t/steps)
  weno_z_borges_p2_results/torch_weno_z.py 14-79 (WENO5-Z: p 2, eps h^2, tau5 = |b0 - b2|; WENO7-Z: p 3,
                                  eps h^3, tau7 = |-b0 - 3 b1 + 3 b2 + b3|; velocity +1 in the reference)

Pinned by tests/test_adv1d_oracle.py against fixtures that tests/golden/make_golden_1d.py produced
by running the reference's own torch functions.

A closure is described by (kind, precision, packed parameters): kind 5 (189 parameters) or 7 (908),
precision "f64", "f32" or "bf16". JS weights use closure=None, WENO-Z weights closure="z".
"""
from __future__ import annotations

import math

import numpy as np

S3 = math.sqrt(3.0)

# ------------------------------------------------------------------------------------------------
# WENO5
# ------------------------------------------------------------------------------------------------
D5 = {1: np.array([0.1, 0.6, 0.3]), 2: np.array([0.3, 0.6, 0.1])}


def stencils(u: np.ndarray, width: int) -> np.ndarray:
    """Periodic stencils centred on each cell: (n, width)."""
    h = width // 2
    up = np.concatenate([u[-h:], u, u[:h]])
    idx = np.arange(u.size)[:, None] + np.arange(width)[None, :]
    return up[idx]


def candidates5(q: np.ndarray, lr: int) -> np.ndarray:
    q0, q1, q2, q3, q4 = q.T
    if lr == 1:
        return np.stack([(1 / 3) * q0 - (7 / 6) * q1 + (11 / 6) * q2,
                         -(1 / 6) * q1 + (5 / 6) * q2 + (1 / 3) * q3,
                         (1 / 3) * q2 + (5 / 6) * q3 - (1 / 6) * q4], axis=1)
    return np.stack([-(1 / 6) * q0 + (5 / 6) * q1 + (1 / 3) * q2,
                     (1 / 3) * q1 + (5 / 6) * q2 - (1 / 6) * q3,
                     (11 / 6) * q2 - (7 / 6) * q3 + (1 / 3) * q4], axis=1)


def deltas5(q):
    q0, q1, q2, q3, q4 = q.T
    d20, d21, d22 = q0 - 2 * q1 + q2, q1 - 2 * q2 + q3, q2 - 2 * q3 + q4
    return np.stack([(13 / 12) * np.abs(d20) + 0.25 * np.abs(q0 - 4 * q1 + 3 * q2),
                     (13 / 12) * np.abs(d21) + 0.25 * np.abs(q1 - q3),
                     (13 / 12) * np.abs(d22) + 0.25 * np.abs(3 * q2 - 4 * q3 + q4)], axis=1)


def gamma_s(q):
    eps = 1.0e-15
    d2 = q[:, :-2] - 2.0 * q[:, 1:-1] + q[:, 2:]
    den = np.abs(q[:, 1:-1] - q[:, :-2]) + np.abs(q[:, 2:] - q[:, 1:-1]) + eps
    return np.clip(np.max(np.abs(d2) / den, axis=1), 0.0, 1.0)


def plateau(q, deltas):
    qs = np.maximum(np.max(np.abs(q), axis=1), 1.0)
    return np.max(deltas, axis=1) <= 1.0e-13 * qs


def features(q, deltas, scale_offset: float):
    """(norm deltas..., gamma, clip((log10(rel) + off)/off)); WENO5 deploys off=4, WENO7 off=16."""
    dmax = np.max(deltas, axis=1)
    norm = deltas / np.maximum(dmax, 1.0e-15)[:, None]
    qs = np.maximum(np.max(np.abs(q), axis=1), 1.0)
    rel = np.maximum(dmax / qs, 1.0e-30)
    sc = np.clip((np.log10(rel) + scale_offset) / scale_offset, 0.0, 1.0)
    return np.concatenate([norm, gamma_s(q)[:, None], sc[:, None]], axis=1)


# ------------------------------------------------------------------------------------------------
# MLP with reflection average
# ------------------------------------------------------------------------------------------------
def unpack(kind: int, packed: np.ndarray) -> list[np.ndarray]:
    dims = (5, 10, 6, 6, 3) if kind == 5 else (6, 24, 16, 16, 4)
    out, o = [], 0
    for a, b in zip(dims[:-1], dims[1:]):
        out.append(packed[o:o + a * b].reshape(a, b))
        o += a * b
        out.append(packed[o:o + b])
        o += b
    if o != packed.size:
        raise ValueError(f"expected {o} parameters, got {packed.size}")
    return out


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32)
    return np.where(np.isfinite(x), out, x)


def mlp(x: np.ndarray, params: list[np.ndarray], prec: str) -> np.ndarray:
    """softmax(6 tanh(raw/6)) of the swish MLP, in the closure precision; returned as float64."""
    if prec == "f64":
        h = x.astype(np.float64)
        ws = [p.astype(np.float64) for p in params]
        rnd = lambda a: a  # noqa: E731
    else:
        h = x.astype(np.float32)
        ws = [p.astype(np.float32) for p in params]
        rnd = bf16 if prec == "bf16" else (lambda a: a)  # noqa: E731
        if prec == "bf16":
            h = bf16(h)
            ws = [bf16(p) for p in ws]
    for layer in range(3):
        z = h @ ws[2 * layer] + ws[2 * layer + 1]
        h = rnd(z / (1 + np.exp(-z)))
    raw = h @ ws[6] + ws[7]
    bad = 6 * np.tanh(raw / 6)
    e = np.exp(bad - np.max(bad, axis=1, keepdims=True))
    return (e / np.sum(e, axis=1, keepdims=True)).astype(np.float64)


def reflected_ratios(x: np.ndarray, kind: int, params, prec: str) -> np.ndarray:
    nd = 3 if kind == 5 else 4
    xr = np.concatenate([x[:, :nd][:, ::-1], x[:, nd:]], axis=1)
    return 0.5 * (mlp(x, params, prec) + mlp(xr, params, prec)[:, ::-1])


# ------------------------------------------------------------------------------------------------
# WENO7
# ------------------------------------------------------------------------------------------------
C7 = {
    1: np.array([[-1 / 4, 13 / 12, -23 / 12, 25 / 12], [1 / 12, -5 / 12, 13 / 12, 1 / 4],
                 [-1 / 12, 7 / 12, 7 / 12, -1 / 12], [1 / 4, 13 / 12, -5 / 12, 1 / 12]]),
    2: np.array([[1 / 12, -5 / 12, 13 / 12, 1 / 4], [-1 / 12, 7 / 12, 7 / 12, -1 / 12],
                 [1 / 4, 13 / 12, -5 / 12, 1 / 12], [25 / 12, -23 / 12, 13 / 12, -1 / 4]]),
}
D7 = {1: np.array((1.0, 12.0, 18.0, 4.0)) / 35.0, 2: np.array((4.0, 18.0, 12.0, 1.0)) / 35.0}
DELTA7_COEFF = np.array((1.0 / 36.0, 13.0 / 12.0, 781.0 / 720.0))


def delta_forms7(q):
    q0, q1, q2, q3, q4, q5, q6 = q.T
    return np.stack([
        np.stack([-2 * q0 + 9 * q1 - 18 * q2 + 11 * q3, -q0 + 4 * q1 - 5 * q2 + 2 * q3, -q0 + 3 * q1 - 3 * q2 + q3], -1),
        np.stack([q1 - 6 * q2 + 3 * q3 + 2 * q4, q2 - 2 * q3 + q4, -q1 + 3 * q2 - 3 * q3 + q4], -1),
        np.stack([-2 * q2 - 3 * q3 + 6 * q4 - q5, q2 - 2 * q3 + q4, -q2 + 3 * q3 - 3 * q4 + q5], -1),
        np.stack([-11 * q3 + 18 * q4 - 9 * q5 + 2 * q6, 2 * q3 - 5 * q4 + 4 * q5 - q6, -q3 + 3 * q4 - 3 * q5 + q6], -1),
    ], axis=1)


def candidates7(q, lr):
    c = C7[lr]
    return np.stack([np.sum(q[:, k:k + 4] * c[k], axis=1) for k in range(4)], axis=1)


# ------------------------------------------------------------------------------------------------
# Reconstruction at both physical faces of every cell's stencil
# ------------------------------------------------------------------------------------------------
def beta5(q):
    q0, q1, q2, q3, q4 = q.T
    return np.stack([(13 / 12) * (q0 - 2 * q1 + q2) ** 2 + 0.25 * (q0 - 4 * q1 + 3 * q2) ** 2,
                     (13 / 12) * (q1 - 2 * q2 + q3) ** 2 + 0.25 * (q1 - q3) ** 2,
                     (13 / 12) * (q2 - 2 * q3 + q4) ** 2 + 0.25 * (3 * q2 - 4 * q3 + q4) ** 2], axis=1)


def face_values(u: np.ndarray, scheme: int, closure, h: float | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Left and right states at face i+1/2 for every i (lr=1 of cell i, lr=2 of cell i+1); h is the cell
    width (WENO-Z only)."""
    width = 5 if scheme == 5 else 7
    q = stencils(u, width)
    if scheme == 5:
        dl = deltas5(q)
        cand = {1: candidates5(q, 1), 2: candidates5(q, 2)}
        dtab, bscale, off = D5, 3.0, 4.0
        beta_cls = None
    else:
        forms = delta_forms7(q)
        dl = np.sum(np.abs(forms) * DELTA7_COEFF, axis=-1)
        cand = {1: candidates7(q, 1), 2: candidates7(q, 2)}
        dtab, bscale, off = D7, 4.0, 16.0
        beta_cls = np.sum(forms * forms * DELTA7_COEFF, axis=-1)
    vals = {}
    if isinstance(closure, str) and closure == "z":
        if h is None:
            raise ValueError("WENO-Z needs the cell width h")
        if scheme == 5:
            beta = beta5(q)
            tau, eps, p = np.abs(beta[:, 0] - beta[:, 2]), h ** 2, 2
        else:
            beta = beta_cls
            tau, eps, p = np.abs(-beta[:, 0] - 3.0 * beta[:, 1] + 3.0 * beta[:, 2] + beta[:, 3]), h ** 3, 3
        ratio = tau[:, None] / (beta + eps)
        for lr in (1, 2):
            a = dtab[lr][None, :] * (1.0 + ratio ** p)
            w = a / np.sum(a, axis=1, keepdims=True)
            vals[lr] = np.sum(w * cand[lr], axis=1)
    elif closure is None:
        beta = beta5(q) if scheme == 5 else beta_cls
        for lr in (1, 2):
            a = dtab[lr][None, :] / np.square(beta + 1.0e-6)
            w = a / np.sum(a, axis=1, keepdims=True)
            vals[lr] = np.sum(w * cand[lr], axis=1)
    else:
        kind, prec, packed = closure
        params = unpack(kind, np.asarray(packed, dtype=np.float64))
        plat = plateau(q, dl)
        x = features(q, dl, off)
        r = reflected_ratios(x, kind, params, prec)
        for lr in (1, 2):
            a = dtab[lr][None, :] / np.power(bscale * r + 1.0e-12, 2.0)
            w = a / np.sum(a, axis=1, keepdims=True)
            w = np.where(plat[:, None], dtab[lr][None, :], w)
            vals[lr] = np.sum(w * cand[lr], axis=1)
    left = vals[1]
    right = np.roll(vals[2], -1)
    return left, right


def rhs(u, a, dx, scheme, closure, reverse=False):
    left, right = face_values(u, scheme, closure, dx)
    face = (right if a > 0 else left) if reverse else (left if a > 0 else right)
    flux = a * face
    return -(flux - np.roll(flux, 1)) * (1.0 / dx)


def ssprk3_step(u, a, dt, dx, scheme, closure):
    """rk3_advection.py:118-131."""
    u1 = u + dt * rhs(u, a, dx, scheme, closure)
    u2 = 0.75 * u + 0.25 * (u1 + dt * rhs(u1, a, dx, scheme, closure))
    return u / 3.0 + (2.0 / 3.0) * (u2 + dt * rhs(u2, a, dx, scheme, closure))


def shu_rk4_step(u, a, dt, dx, scheme, closure):
    """rk4_advection.py:137-195: L and the downwind operator L~ share the face states."""
    l0 = rhs(u, a, dx, scheme, closure)
    lt0 = rhs(u, a, dx, scheme, closure, reverse=True)
    u1 = u + 0.5 * dt * l0
    l1 = rhs(u1, a, dx, scheme, closure)
    lt1 = rhs(u1, a, dx, scheme, closure, reverse=True)
    u2 = (649.0 / 1600.0) * u - (10890423.0 / 25193600.0) * dt * lt0 + (951.0 / 1600.0) * u1 \
        + (5000.0 / 7873.0) * dt * l1
    l2 = rhs(u2, a, dx, scheme, closure)
    u3 = (53989.0 / 2500000.0) * u - (102261.0 / 5000000.0) * dt * lt0 + (4806213.0 / 20000000.0) * u1 \
        - (5121.0 / 20000.0) * dt * lt1 + (23619.0 / 32000.0) * u2 + (7873.0 / 10000.0) * dt * l2
    l3 = rhs(u3, a, dx, scheme, closure)
    return (1.0 / 5.0) * u + (1.0 / 10.0) * dt * l0 + (6127.0 / 30000.0) * u1 + (1.0 / 6.0) * dt * l1 \
        + (7873.0 / 30000.0) * u2 + (1.0 / 3.0) * u3 + (1.0 / 6.0) * dt * l3


def cfl_schedule(distance_cells: float, cfl: float) -> list[float]:
    """rk3_advection.py:149-168: full CFL steps plus one shortened step."""
    full = int(math.floor(distance_cells / cfl))
    rem = distance_cells - full * cfl
    tol = 2.0e-13 * max(1.0, distance_cells)
    if rem < tol:
        rem = 0.0
    elif cfl - rem < tol:
        full += 1
        rem = 0.0
    sched = [float(cfl)] * full
    if rem > 0.0:
        sched.append(float(rem))
    if not sched:
        sched.append(float(distance_cells))
    return sched


def run(u0, a, dx, dts, scheme, closure, integrator):
    u = np.array(u0, dtype=np.float64, copy=True)
    step = ssprk3_step if integrator == "ssprk3" else shu_rk4_step
    for dt in dts:
        u = step(u, a, dt, dx, scheme, closure)
    return u
