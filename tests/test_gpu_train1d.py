"""CUDA closure training (forward loss + hand-written adjoint) against the reference's autograd gradients,
the autograd oracle, finite differences and size-independent properties."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import train1d_oracle as O
from weno_sr_publishing_b200 import adv1d as D
from weno_sr_publishing_b200 import profiles as P
from weno_sr_publishing_b200 import train1d as T

pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden"
M = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
DEV = "cuda:0"
CASES = ("trained_f64", "trained_f32", "perturbed_f64", "init_f64", "init_f32")
# parameter-gradient tolerances (max-norm relative): FP64 closures differ from autograd only in rounding;
# the FP32 closure differs in the MLP's exp/reciprocal rounding
GTOL = {"f64": 1e-9, "f32": 2e-3}


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _batch(desc, vel, n, steps, u0=None, every=32):
    dev = torch.device(DEV)
    return T.TrajectoryBatch(torch.as_tensor(np.asarray(desc, dtype=np.float64), device=dev),
                             torch.as_tensor(np.asarray(vel, dtype=np.float64), device=dev), n, steps, 0.5 / n,
                             None if u0 is None else torch.as_tensor(np.asarray(u0), device=dev), every)


def _fixture(case):
    g = np.load(G / "train1d_grads.npz")
    return {k[len(case) + 1:]: g[k] for k in g.files if k.startswith(case + "_")}


@pytest.mark.parametrize("case", CASES)
def test_matches_reference_autograd_fixture(case):
    f = _fixture(case)
    prec = "f32" if case.endswith("f32") else "f64"
    n, steps = int(f["n"]), int(f["steps"])
    b = _batch(f["desc"], f["vel"], n, steps, f["u0"], every=3)
    loss, grad, gu0, final = T.loss_and_grads(f["params"], b, prec, want_u0=True)
    ltol = 1e-12 if prec == "f64" else 1e-6
    assert abs(float(loss) - float(f["loss"])) <= ltol * float(f["loss"])
    assert _rel(final.cpu().numpy(), f["final"]) <= (1e-12 if prec == "f64" else 2e-6)
    assert _rel(grad.cpu().numpy(), f["grad"]) <= GTOL[prec], _rel(grad.cpu().numpy(), f["grad"])
    # dL/du0 is ill-conditioned at stencils just above the plateau threshold (max delta ~1e-13: the
    # normalised deltas and gamma divide by differences at rounding level, and autograd itself differs
    # by a few percent there from the same formulas evaluated in another order), so it is compared in
    # norm here and tightly on smooth profiles below
    assert _nrel(gu0.cpu().numpy(), f["grad_u0"]) <= 5e-2


def test_initial_state_from_profiles_matches_host_averages():
    rng = np.random.default_rng(1)
    n, B = 96, 14
    desc, _ = P.make_profiles(rng, B, n)
    vel = T.balanced_velocities(B)
    p = np.concatenate([np.load(M / "weno5_sr_fp64_step012250.npz")[k].reshape(-1) for k in T.PARAM_NAMES])
    gpu0, _, _, fin0 = T.loss_and_grads(p, _batch(desc, vel, n, 5), "f64")
    u0 = P.cell_averages(desc, n, 0.0)
    gpu1, _, _, fin1 = T.loss_and_grads(p, _batch(desc, vel, n, 5, u0), "f64")
    assert _rel(fin0.cpu().numpy(), fin1.cpu().numpy()) <= 1e-13
    assert abs(float(gpu0) - float(gpu1)) <= 1e-10 * float(gpu1)


def test_forward_states_equal_the_1d_path():
    rng = np.random.default_rng(2)
    n, B, steps = 64, 8, 9
    desc, _ = P.make_profiles(rng, B, n)
    vel = T.balanced_velocities(B)
    u0 = P.cell_averages(desc, n, 0.0)
    p = np.concatenate([np.load(M / "weno5_sr_fp32_step016500.npz")[k].reshape(-1).astype(np.float64)
                        for k in T.PARAM_NAMES])
    for prec in ("f64", "f32"):
        _, _, _, fin = T.loss_and_grads(p, _batch(desc, vel, n, steps, u0), prec)
        outs, _ = D.run_batched(list(u0), vel, 1.0 / n, steps, 0.5 / n, scheme=5,
                                model=D.Closure(5, p, prec), device=DEV)
        assert np.array_equal(fin.cpu().numpy(), torch.stack(outs).cpu().numpy())


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gradients_match_oracle_multi_segment(prec):
    """B = 12 mixed families, N = 48, 37 steps with checkpoints every 8 (five segments)."""
    rng = np.random.default_rng(7)
    n, B, steps = 48, 12, 37
    desc, _ = P.make_profiles(rng, B, n)
    vel = T.balanced_velocities(B)
    src = "weno5_sr_fp64_step012250.npz" if prec == "f64" else "weno5_sr_fp32_step016500.npz"
    p = np.concatenate([np.load(M / src)[k].reshape(-1).astype(np.float64) for k in T.PARAM_NAMES])
    u0 = P.cell_averages(desc, n, 0.0)
    targets = np.stack([P.cell_averages(desc, n, vel * (k * 0.5 / n)) for k in range(1, steps + 1)], axis=1)
    lo, go, guo, fo = O.loss_and_grads(p, u0, targets, vel, 0.5 / n, float(n), prec)
    loss, grad, gu0, fin = T.loss_and_grads(p, _batch(desc, vel, n, steps, u0, every=8), prec, want_u0=True)
    assert abs(float(loss) - lo) <= (1e-11 if prec == "f64" else 1e-5) * lo
    assert _rel(grad.cpu().numpy(), go) <= GTOL[prec]
    assert _nrel(gu0.cpu().numpy(), guo) <= 5e-2


LONG = dict(n=64, B=4, steps=2048, every=32)  # 1024 cells of propagation at CFL 0.5, 64 checkpoint segments


def _long_case(prec):
    rng = np.random.default_rng(31)
    n, B, steps = LONG["n"], LONG["B"], LONG["steps"]
    desc, _ = P.make_profiles(rng, B, n)
    vel = T.balanced_velocities(B)
    src = "weno5_sr_fp64_step012250.npz" if prec == "f64" else "weno5_sr_fp32_step016500.npz"
    p = np.concatenate([np.load(M / src)[k].reshape(-1).astype(np.float64) for k in T.PARAM_NAMES])
    u0 = P.cell_averages(desc, n, 0.0)
    return desc, vel, p, u0


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gradients_match_oracle_at_1024_cells_of_propagation(prec):
    """The unroll length of the training workload's longest distance: B = 4 mixed families, N = 64,
    2048 SSPRK3 steps (1024 cells at CFL 0.5) with a checkpoint every 32 steps, so the adjoint recomputes 64
    segments; the parameter gradient is compared element-wise with autograd through the whole unroll."""
    desc, vel, p, u0 = _long_case(prec)
    n, steps = LONG["n"], LONG["steps"]
    targets = np.stack([P.cell_averages(desc, n, vel * (k * 0.5 / n)) for k in range(1, steps + 1)], axis=1)
    lo, go, guo, fo = O.loss_and_grads(p, u0, targets, vel, 0.5 / n, float(n), prec)
    loss, grad, gu0, fin = T.loss_and_grads(p, _batch(desc, vel, n, steps, u0, every=LONG["every"]), prec,
                                            want_u0=True)
    assert abs(float(loss) - lo) <= (1e-10 if prec == "f64" else 1e-5) * lo
    assert _rel(fin.cpu().numpy(), fo) <= (1e-10 if prec == "f64" else 1e-5)
    assert _rel(grad.cpu().numpy(), go) <= GTOL[prec], _rel(grad.cpu().numpy(), go)
    assert _nrel(gu0.cpu().numpy(), guo) <= 5e-2


def test_directional_finite_differences_at_1024_cells_of_propagation():
    """Central differences of the FP64 loss over the full 2048-step unroll along random parameter directions."""
    desc, vel, p, u0 = _long_case("f64")
    n, steps = LONG["n"], LONG["steps"]
    _, grad, _, _ = T.loss_and_grads(p, _batch(desc, vel, n, steps, u0, every=LONG["every"]), "f64")
    grad = grad.cpu().numpy()
    rng = np.random.default_rng(37)

    def L(pp):
        return float(T.loss_and_grads(pp, _batch(desc, vel, n, steps, u0, every=LONG["every"]), "f64")[0])

    errs = []
    for _ in range(4):
        v = rng.standard_normal(p.size)
        h = 1e-6
        fd = (L(p + h * v) - L(p - h * v)) / (2 * h)
        errs.append(abs(fd - grad @ v) / max(abs(grad @ v), 1e-12))
    assert np.median(errs) <= 1e-4, errs


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_initial_state_gradient_matches_oracle_on_smooth_profiles(prec):
    """Without near-plateau stencils the state adjoint is well conditioned and agrees tightly."""
    rng = np.random.default_rng(8)
    n, B, steps = 64, 8, 20
    desc, _ = P.make_profiles(rng, B, n, family="smooth")
    vel = T.balanced_velocities(B)
    src = "weno5_sr_fp64_step012250.npz" if prec == "f64" else "weno5_sr_fp32_step016500.npz"
    p = np.concatenate([np.load(M / src)[k].reshape(-1).astype(np.float64) for k in T.PARAM_NAMES])
    u0 = P.cell_averages(desc, n, 0.0)
    targets = np.stack([P.cell_averages(desc, n, vel * (k * 0.5 / n)) for k in range(1, steps + 1)], axis=1)
    lo, go, guo, fo = O.loss_and_grads(p, u0, targets, vel, 0.5 / n, float(n), prec)
    loss, grad, gu0, fin = T.loss_and_grads(p, _batch(desc, vel, n, steps, u0, every=6), prec, want_u0=True)
    assert _rel(grad.cpu().numpy(), go) <= GTOL[prec]
    assert _nrel(gu0.cpu().numpy(), guo) <= (1e-9 if prec == "f64" else 1e-3)


def test_checkpoint_interval_does_not_change_gradients():
    rng = np.random.default_rng(9)
    n, B, steps = 40, 6, 21
    desc, _ = P.make_profiles(rng, B, n)
    vel = T.balanced_velocities(B)
    p = np.concatenate([np.load(M / "weno5_sr_fp64_step012250.npz")[k].reshape(-1) for k in T.PARAM_NAMES])
    ref = None
    for every in (1, 4, 7, 21, 32):
        loss, grad, gu0, _ = T.loss_and_grads(p, _batch(desc, vel, n, steps, every=every), "f64", want_u0=True)
        cur = (float(loss), grad.cpu().numpy(), gu0.cpu().numpy())
        if ref is None:
            ref = cur
        else:
            assert cur[0] == ref[0]
            assert np.array_equal(cur[1], ref[1]) and np.array_equal(cur[2], ref[2]), every


def test_directional_finite_differences_fp64():
    """Central differences of the CUDA loss along random parameter and state directions."""
    rng = np.random.default_rng(13)
    n, B, steps = 32, 4, 6
    desc, _ = P.make_profiles(rng, B, n, family="smooth")
    vel = T.balanced_velocities(B)
    p = np.concatenate([np.load(M / "weno5_sr_fp64_step012250.npz")[k].reshape(-1) for k in T.PARAM_NAMES])
    u0 = P.cell_averages(desc, n, 0.0)
    _, grad, gu0, _ = T.loss_and_grads(p, _batch(desc, vel, n, steps, u0), "f64", want_u0=True)
    grad, gu0 = grad.cpu().numpy(), gu0.cpu().numpy()

    def L(pp, uu):
        return float(T.loss_and_grads(pp, _batch(desc, vel, n, steps, uu), "f64")[0])

    errs = []
    for _ in range(4):
        v = rng.standard_normal(p.size)
        h = 1e-6
        fd = (L(p + h * v, u0) - L(p - h * v, u0)) / (2 * h)
        errs.append(abs(fd - grad @ v) / max(abs(grad @ v), 1e-12))
    assert np.median(errs) <= 1e-4, errs
    w = rng.standard_normal(u0.shape) * np.abs(u0).max()
    h = 1e-8
    fd = (L(p, u0 + h * w) - L(p, u0 - h * w)) / (2 * h)
    assert abs(fd - np.sum(gu0 * w)) <= 1e-3 * abs(np.sum(gu0 * w))


def test_full_size_batch_properties():
    """B = 1024, N = 256, distance 2 cells: the batch mean splits over sub-batches, gradients add, and a
    repeated call is bitwise identical."""
    rng = np.random.default_rng(17)
    n, B, steps = 256, 1024, 4
    desc, _ = P.make_profiles(rng, B, n)
    vel = T.balanced_velocities(B)
    p = T.ClosureMLP(seed=83, dtype=torch.float32)
    with torch.no_grad():
        for k in T.PARAM_NAMES:
            getattr(p, k).add_(0.1 * torch.randn(getattr(p, k).shape, dtype=torch.float32))
    packed = p.packed().detach().double().numpy()
    full = T.loss_and_grads(packed, _batch(desc, vel, n, steps), "f32")
    again = T.loss_and_grads(packed, _batch(desc, vel, n, steps), "f32")
    assert float(full[0]) == float(again[0]) and torch.equal(full[1], again[1])
    assert np.isfinite(full[1].cpu().numpy()).all()
    parts = [T.loss_and_grads(packed, _batch(desc[s:s + 256], vel[s:s + 256], n, steps), "f32") for s in range(0, B, 256)]
    lsum = sum(float(x[0]) for x in parts) / 4
    gsum = sum(x[1].cpu().numpy() for x in parts) / 4
    assert abs(lsum - float(full[0])) <= 1e-12 * float(full[0])
    assert _rel(gsum, full[1].cpu().numpy()) <= 1e-10


def test_autograd_function_fills_parameter_gradients():
    rng = np.random.default_rng(21)
    n, B = 32, 6
    desc, _ = P.make_profiles(rng, B, n)
    model = T.ClosureMLP.from_checkpoint(M / "weno5_sr_fp64_step012250.npz").to(DEV)
    b = _batch(desc, T.balanced_velocities(B), n, 5)
    loss = T.trajectory_loss(model, b)
    loss.backward()
    got = torch.cat([getattr(model, k).grad.reshape(-1) for k in T.PARAM_NAMES]).cpu().numpy()
    _, ref, _, _ = T.loss_and_grads(model.packed().detach().cpu().numpy(), b, "f64")
    assert np.array_equal(got, ref.cpu().numpy())


def test_invalid_arguments_raise():
    rng = np.random.default_rng(0)
    desc, _ = P.make_profiles(rng, 2, 16)
    p = np.zeros(189)
    with pytest.raises(ValueError):
        T.loss_and_grads(p, _batch(desc, [1.0, -1.0], 4, 2), "f64")  # n < 5
    with pytest.raises(ValueError):
        T.loss_and_grads(p, _batch(desc, [1.0, -1.0], 2048, 2), "f64")  # n > 1024


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_training_from_initialisation_beats_js(tmp_path, precision):
    """300 Adam steps from the reference's initialisation (FP32 or FP64 closure, N = 96, B = 256, distances 2,
    8, 64 cells) give a closure whose error under the reference's evaluation protocol (rk3_advection.py:533-560,
    distance 20 cells, N = 96, balanced velocities) is below WENO5-JS for every profile family."""
    cfg = T.TrainConfig(out_dir=tmp_path / "run", steps=300, grid=96, batch=256, distances=(2, 8, 64),
                        precision=precision, lr=1e-3, lr_final=2e-4, log_interval=50, checkpoint_interval=1000,
                        state_interval=1000, device=DEV)
    out = T.train(cfg)
    assert out["skipped"] == 0
    rng = np.random.default_rng(104729)
    ratios = []
    for fam in P.FAMILIES:
        desc, _ = P.make_profiles(rng, 8, 96, fam)
        vel = T.balanced_velocities(8)
        sr = T.final_state_error_signed(out["model"].closure(), desc, 96, 20.0, 0.5, vel, DEV)[0]
        js = T.final_state_error_signed("classical", desc, 96, 20.0, 0.5, vel, DEV)[0]
        ratios.append(sr / js)
    assert max(ratios) < 1.0, ratios
    assert float(np.mean(ratios)) < 0.7, ratios
    # the written checkpoint is a reference-format closure
    last = tmp_path / "run" / "checkpoints" / "model_step_000300.npz"
    m = T.ClosureMLP.from_checkpoint(last, torch.float32 if precision == "f32" else torch.float64)
    assert torch.equal(m.packed(), out["model"].packed().detach().cpu())


def test_resume_continues_bitwise(tmp_path):
    """20 steps, then 20 more resumed from the saved state, equal 40 uninterrupted steps."""
    kw = dict(steps=40, grid=64, batch=32, distances=(2, 8), precision="f64", lr=1e-3, lr_final=2e-4,
              log_interval=10, checkpoint_interval=1000, state_interval=20, device=DEV)
    a = T.train(T.TrainConfig(out_dir=tmp_path / "a", **kw))
    T.train(T.TrainConfig(out_dir=tmp_path / "b", **kw), max_steps=20)
    b = T.train(T.TrainConfig(out_dir=tmp_path / "b", **kw), resume=tmp_path / "b" / "state" / "latest.pt")
    assert b["completed"] == 40
    assert torch.equal(a["model"].packed(), b["model"].packed())
