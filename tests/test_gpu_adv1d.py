"""CUDA batched 1D advection against the reference fixtures, the published GSTE table and the oracle."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import adv1d_oracle as A
from oracle.oracle import pack_params
from weno_sr_publishing_b200 import adv1d as D
from weno_sr_publishing_b200 import weno_z as Z

pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden"
M = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
P64 = pack_params(dict(np.load(M / "weno5_sr_fp64_step012250.npz")))
P32 = pack_params(dict(np.load(M / "weno5_sr_fp32_step016500.npz")))
P7 = pack_params(dict(np.load(M / "weno7_sr_fp64_step016750.npz")))
MODEL5 = {"js": "classical", "sr_f64": D.Closure(5, P64, "f64"), "sr_f32": D.Closure(5, P32, "f32"),
          "sr_bf16": D.Closure(5, P32, "bf16")}
MODEL7 = {"js": "classical", "sr_f64": D.Closure(7, P7, "f64"), "sr_f32": D.Closure(7, P7, "f32"),
          "sr_bf16": D.Closure(7, P7, "bf16")}
ORACLE5 = {"js": None, "sr_f64": (5, "f64", P64), "sr_f32": (5, "f32", P32), "sr_bf16": (5, "bf16", P32)}
ORACLE7 = {"js": None, "sr_f64": (7, "f64", P7), "sr_f32": (7, "f32", P7), "sr_bf16": (7, "bf16", P7)}
# relative max-norm tolerances against the reference / the oracle (FP32 closures differ in exp/rcp rounding)
TOL = {"js": 1e-13, "sr_f64": 1e-12, "sr_f32": 2e-6, "sr_bf16": 2e-2}
DEV = "cuda:0"


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("case,n", [(0, 37), (1, 64), (2, 100)])
@pytest.mark.parametrize("key", ["js", "sr_f64", "sr_f32"])
def test_weno5_ssprk3_matches_reference_fixture(case, n, key):
    g = np.load(G / "adv1d_steps.npz")
    u0 = torch.as_tensor(g[f"c{case}_u0"], device=DEV)
    vel = torch.tensor([1.0, -1.0], dtype=torch.float64)
    dx = 1.0 / n
    u = u0
    for _ in range(3):
        u = D.ssprk3_step_signed(MODEL5[key], u, 0.5 * dx, 1.0 / dx, vel)
    assert _rel(u.cpu().numpy(), g[f"c{case}_w5_{key}_3steps"]) <= TOL[key]
    u = D.rollout_distance(MODEL5[key], u0, 2.3, 0.5, vel)
    assert _rel(u.cpu().numpy(), g[f"c{case}_w5_{key}_dist"]) <= TOL[key]


@pytest.mark.parametrize("case,n", [(0, 37), (1, 64), (2, 100)])
@pytest.mark.parametrize("key", ["js", "sr_f64"])
def test_weno7_shu_rk4_matches_reference_fixture(case, n, key):
    g = np.load(G / "adv1d_steps.npz")
    u0 = torch.as_tensor(g[f"c{case}_u0"], device=DEV)
    vel = torch.tensor([1.0, -1.0], dtype=torch.float64)
    u = D.rollout_signed(MODEL7[key], u0, 3, 0.5, vel)
    assert _rel(u.cpu().numpy(), g[f"c{case}_w7_{key}_3steps"]) <= TOL[key]


@pytest.mark.parametrize("method,model,stepper,l1,tol", [
    ("weno5_js", "js", "w5", 0.04976537479001931, 1e-10),
    ("weno5_sr_f64", "sr_f64", "w5", 0.03756399031896309, 1e-10),
    ("weno5_sr_f32", "sr_f32", "w5", 0.03645371035740613, 1e-6),
    ("weno7_js", "js", "w7", 0.029739185322686722, 1e-10),
    ("weno7_sr_f64", "sr_f64", "w7", 0.02341602561621716, 1e-10),
])
def test_gste_reproduces_published_l1(method, model, stepper, l1, tol):
    """GSTE, N=200 on [-1,1], CFL 0.6, t=10 (experiments/01_gste_long_time_advection)."""
    g = np.load(G / "gste.npz")
    if stepper == "w5":
        mdl = D.Closure(5, P32, "f32") if model == "sr_f32" else MODEL5[model]
        final, meta = D.integrate_ssprk3(mdl, D.ssprk3_step_signed, g["initial"], 0.6, 10.0, DEV)
    else:
        final, meta = D.integrate_ssprk3(MODEL7[model], D.shu_rk4_step_signed, g["initial"], 0.6, 10.0, DEV)
    assert meta["steps"] == 1667
    err = float(np.mean(np.abs(final - g["exact"])))
    assert abs(err - l1) <= tol * max(l1, 1.0), (err, l1)
    if model != "sr_f32":
        assert np.abs(final - g[f"{method}_final"]).max() <= 1e-9


def _ragged(seed, scheme):
    rng = np.random.default_rng(seed)
    B = 7
    states, vel, dx, nf, dtf, dtl = [], [], [], [], [], []
    for b in range(B):
        n = int(rng.integers(20, 91))
        x = (np.arange(n) + 0.5) / n
        u = 0.5 + 0.3 * np.sin(2 * np.pi * x * rng.integers(1, 4)) + np.where(x > rng.uniform(0.3, 0.7), 0.4, 0.0)
        states.append(u)
        vel.append(1.0 if b % 2 == 0 else -1.0)
        dx.append(1.0 / n)
        nf.append(int(rng.integers(1, 6)))
        dtf.append(0.5 / n)
        dtl.append(0.0 if b % 3 else 0.2 / n)
    return states, vel, dx, nf, dtf, dtl


@pytest.mark.parametrize("scheme,integ", [(5, "ssprk3"), (7, "shu_rk4")])
@pytest.mark.parametrize("key", ["js", "sr_f64", "sr_f32", "sr_bf16"])
def test_ragged_batch_matches_oracle(scheme, integ, key):
    states, vel, dx, nf, dtf, dtl = _ragged(3, scheme)
    model = (MODEL5 if scheme == 5 else MODEL7)[key]
    outs, info = D.run_batched(states, vel, dx, nf, dtf, dtl, scheme=scheme, model=model, integrator=integ, device=DEV)
    closure = (ORACLE5 if scheme == 5 else ORACLE7)[key]
    for b, u in enumerate(states):
        dts = [dtf[b]] * nf[b] + ([dtl[b]] if dtl[b] > 0 else [])
        ref = A.run(u, vel[b], dx[b], dts, scheme, closure, integ)
        assert _rel(outs[b].cpu().numpy(), ref) <= TOL[key], (b, key)


@pytest.mark.parametrize("scheme,integ,key", [(5, "ssprk3", "sr_f64"), (5, "ssprk3", "sr_f32"), (7, "shu_rk4", "sr_f64"),
                                              (5, "ssprk3", "js")])
def test_mass_conservation_and_reflection_symmetry_1000(scheme, integ, key):
    """Periodic mass is conserved and flip(step(+1, u)) == step(-1, flip(u)) (the reference's self-test)."""
    rng = np.random.default_rng(11)
    n, B = 1000, 16
    states = [np.where(rng.uniform(size=n) > 0.7, 1.0, 0.0) * rng.uniform() + np.sin(np.linspace(0, 6, n)) for _ in range(B)]
    model = (MODEL5 if scheme == 5 else MODEL7)[key]
    fw, _ = D.run_batched(states, [1.0] * B, 1.0 / n, 20, 0.4 / n, scheme=scheme, model=model, integrator=integ,
                          device=DEV)
    bw, _ = D.run_batched([s[::-1].copy() for s in states], [-1.0] * B, 1.0 / n, 20, 0.4 / n, scheme=scheme,
                          model=model, integrator=integ, device=DEV)
    for b in range(B):
        f = fw[b].cpu().numpy()
        assert abs(f.sum() - states[b].sum()) <= 1e-11 * np.abs(states[b]).sum()
        assert np.abs(f - bw[b].cpu().numpy()[::-1]).max() <= 1e-12


def test_invalid_batches_raise():
    with pytest.raises(ValueError):
        D.run_batched([np.zeros(3)], [1.0], 0.1, 1, 0.01, scheme=5, device=DEV)
    with pytest.raises(ValueError):
        D.run_batched([np.zeros(10)], [1.0], 0.1, 1, 0.01, scheme=7, model=MODEL5["sr_f64"], device=DEV)


@pytest.mark.parametrize("case,n", [(0, 37), (1, 64), (2, 100)])
@pytest.mark.parametrize("scheme,key", [(5, "w5"), (7, "w7")])
def test_weno_z_matches_reference_fixture(case, n, scheme, key):
    """weno_z.ssprk3_step / shu_rk4_step against torch_weno_z's own steppers (3 steps, velocity +1)."""
    g = np.load(G / "adv1d_z.npz")
    u = torch.as_tensor(g[f"c{case}_u0"], device=DEV)
    dx = 1.0 / n
    step = Z.ssprk3_step if scheme == 5 else Z.shu_rk4_step
    for _ in range(3):
        u = step(u, 0.5 * dx, 1.0 / dx)
    assert _rel(u.cpu().numpy(), g[f"c{case}_{key}_3steps"]) <= TOL["js"]


@pytest.mark.parametrize("key,l1", [("weno5_z", 4.198206e-2), ("weno7_z", 2.928891e-2)])
def test_gste_z_reproduces_published_l1(key, l1):
    """The WENO-Z GSTE rows (N=200, t=10, CFL 0.6; weno_z_borges_p2_results/README.md), all steps in one launch."""
    g = np.load(G / "adv1d_z.npz")
    final, steps, dt, _ = Z.integrate(g["initial"], 10.0, 0.6, Z.ssprk3_step if key == "weno5_z" else Z.shu_rk4_step,
                                      DEV)
    assert steps == int(g[f"{key}_steps"]) and dt == float(g[f"{key}_dt"])
    assert abs(float(np.mean(np.abs(final - g["exact"]))) - l1) <= 5e-9
    assert np.abs(final - g[f"{key}_final"]).max() <= 1e-9


@pytest.mark.parametrize("scheme,integ", [(5, "ssprk3"), (7, "shu_rk4")])
def test_weno_z_ragged_batch_matches_oracle(scheme, integ):
    """Ragged rows, both velocity signs and a shortened last step against the oracle's WENO-Z."""
    states, vel, dx, nf, dtf, dtl = _ragged(5, scheme)
    outs, _ = D.run_batched(states, vel, dx, nf, dtf, dtl, scheme=scheme, model="z", integrator=integ, device=DEV)
    for b, u in enumerate(states):
        dts = [dtf[b]] * nf[b] + ([dtl[b]] if dtl[b] > 0 else [])
        ref = A.run(u, vel[b], dx[b], dts, scheme, "z", integ)
        assert _rel(outs[b].cpu().numpy(), ref) <= TOL["js"], b


def test_host_batch_in_and_out_in_one_copy():
    """Host rows (numpy and CPU tensors) go up in one copy; to_host=True returns numpy views of one read-back, equal to
    the device results."""
    states, vel, dx, nf, dtf, dtl = _ragged(7, 5)
    dev_out, _ = D.run_batched(states, vel, dx, nf, dtf, dtl, scheme=5, model=MODEL5["sr_f32"], device=DEV)
    mixed = [torch.as_tensor(s) if b % 2 else s for b, s in enumerate(states)]
    host_out, _ = D.run_batched(mixed, vel, dx, nf, dtf, dtl, scheme=5, model=MODEL5["sr_f32"], device=DEV,
                                to_host=True)
    assert all(isinstance(h, np.ndarray) for h in host_out)
    for d, h in zip(dev_out, host_out):
        np.testing.assert_array_equal(d.cpu().numpy(), h)
