"""CPU checks of the training oracle, the profile families and the host-side training logic."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch
from scipy.integrate import quad

from oracle import train1d_oracle as O
from weno_sr_publishing_b200 import profiles as P
from weno_sr_publishing_b200 import train1d as T

G = Path(__file__).resolve().parent / "golden"
CASES = ("trained_f64", "trained_f32", "perturbed_f64", "init_f64", "init_f32")


def _fixture(case):
    g = np.load(G / "train1d_grads.npz")
    return {k[len(case) + 1:]: g[k] for k in g.files if k.startswith(case + "_")}


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_reference_autograd(case):
    f = _fixture(case)
    prec = "f32" if case.endswith("f32") else "f64"
    loss, grad, gu0, final = O.loss_and_grads(f["params"], f["u0"], f["targets"], f["vel"], float(f["dt"]),
                                              float(f["n"]), prec)
    assert loss == float(f["loss"])
    assert np.array_equal(final, f["final"])
    assert np.abs(grad - f["grad"]).max() <= 1e-12 * np.abs(f["grad"]).max()
    # the initial-state gradient goes through the gamma feature at near-flat stencils, where it amplifies
    # rounding differences of the MLP adjoint: compared in norm
    assert np.linalg.norm(gu0 - f["grad_u0"]) <= 1e-3 * np.linalg.norm(f["grad_u0"])


def test_fixture_targets_are_the_closed_form_averages():
    f = _fixture("trained_f64")
    n, dt = int(f["n"]), float(f["dt"])
    for k in range(int(f["steps"])):
        e = P.cell_averages(f["desc"], n, f["vel"] * ((k + 1) * dt))
        assert np.array_equal(e, f["targets"][:, k])


@pytest.mark.parametrize("precision,dtype", [("f64", torch.float64), ("f32", torch.float32)])
def test_initialisation_matches_the_reference_draw(precision, dtype):
    f = _fixture(f"init_{precision}")
    m = T.ClosureMLP(seed=83, dtype=dtype)
    assert np.array_equal(m.packed().detach().double().numpy(), f["params"])
    assert float(m.w4.abs().sum()) == 0.0 and float(m.b4.abs().sum()) == 0.0


@pytest.mark.parametrize("family", P.FAMILIES)
def test_closed_form_averages_match_quadrature(family):
    rng = np.random.default_rng(3)
    n = 48
    desc, fam = P.make_profiles(rng, 3, n, family)
    assert (fam == P.FAMILIES.index(family)).all()
    for b in range(3):
        for shift in (0.0, 0.31, -1.7):
            avg = P.cell_averages(desc[b:b + 1], n, shift)[0]
            for i in (0, 7, 20, 33, 47):
                pts = np.linspace(i / n, (i + 1) / n, 9)[1:-1]
                v = quad(lambda x: P.point_values(desc[b:b + 1], np.array([x]), shift)[0, 0], i / n, (i + 1) / n,
                         limit=400, points=pts, epsabs=1e-13, epsrel=1e-12)[0] * n
                # boxes are discontinuous: quadrature resolves their edges to about 1e-6
                tol = 1e-5 if family in ("square", "multi", "composite") else 1e-9
                assert abs(v - avg[i]) <= tol * max(1.0, abs(avg[i])), (family, b, shift, i, v, avg[i])


def test_averages_are_periodic_and_conservative():
    rng = np.random.default_rng(4)
    desc, _ = P.make_profiles(rng, 20, 64)
    a0 = P.cell_averages(desc, 64, 0.0)
    assert np.abs(P.cell_averages(desc, 64, 3.0) - a0).max() <= 1e-12 * np.abs(a0).max()
    # translation by whole cells is a roll
    assert np.abs(P.cell_averages(desc, 64, 5.0 / 64) - np.roll(a0, 5, axis=1)).max() <= 1e-11 * np.abs(a0).max()
    # the mean over a period does not depend on the shift
    assert np.abs(P.cell_averages(desc, 64, 0.123).mean(1) - a0.mean(1)).max() <= 1e-12 * np.abs(a0).max()


def test_schedule_helpers():
    assert T.steps_for_distance(1024, 0.5) == 2048
    with pytest.raises(ValueError):
        T.steps_for_distance(3, 0.7)
    idx = [T.distance_index_for_step(s, 7, 83) for s in range(1, 15)]
    assert sorted(idx[:7]) == list(range(7)) and sorted(idx[7:]) == list(range(7))
    v = T.balanced_velocities(6)
    assert list(v) == [1, 1, 1, -1, -1, -1]
    sched = T.make_scheduler(torch.optim.SGD([torch.zeros(1, requires_grad=True)], lr=1.0), 1e-4, 2e-5, 100)
    assert sched.lr_lambdas[0](0) == pytest.approx(1.0) and sched.lr_lambdas[0](100) == pytest.approx(0.2)
