"""CPU: the exact Riemann solver and the shock-tube initial states against the reference's own code
(tests/golden/riemann_exact.npz, written by tests/golden/make_golden_riemann.py) and textbook values."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from weno_sr_publishing_b200 import riemann as R

G = Path(__file__).resolve().parent / "golden" / "riemann_exact.npz"
TUBE = {"sod": R.SOD, "lax": R.LAX}


@pytest.fixture(scope="module")
def gold():
    if not G.exists():
        pytest.skip("riemann_exact.npz not generated")
    return np.load(G)


def test_sod_star_state_textbook():
    # Toro, Riemann Solvers and Numerical Methods for Fluid Dynamics, Table 4.3 (test 1)
    p, u = R.star_state(R.SOD.left, R.SOD.right)
    assert abs(p - 0.30313) < 5e-6 and abs(u - 0.92745) < 5e-6


@pytest.mark.parametrize("name", ["sod", "lax"])
def test_star_state_and_waves_match_reference(gold, name):
    t = TUBE[name]
    np.testing.assert_allclose(R.star_state(t.left, t.right), gold[f"{name}_star"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(R.wave_speeds(t.left, t.right), gold[f"{name}_speeds"], rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("name", ["sod", "lax"])
def test_sampling_matches_reference(gold, name):
    t = TUBE[name]
    rho, vel, prs = R.sample(gold[f"{name}_xi"], t.left, t.right)
    np.testing.assert_allclose(np.stack([rho, vel, prs], axis=1), gold[f"{name}_sample"], rtol=1e-12, atol=1e-14)


def test_exact_cell_averages_match_reference(gold):
    dx = 0.01
    x = (np.arange(100) + 0.5) * dx
    sod = R.cell_averages(x, dx, 0.2, 0.5, R.SOD.left, R.SOD.right, split=False)
    np.testing.assert_allclose(sod, gold["sod_exact_t02"], rtol=1e-12, atol=1e-14)
    dx = 0.05
    x = -5.0 + (np.arange(200) + 0.5) * dx
    for q in (15, 20):
        lax = R.cell_averages(x, dx, 1.3, 0.0, R.LAX.left, R.LAX.right, quadrature=q)
        np.testing.assert_allclose(lax, gold[f"lax_exact_t13_q{q}"], rtol=1e-12, atol=1e-14)


def test_split_averages_conserve_mass_momentum_energy():
    """While every wave stays inside, the exact averages keep the totals of the initial step (minus the
    boundary fluxes, zero here), up to the quadrature of the rarefaction fan."""
    for t in (R.SOD, R.LAX):
        n = 400
        dx = (t.x_max - t.x_min) / n
        x = t.x_min + (np.arange(n) + 0.5) * dx
        a0 = R.cell_averages(x, dx, 0.0, t.x0, t.left, t.right).sum(axis=0) * dx
        a1 = R.cell_averages(x, dx, t.t_end, t.x0, t.left, t.right).sum(axis=0) * dx
        # boundary fluxes of the constant states at both ends over [0, t_end]
        for side, sgn in ((t.left, 1.0), (t.right, -1.0)):
            rho, u, p = side
            e = p / 0.4 + 0.5 * rho * u * u
            a0 = a0 + sgn * t.t_end * np.array([rho * u, rho * u * u + p, 0.0, u * (e + p)])
        np.testing.assert_allclose(a1, a0, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", ["sod", "lax"])
def test_tube_initial_states_match_reference(gold, name):
    got = R.tube_initial_state(TUBE[name])
    np.testing.assert_allclose(got, gold[f"{name}_initial"], rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("n", [1001, 2000])
def test_titarev_toro_initial_state_matches_reference(gold, n):
    np.testing.assert_allclose(R.titarev_toro_state(n), gold[f"tt_initial_{n}"], rtol=1e-15, atol=1e-15)


def test_vacuum_generating_data_raise():
    with pytest.raises(ValueError):
        R.star_state((1.0, -20.0, 1.0), (1.0, 20.0, 1.0))
