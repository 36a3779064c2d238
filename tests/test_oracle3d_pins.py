"""CPU: the 3D oracle against the reference's own Warp solver (fixtures), and flux properties."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from weno_sr_publishing_b200 import problems as PR

G = Path(__file__).resolve().parent / "golden"
M = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
P64 = {k: v for k, v in np.load(M / "weno5_sr_fp64_step012250.npz").items() if k != "meta_json"}
P32 = {k: v for k, v in np.load(M / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}
INNER = (slice(3, -3),) * 3


def _fixture(case):
    path = G / f"3d_{case}.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    return np.load(path)


@pytest.mark.parametrize("case,method,params,tol", [("ic", "js", None, 0.0), ("js", "js", None, 0.0),
                                                    ("sr_f64", "sr_f64", P64, 1e-14), ("sr_f32", "sr_f32", P32, 1e-8),
                                                    ("z", "z", None, 0.0)])
def test_oracle_reproduces_reference_solver(case, method, params, tol):
    g = _fixture(case)
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    h = (float(g["dx"]), float(g["dy"]), float(g["dz"]))
    t_end = 2.0e-5 if case == "ic" else 1.0
    out, dts = O.euler3d_run(g["q_init"], nx, ny, nz, *h, float(g["cfl"]), 1, method, params=params, t_end=t_end,
                             stage_only=True)
    assert dts[0] == float(g["stage1_dt"])
    ref = g["q_stage1"][INNER]
    assert np.abs(out[INNER] - ref).max() <= tol * np.abs(ref).max()
    steps = len(g["dts"])
    out, dts = O.euler3d_run(g["q_init"], nx, ny, nz, *h, float(g["cfl"]), steps, method, params=params, t_end=t_end)
    assert np.abs(dts - g["dts"]).max() <= tol * np.abs(g["dts"]).max()
    ref = g[f"q_step{steps}"][INNER]
    assert np.abs(out[INNER] - ref).max() <= tol * np.abs(ref).max()


def test_reference_initial_state_is_reproduced():
    g = _fixture("ic")
    assert np.array_equal(PR.shockbubble_reference_state(6, 5, 5), g["q_init"])


def _states(n, seed):
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.2, 3.0, n)
    vel = rng.uniform(-2.0, 2.0, (n, 3))
    p = rng.uniform(0.1, 5.0, n)
    E = p / 0.4 + 0.5 * rho * np.sum(vel * vel, axis=1)
    return np.column_stack([rho, rho * vel[:, 0], rho * vel[:, 1], rho * vel[:, 2], E])


def _physical(u, d):
    rho = u[:, 0]
    vel = u[:, 1:4] / rho[:, None]
    p = 0.4 * (u[:, 4] - 0.5 * rho * np.sum(vel * vel, axis=1))
    un = vel[:, d - 1]
    f = u * un[:, None]
    f[:, d] += p
    f[:, 4] += p * un
    return f


@pytest.mark.parametrize("d", [1, 2, 3])
def test_hllc3d_consistency_and_mirror_symmetry(d):
    u = _states(200, d)
    assert np.allclose(O.hllc5(u, u, d), _physical(u, d), rtol=1e-13, atol=1e-13)
    ul, ur = _states(200, 10 + d), _states(200, 20 + d)
    f = O.hllc5(ul, ur, d)
    # mirror x_d -> -x_d: swap the states, flip the normal momentum; the flux flips except its normal component
    flip = np.ones(5)
    flip[d] = -1.0
    g = O.hllc5(ur * flip, ul * flip, d)
    assert np.allclose(g, -f * flip, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("d", [1, 2, 3])
def test_hllc3d_reduces_to_the_2d_flux(d):
    """With zero velocity along the third axis the 3D HLLC equals the 2D HLLC of the oracle."""
    if d == 3:
        pytest.skip("the 2D flux has no z direction")
    u = _states(100, 40 + d)
    ul, ur = u.copy(), _states(100, 50 + d)
    for a in (ul, ur):
        a[:, 4] -= 0.5 * a[:, 3] ** 2 / a[:, 0]
        a[:, 3] = 0.0
    f3 = O.hllc5(ul, ur, d)
    f2 = np.stack([O.hllc(a[[0, 1, 2, 4]], b[[0, 1, 2, 4]], d) for a, b in zip(ul, ur)])
    assert np.allclose(f3[:, [0, 1, 2, 4]], f2, rtol=1e-13, atol=1e-13)
    assert np.abs(f3[:, 3]).max() == 0.0


def test_evilin_consistency():
    u = _states(100, 7)
    for d in (1, 2, 3):
        assert np.allclose(O.evilin5(u, u, d, 0.3), _physical(u, d), rtol=1e-12, atol=1e-12)
