"""CUDA 3D Euler WENO5 step against the reference's own solver (fixtures), the C oracle and properties."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from weno_sr_publishing_b200 import euler3d as E3
from weno_sr_publishing_b200 import problems as PR

pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden"
M = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
DEV = "cuda:0"
P64 = {k: v for k, v in np.load(M / "weno5_sr_fp64_step012250.npz").items() if k != "meta_json"}
P32 = {k: v for k, v in np.load(M / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}
PARAMS = {"js": None, "sr_f64": P64, "sr_f32": P32, "z": None}
# relative max-norm tolerances against the reference / the oracle: the JS path is bitwise, the SR closures
# differ in exp/log/reciprocal rounding (and the FP32 closure forms its features in FP32); WENO-Z is built
# without contraction and with IEEE divisions like JS, so it is bitwise too
TOL = {"js": 0.0, "sr_f64": 1e-12, "sr_f32": 2e-6, "z": 0.0}
INNER = (slice(3, -3),) * 3


def _rel(a, b):
    a, b = np.asarray(a)[INNER], np.asarray(b)[INNER]
    return float(np.abs(a - b).max() / np.abs(b).max())


def _fixture(case):
    path = G / f"3d_{case}.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    return np.load(path)


@pytest.mark.parametrize("case,method", [("ic", "js"), ("js", "js"), ("sr_f64", "sr_f64"), ("sr_f32", "sr_f32"),
                                         ("z", "z")])
def test_matches_reference_solver(case, method):
    g = _fixture(case)
    nx, ny, nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
    dx, dy, dz, cfl = float(g["dx"]), float(g["dy"]), float(g["dz"]), float(g["cfl"])
    q = torch.as_tensor(g["q_init"], device=DEV).contiguous()
    E3.stage(q, nx, ny, nz, dx, dy, dz, float(g["stage1_dt"]), 1, method, mlp_params=PARAMS[method])
    assert _rel(q.cpu().numpy(), g["q_stage1"]) <= TOL[method]
    q = torch.as_tensor(g["q_init"], device=DEV).contiguous()
    t_end = 2.0e-5 if case == "ic" else 1.0
    res = E3.run(q, nx, ny, nz, dx, dy, dz, cfl, method, mlp_params=PARAMS[method], t_end=t_end,
                 steps=len(g["dts"]))
    assert res.steps == len(g["dts"])
    assert np.abs(res.dts - g["dts"]).max() <= TOL[method] * np.abs(g["dts"]).max()
    assert _rel(q.cpu().numpy(), g[f"q_step{len(g['dts'])}"]) <= TOL[method]


def _random_state(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx,
                          indexing="ij")
    front = x + 0.3 * y - 0.4 * z + 0.1 * rng.uniform() > 0.6
    rho = np.where(front, 0.7, 1.2) + 0.1 * np.sin(2 * np.pi * (y + z))
    u = np.where(front, 0.1, 0.3)
    v = 0.2 * np.cos(2 * np.pi * x)
    w = 0.1 * np.sin(2 * np.pi * y)
    p = np.where(front, 0.8, 1.2) + 0.05 * np.cos(2 * np.pi * z)
    inner = np.stack([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)], axis=-1)
    return np.pad(inner, ((3, 3), (3, 3), (3, 3), (0, 0)), mode="edge")


@pytest.mark.parametrize("flux", ["evilin", "hllc"])
@pytest.mark.parametrize("method", ["js", "sr_f64", "sr_f32", "z"])
def test_matches_oracle_ragged_grid(method, flux):
    nx, ny, nz = 19, 11, 9
    h = (1.0 / nx, 1.0 / ny, 0.8 / nz)
    q0 = _random_state(nx, ny, nz, 3)
    ref, dts = O.euler3d_run(q0, nx, ny, nz, *h, 0.3, 3, method, flux, PARAMS[method])
    q = torch.as_tensor(q0, device=DEV).contiguous()
    res = E3.run(q, nx, ny, nz, *h, 0.3, method, flux, PARAMS[method], steps=3)
    assert np.abs(res.dts - dts).max() <= TOL[method] * dts.max()
    assert _rel(q.cpu().numpy(), ref) <= TOL[method]


def test_inflow_boundary_matches_oracle():
    sb = PR.ShockBubble.seeded(1, 24, 10, 10)
    q0 = sb.state()
    dx, dy, dz = sb.spacing
    ref, dts = O.euler3d_run(q0, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, 4, "js", "hllc", None, inflow=sb.inflow())
    q = torch.as_tensor(q0, device=DEV).contiguous()
    res = E3.run(q, sb.nx, sb.ny, sb.nz, dx, dy, dz, 0.4, "js", "hllc", inflow=sb.inflow(), steps=4)
    assert np.array_equal(res.dts, dts)
    assert np.array_equal(q.cpu().numpy()[INNER], ref[INNER])


def test_uniform_flow_is_preserved():
    nx, ny, nz = 12, 10, 8
    inner = np.broadcast_to(np.array([1.3, 1.3 * 0.4, -1.3 * 0.2, 1.3 * 0.1, 2.0 / 0.4 + 0.5 * 1.3 * 0.21]),
                            (nz, ny, nx, 5))
    q0 = np.pad(inner, ((3, 3), (3, 3), (3, 3), (0, 0)), mode="edge")
    for method in ("js", "sr_f64"):
        q = torch.as_tensor(q0, device=DEV).contiguous()
        E3.run(q, nx, ny, nz, 0.1, 0.1, 0.1, 0.4, method, "hllc", PARAMS[method], steps=3)
        assert np.abs(q.cpu().numpy()[INNER] - q0[INNER]).max() <= 1e-13 * np.abs(q0).max()


def test_planar_data_stays_planar():
    """Data that vary along x only stay uniform on every y-z plane, bit for bit (every cell of a plane sees
    the same inputs), for the SR closure and both fluxes."""
    nx, ny, nz = 16, 7, 6
    x = (np.arange(nx) + 0.5) / nx
    rho = 1.0 + 0.4 * np.tanh((x - 0.5) * 20)
    u, p = 0.3 + 0 * x, 1.0 + 0.2 * np.sin(2 * np.pi * x)
    line = np.stack([rho, rho * u, 0 * x, 0 * x, p / 0.4 + 0.5 * rho * u * u], axis=-1)
    q0 = np.pad(np.broadcast_to(line, (nz, ny, nx, 5)), ((3, 3), (3, 3), (3, 3), (0, 0)), mode="edge")
    for flux in ("evilin", "hllc"):
        q = torch.as_tensor(np.ascontiguousarray(q0), device=DEV)
        E3.run(q, nx, ny, nz, 1.0 / nx, 0.1, 0.1, 0.4, "sr_f64", flux, P64, steps=3)
        out = q.cpu().numpy()[INNER]
        assert np.array_equal(out, np.broadcast_to(out[:1, :1], out.shape))
        assert np.abs(out[..., 2:4]).max() == 0.0


def test_max_speed_and_t_end_clipping():
    nx, ny, nz = 8, 7, 6
    q0 = _random_state(nx, ny, nz, 5)
    q = torch.as_tensor(q0, device=DEV).contiguous()
    assert E3.max_speed(q, nx, ny, nz) == O.euler3d_max_speed(q0, nx, ny, nz)
    ref, dts = O.euler3d_run(q0, nx, ny, nz, 0.1, 0.1, 0.1, 0.4, 50, "js", "evilin", t_end=0.05)
    res = E3.run(q, nx, ny, nz, 0.1, 0.1, 0.1, 0.4, "js", t_end=0.05)
    assert res.steps == len(dts) and res.t == 0.05
    assert np.array_equal(res.dts, dts)
    assert np.array_equal(q.cpu().numpy()[INNER], ref[INNER])


def test_invalid_arguments_raise():
    q = torch.zeros((10, 10, 10, 5), dtype=torch.float64, device=DEV)
    with pytest.raises(ValueError):
        E3.run(q, 4, 4, 4, 0.1, 0.1, 0.1, 0.4, "js", steps=1)  # fewer than 5 cells
    q = torch.zeros((11, 11, 11, 5), dtype=torch.float64, device=DEV)
    with pytest.raises(ValueError):
        E3.run(q, 5, 5, 5, 0.1, 0.1, 0.1, 0.4, "sr_f64", steps=1)  # SR without parameters


def test_step_file_of_device_state(tmp_path):
    """The device state written as a step file (uint32 nz ny nx, f64 time, f64 primitive) reads back as the
    primitive interior of the oracle's state."""
    from weno_sr_publishing_b200 import binary_io as B  # noqa: PLC0415
    nx, ny, nz = 12, 9, 7
    q0 = _random_state(nx, ny, nz, 11)
    ref, dts = O.euler3d_run(q0, nx, ny, nz, 0.1, 0.1, 0.1, 0.4, 2, "js", "hllc")
    q = torch.as_tensor(q0, device=DEV).contiguous()
    res = E3.run(q, nx, ny, nz, 0.1, 0.1, 0.1, 0.4, "js", "hllc", steps=2)
    B.write_state(tmp_path / "step.bin", res.t, q, nx, ny, nz)
    t, prim = B.read_step(tmp_path / "step.bin")
    assert t == res.t and prim.shape == (nz, ny, nx, 5)
    np.testing.assert_array_equal(prim, B.primitive_interior(ref, nx, ny, nz))


def test_js_fallback_when_closure_is_not_finite():
    """WSR_OPT_JS_FALLBACK in 3D: with NaN output biases every non-plateau stencil takes WENO5-JS weights, so a
    step equals the WENO5-JS step up to the rounding of the two JS evaluations (reciprocals vs IEEE divisions);
    the fallbacks are counted. Without the option the NaN reaches the state."""
    nx, ny, nz = 12, 10, 8
    q0 = _random_state(nx, ny, nz, 4)
    dx = dy = dz = 1.0 / nx
    bad = {k: np.array(v, copy=True) for k, v in P64.items()}
    bad["b4"][:] = np.nan
    q_js = torch.as_tensor(q0, device=DEV).contiguous()
    E3.run(q_js, nx, ny, nz, dx, dy, dz, 0.4, "js", "hllc", steps=2)
    q_fb = torch.as_tensor(q0, device=DEV).contiguous()
    ws = E3.workspace(nx, ny, nz, DEV)
    E3.run(q_fb, nx, ny, nz, dx, dy, dz, 0.4, "sr_f64", "hllc", bad, steps=2, opts=2, ws=ws)  # OPT_JS_FALLBACK
    assert E3.counters(ws)["fallbacks"] > 0
    assert _rel(q_fb.cpu().numpy(), q_js.cpu().numpy()) <= 1e-12
    q_nan = torch.as_tensor(q0, device=DEV).contiguous()
    E3.run(q_nan, nx, ny, nz, dx, dy, dz, 0.4, "sr_f64", "hllc", bad, steps=1)
    assert not bool(torch.isfinite(q_nan[INNER]).all())


def test_weno_z_shock_bubble_completes_in_the_published_step_count():
    """The paper's 3D WENO5-Z row: Ma = 3 shock-bubble, 224 x 88 x 88, CFL 0.25, t = 1e-4, EVILIN, complete in
    840 steps (weno_z_borges_p2_results/README.md, run_shockbubble_3d.py)."""
    nx, ny, nz = 224, 88, 88
    dx, dy, dz = 0.225 / nx, 0.089 / ny, 0.089 / nz
    q = torch.as_tensor(PR.shockbubble_reference_state(nx, ny, nz), device=DEV).contiguous()
    res = E3.run(q, nx, ny, nz, dx, dy, dz, 0.25, "z", "evilin", t_end=1.0e-4)
    assert res.steps == 840
    assert abs(res.t - 1.0e-4) <= 1e-18
    inner = q[3:-3, 3:-3, 3:-3].cpu().numpy()
    assert np.isfinite(inner).all()
    rho = inner[..., 0]
    p = 0.4 * (inner[..., 4] - 0.5 * (inner[..., 1] ** 2 + inner[..., 2] ** 2 + inner[..., 3] ** 2) / rho)
    assert rho.min() > 0.0 and p.min() > 0.0
