"""Parity of the CUDA 2D path (through the C ABI) with the CPU oracle and the reference fixtures."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from weno_sr_publishing_b200 import euler2d as E
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200.params import Params
from weno_sr_publishing_b200.solvers import weno5_hllc, weno5_hllc_mixed, weno5_hllc_refsym, weno5_hllc_z_min

pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden"
MODELS = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")
P64 = {k: v for k, v in np.load(MODELS / "weno5_sr_fp64_step012250.npz").items() if k in NAMES}
P32 = {k: v for k, v in np.load(MODELS / "weno5_sr_fp32_step016500.npz").items() if k in NAMES}
PARAMS = {"js": None, "z": None, "sr_f64": P64, "sr_f32": P32, "sr_bf16": P32}
# Relative max-norm tolerances of one stage against the oracle (FMA contraction and CUDA's libm account
# for the FP64 differences; the FP32/BF16 closures differ in expf/tanhf rounding).
STAGE_TOL = {"js": 1e-13, "z": 1e-12, "sr_f64": 1e-12, "sr_f32": 2e-6, "sr_bf16": 5e-3}
CASES = ["rough_trans", "quadrant_trans", "smooth_periodic"]
DEV = "cuda:0"


def _interior(a, nx, ny):
    return a[3:3 + ny, 3:3 + nx]


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _t(a):
    return torch.as_tensor(np.ascontiguousarray(a), device=DEV)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("method", ["js", "z", "sr_f64", "sr_f32", "sr_bf16"])
@pytest.mark.parametrize("rk", [1, 2, 3])
def test_stage_matches_oracle(case, method, rk):
    e = np.load(G / f"euler2d_{case}.npz")
    nx, ny, bc = int(e["nx"]), int(e["ny"]), str(e["bc"])
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    u0 = e["initial"]
    rng = np.random.default_rng(rk)
    u_stage = u0 * (1.0 + 0.01 * rng.uniform(-1, 1, u0.shape)) if rk > 1 else u0
    dt = 0.3 * min(p.dx, p.dy) / O.max_speed(u0, nx, ny)
    ref = O.euler2d_stage(u_stage, u0, np.zeros_like(u0), nx, ny, p.dx, p.dy, dt, rk, method, bc,
                          params=PARAMS[method])
    out = torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV)
    E.stage(_t(u_stage), _t(u0), out, p, dt, rk, method, bc, mlp_params=PARAMS[method])
    got = out.cpu().numpy()
    assert np.all(got[:3] == 0) and np.all(got[:, :3] == 0), "ghost cells must not be written"
    err = _rel(_interior(got, nx, ny), _interior(ref, nx, ny))
    assert err <= STAGE_TOL[method], err


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("method,adapter,tol", [("js", weno5_hllc, 1e-12), ("sr_f64", weno5_hllc_refsym, 1e-12),
                                                ("sr_f32", weno5_hllc_mixed, 2e-6)])
def test_run_to_time_matches_reference_fixture(case, method, adapter, tol):
    e = np.load(G / f"euler2d_{case}.npz")
    nx, ny, bc = int(e["nx"]), int(e["ny"]), str(e["bc"])
    t_end = float(e["t_end"])
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4, t_end=t_end)
    mlp = None if method == "js" else {k: torch.as_tensor(v, device=DEV) for k, v in PARAMS[method].items()}
    final, dts, steps, t = adapter.run_to_time(e["initial"], p, t_end, DEV, mlp, bc, report_interval=0)
    assert steps == int(e[f"{method}_steps"])
    assert abs(t - float(e[f"{method}_t"])) <= 1e-14
    np.testing.assert_allclose(dts, e[f"{method}_dts"], rtol=1e-12 if method != "sr_f32" else 1e-6, atol=0)
    ref = e[f"{method}_final"]
    assert _rel(_interior(final, nx, ny), _interior(ref, nx, ny)) <= tol
    # ghost cells follow the reference's buffer swaps (initial ghosts or zeros by step parity)
    ghost = final.copy()
    ghost[3:3 + ny, 3:3 + nx] = 0.0
    ref_ghost = ref.copy()
    ref_ghost[3:3 + ny, 3:3 + nx] = 0.0
    np.testing.assert_array_equal(ghost, ref_ghost)


@pytest.mark.parametrize("case", ["rough_trans", "smooth_periodic"])
def test_z_run_to_time_matches_reference_fixture(case):
    """WENO5-Z through the weno5_hllc_z_min adapter against the reference's minimal Z solver (dx != dy)."""
    path = G / "euler2d_z.npz"
    if not path.exists():
        pytest.skip("euler2d_z.npz not generated")
    z = np.load(path)
    nx, ny, bc, t_end = int(z[f"{case}_nx"]), int(z[f"{case}_ny"]), str(z[f"{case}_bc"]), float(z[f"{case}_t_end"])
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4, t_end=t_end)
    final, dts, steps, t = weno5_hllc_z_min.run_to_time(z[f"{case}_initial"], p, t_end, DEV, bc)
    assert steps == int(z[f"{case}_steps"]) and abs(t - float(z[f"{case}_t"])) <= 1e-14
    np.testing.assert_allclose(dts, z[f"{case}_dts"], rtol=1e-12, atol=0)
    assert _rel(_interior(final, nx, ny), _interior(z[f"{case}_final"], nx, ny)) <= 1e-12
    arrays = weno5_hllc_z_min.allocate_forward(z[f"{case}_initial"], p, DEV)
    weno5_hllc_z_min.launch_stage(arrays["u0"], arrays["u0"], arrays["u1"], arrays["s1"], p, dts[0], 1, DEV, bc)
    got = arrays["u1"].cpu().numpy()
    assert _rel(_interior(got, nx, ny), _interior(z[f"{case}_stage1"], nx, ny)) <= 1e-12


@pytest.mark.parametrize("method,tol", [("js", 1e-11), ("z", 1e-11), ("sr_f64", 1e-11), ("sr_f32", 1e-5)])
def test_quadrant_64x48_ten_steps_vs_oracle(method, tol):
    nx, ny = 64, 48
    init = problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(3), 4)
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4, t_end=1.0)
    ref, rdts, rsteps, _ = O.euler2d_run(init, nx, ny, p.dx, p.dy, 0.4, 1.0, method, "transmissive",
                                         params=PARAMS[method], fixed_steps=10)
    bufs = [_t(init)] + [torch.zeros_like(_t(init)) for _ in range(3)]
    res = E.run(bufs, p, 1.0, method, "transmissive", mlp_params=PARAMS[method], fixed_steps=10)
    assert res.steps == rsteps == 10
    got = bufs[res.final_slot].cpu().numpy()
    assert _rel(_interior(got, nx, ny), _interior(ref, nx, ny)) <= tol
    np.testing.assert_allclose(res.dts, rdts, rtol=100 * tol)


@pytest.mark.parametrize("method", ["js", "z", "sr_f32"])
def test_uniform_flow_is_preserved(method):
    nx, ny = 40, 33
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    u = np.zeros(p.padded_shape)
    u[...] = problems.conserved_from_primitive(np.float64(1.3), 0.7, -0.4, 0.9)
    bufs = [_t(u)] + [torch.zeros_like(_t(u)) for _ in range(3)]
    res = E.run(bufs, p, 1.0, method, "periodic", mlp_params=PARAMS[method], fixed_steps=5)
    got = _interior(bufs[res.final_slot].cpu().numpy(), nx, ny)
    assert _rel(got, _interior(u, nx, ny)) <= 1e-14


@pytest.mark.parametrize("method", ["js", "z", "sr_f64", "sr_f32"])
def test_periodic_mass_conservation_256(method):
    nx = ny = 256
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    init = problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(1), 2)
    init[:3], init[-3:], init[:, :3], init[:, -3:] = 0, 0, 0, 0
    bufs = [_t(init)] + [torch.zeros_like(_t(init)) for _ in range(3)]
    res = E.run(bufs, p, 1.0, method, "periodic", mlp_params=PARAMS[method], fixed_steps=8)
    got = _interior(bufs[res.final_slot].cpu().numpy(), nx, ny)
    m0 = _interior(init, nx, ny).sum(axis=(0, 1))
    m1 = got.sum(axis=(0, 1))
    assert np.all(np.abs(m1 - m0) <= 1e-11 * np.abs(m0).max())


@pytest.mark.parametrize("method", ["js", "z", "sr_f64"])
def test_xy_transpose_symmetry(method):
    nx = ny = 36
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    init = problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(5), 3)
    tr = np.ascontiguousarray(init.transpose(1, 0, 2)[..., [0, 2, 1, 3]])
    outs = []
    for u in (init, tr):
        bufs = [_t(u)] + [torch.zeros_like(_t(u)) for _ in range(3)]
        res = E.run(bufs, p, 1.0, method, "transmissive", mlp_params=PARAMS[method], fixed_steps=4)
        outs.append(bufs[res.final_slot].cpu().numpy())
    back = outs[1].transpose(1, 0, 2)[..., [0, 2, 1, 3]]
    assert _rel(_interior(back, nx, ny), _interior(outs[0], nx, ny)) <= 1e-12


def test_max_speed_matches_oracle():
    nx, ny = 301, 157
    init = problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(9), 2)
    p = Params(nx=nx, ny=ny)
    assert E.max_speed(_t(init), p) == O.max_speed(init, nx, ny)


def test_js_fallback_when_closure_is_not_finite():
    nx, ny = 24, 20
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    init = problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(2), 3)
    bad = {k: np.array(v, copy=True) for k, v in P64.items()}
    bad["b4"][:] = np.nan  # every non-plateau closure evaluation becomes NaN
    outs = {}
    for name, method, params, opts in (("js", "js", None, 0), ("fb", "sr_f64", bad, E.N.OPT_JS_FALLBACK)):
        bufs = [_t(init)] + [torch.zeros_like(_t(init)) for _ in range(3)]
        res = E.run(bufs, p, 1.0, method, "transmissive", mlp_params=params, opts=opts, fixed_steps=2)
        outs[name] = (bufs[res.final_slot].cpu().numpy(), res.fallbacks)
    assert outs["fb"][1] > 0
    assert _rel(_interior(outs["fb"][0], nx, ny), _interior(outs["js"][0], nx, ny)) <= 1e-13
    # without the option the NaN propagates, as in the reference, and the health check stops the run
    bufs = [_t(init)] + [torch.zeros_like(_t(init)) for _ in range(3)]
    res = E.run(bufs, p, 1.0, "sr_f64", "transmissive", mlp_params=bad, check_health=True)
    assert res.steps == 1


def test_invalid_arguments_raise():
    p = Params(nx=2, ny=8)
    u = torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV)
    with pytest.raises(ValueError):
        E.stage(u, u, u, p, 1e-3, 1, "js", "transmissive")
    p = Params(nx=8, ny=8)
    u = torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV)
    with pytest.raises(ValueError):
        E.stage(u, u, u, p, 1e-3, 4, "js", "transmissive")
    with pytest.raises(ValueError):
        E.stage(u, u, u, p, 1e-3, 1, "js", "reflective")
    with pytest.raises(ValueError):
        E.stage(u, u, u, p, 1e-3, 1, "sr_f64", "transmissive", mlp_params=None)


# FORCE flux (warp_weno5_helpers.py:401-435): the oracle's FORCE is bit-identical to the reference's; the CUDA
# path's FORCE stage and runs are held to the HLLC stage tolerances.
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("method", ["js", "sr_f64", "sr_f32"])
@pytest.mark.parametrize("rk", [1, 2, 3])
def test_force_stage_matches_oracle(case, method, rk):
    e = np.load(G / f"euler2d_{case}.npz")
    nx, ny, bc = int(e["nx"]), int(e["ny"]), str(e["bc"])
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    u0 = e["initial"]
    rng = np.random.default_rng(10 + rk)
    u_stage = u0 * (1.0 + 0.01 * rng.uniform(-1, 1, u0.shape)) if rk > 1 else u0
    dt = 0.3 * min(p.dx, p.dy) / O.max_speed(u0, nx, ny)
    ref = O.euler2d_stage(u_stage, u0, np.zeros_like(u0), nx, ny, p.dx, p.dy, dt, rk, method, bc, flux="force",
                          params=PARAMS[method])
    out = torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV)
    E.stage(_t(u_stage), _t(u0), out, p, dt, rk, method, bc, mlp_params=PARAMS[method], flux="force")
    err = _rel(_interior(out.cpu().numpy(), nx, ny), _interior(ref, nx, ny))
    assert err <= STAGE_TOL[method], err


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("method,tol", [("js", 1e-11), ("sr_f64", 1e-11), ("sr_f32", 1e-5)])
def test_force_ten_step_run_matches_oracle(case, method, tol):
    e = np.load(G / f"euler2d_{case}.npz")
    nx, ny, bc = int(e["nx"]), int(e["ny"]), str(e["bc"])
    init = e["initial"]
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4, t_end=1.0)
    ref, rdts, rsteps, _ = O.euler2d_run(init, nx, ny, p.dx, p.dy, 0.4, 1.0, method, bc, flux="force",
                                         params=PARAMS[method], fixed_steps=10)
    bufs = [_t(init)] + [torch.zeros_like(_t(init)) for _ in range(3)]
    res = E.run(bufs, p, 1.0, method, bc, mlp_params=PARAMS[method], flux="force", fixed_steps=10)
    assert res.steps == rsteps == 10
    got = bufs[res.final_slot].cpu().numpy()
    assert _rel(_interior(got, nx, ny), _interior(ref, nx, ny)) <= tol
    np.testing.assert_allclose(res.dts, rdts, rtol=100 * tol)
    # FORCE is a different scheme: the run must not coincide with the HLLC run
    bufs2 = [_t(init)] + [torch.zeros_like(_t(init)) for _ in range(3)]
    res2 = E.run(bufs2, p, 1.0, method, bc, mlp_params=PARAMS[method], fixed_steps=10)
    assert _rel(_interior(bufs2[res2.final_slot].cpu().numpy(), nx, ny), _interior(got, nx, ny)) > 1e-8


# The BF16 closure with its MLP on the tensor cores (sr_bf16_tc) against the same closure on the FMA pipes (sr_bf16)
# and the oracle: only the FP32 accumulation order inside the tensor core differs, which can move a bfloat16
# activation by one rounding unit at a tie.
@pytest.mark.parametrize("case", CASES)
def test_bf16_tensor_core_closure_matches_fma_closure(case):
    e = np.load(G / f"euler2d_{case}.npz")
    nx, ny, bc = int(e["nx"]), int(e["ny"]), str(e["bc"])
    p = Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4)
    u0 = e["initial"]
    dt = 0.3 * min(p.dx, p.dy) / O.max_speed(u0, nx, ny)
    outs = {}
    for method in ("sr_bf16", "sr_bf16_tc"):
        out = torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV)
        E.stage(_t(u0), _t(u0), out, p, dt, 1, method, bc, mlp_params=P32)
        outs[method] = _interior(out.cpu().numpy(), nx, ny)
    ref = O.euler2d_stage(u0, u0, np.zeros_like(u0), nx, ny, p.dx, p.dy, dt, 1, "sr_bf16", bc, params=P32)
    assert _rel(outs["sr_bf16_tc"], outs["sr_bf16"]) <= 1e-4
    assert _rel(outs["sr_bf16_tc"], _interior(ref, nx, ny)) <= STAGE_TOL["sr_bf16"]
    bufs = [_t(u0)] + [torch.zeros_like(_t(u0)) for _ in range(3)]
    res = E.run(bufs, p, 1.0, "sr_bf16_tc", bc, mlp_params=P32, fixed_steps=5)
    bufs2 = [_t(u0)] + [torch.zeros_like(_t(u0)) for _ in range(3)]
    res2 = E.run(bufs2, p, 1.0, "sr_bf16", bc, mlp_params=P32, fixed_steps=5)
    got, want = bufs[res.final_slot].cpu().numpy(), bufs2[res2.final_slot].cpu().numpy()
    assert _rel(_interior(got, nx, ny), _interior(want, nx, ny)) <= 1e-3


# The eight-threads-per-face reconstruction kernels (the SR default on small grids) against the one-thread-per-face
# kernels: the same per-stencil arithmetic, so runs agree bit for bit, dts, closure tallies and JS fallbacks included
# (JS and WENO-Z ignore the option: both layouts give the one-thread-per-face kernels).
@pytest.mark.parametrize("method", ["js", "z", "sr_f64", "sr_f32", "sr_bf16"])
@pytest.mark.parametrize("bc,flux", [("transmissive", "hllc"), ("periodic", "force"), ("double-mach", "hllc")])
def test_face_thread_layouts_agree_bitwise(method, bc, flux):
    from weno_sr_publishing_b200 import _native as N

    nx, ny = 61, 47
    if bc == "double-mach":
        p = Params(nx=nx, ny=ny, x_length=4.0, y_length=1.0, cfl=0.4)
        init = problems.double_mach_state(nx, ny, quadrature=3)
    else:
        p = Params(nx=nx, ny=ny, x_length=1.0, y_length=0.8, cfl=0.4)
        init = problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(4), 3)
    out = {}
    for layout in (N.OPT_FACE_THREADS_1, N.OPT_FACE_THREADS_8, N.OPT_FACE_THREADS_4):
        bufs = [_t(init)] + [torch.zeros_like(_t(init)) for _ in range(3)]
        ws = E.workspace(nx, ny, DEV)
        res = E.run(bufs, p, 1.0, method, bc, mlp_params=PARAMS[method], flux=flux, fixed_steps=4,
                    opts=layout | N.OPT_COUNT | N.OPT_JS_FALLBACK, ws=ws)
        out[layout] = (bufs[res.final_slot].cpu().numpy(), res.dts, E.counters(ws), res.fallbacks)
    a = out[N.OPT_FACE_THREADS_1]
    for layout in (N.OPT_FACE_THREADS_8, N.OPT_FACE_THREADS_4):
        b = out[layout]
        np.testing.assert_array_equal(_interior(a[0], nx, ny), _interior(b[0], nx, ny))
        assert a[1] == b[1] and a[2] == b[2] and a[3] == b[3]
