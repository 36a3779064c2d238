"""CUDA 2D WENO7 (JS and Z weights) with Shu RK4 (C ABI) against the reference's solver fixtures, the
oracle, and the reference's published vortex, Sod and Lax tables."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from weno_sr_publishing_b200 import accuracy as A
from weno_sr_publishing_b200 import euler2d_w7 as E7
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200 import riemann as R

pytestmark = pytest.mark.gpu

G = Path(__file__).resolve().parent / "golden" / "euler2d_w7.npz"
DEV = "cuda:0"
# The classical WENO7 betas use unnormalised coefficients (up to 17246) that cancel to small values on
# smooth data, and the weights divide by (1e-6 + beta)^2: rounding differences of the contracted (FMA)
# characteristic projections move the right-hand side of the coarse 12 x 10 vortex by ~2e-11 of its maximum
# (the betas themselves are evaluated without contraction, as the reference does).
RHS_TOL = 5e-11
RUN_TOL = 1e-11


def _gold():
    if not G.exists():
        pytest.skip("euler2d_w7.npz not generated")
    return np.load(G)


def _params(g, name):
    nx, ny, x0, x1, y0, y1, cfl, t_end = g[f"{name}_meta"]
    return E7.Params(nx=int(nx), ny=int(ny), x_min=x0, x_max=x1, y_min=y0, y_max=y1, cfl=cfl, t_end=t_end)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", ["vortex", "rough"])
@pytest.mark.parametrize("rev", [0, 1])
def test_rhs_matches_reference(name, rev):
    g = _gold()
    p = _params(g, name)
    u = torch.as_tensor(g[f"{name}_initial"], device=DEV).contiguous()
    got = E7.rhs(u, p, str(g[f"{name}_bc"]), reverse=bool(rev)).cpu().numpy()
    ref = g[f"{name}_rhs_rev{rev}"]
    assert np.abs(got - ref).max() <= RHS_TOL * np.abs(ref).max()


@pytest.mark.parametrize("name", ["vortex", "rough"])
def test_run_from_initial_matches_reference(name):
    g = _gold()
    p = _params(g, name)
    final, summary = E7.run_from_initial(g[f"{name}_initial"], p, device=DEV, boundary=str(g[f"{name}_bc"]))
    assert summary["steps"] == int(g[f"{name}_steps"]) and abs(summary["t"] - float(g[f"{name}_t"])) <= 1e-14
    assert _rel(final[4:-4, 4:-4], g[f"{name}_final"][4:-4, 4:-4]) <= RUN_TOL


@pytest.mark.parametrize("bc", ["periodic", "transmissive"])
def test_ragged_grid_against_oracle(bc):
    nx, ny = 37, 23
    p = E7.Params(nx=nx, ny=ny, cfl=0.4, t_end=0.6)
    init = problems.vortex_point_rk4(nx, ny, 0.0, 3)
    ref, rdts, rsteps, rt = O.w7_run(init, nx, ny, p.dx, p.dy, 0.4, 0.6, bc)
    u = torch.as_tensor(init, device=DEV).contiguous()
    res = E7.run(u, p, bc)
    assert res.steps == rsteps and res.t == pytest.approx(rt, abs=1e-15)
    np.testing.assert_allclose(res.dts, rdts, rtol=1e-12)
    assert _rel(u.cpu().numpy()[4:-4, 4:-4], ref[4:-4, 4:-4]) <= RUN_TOL


def test_report_interval_path_equals_device_loop():
    p = E7.Params(nx=20, ny=16, cfl=0.4, t_end=0.9)
    init = problems.vortex_point_rk4(20, 16, 0.0, 3)
    a, sa = E7.run_from_initial(init, p, device=DEV)
    b, sb = E7.run_from_initial(init, p, device=DEV, report_interval=2)
    assert sa["steps"] == sb["steps"] and sa["t"] == sb["t"]
    np.testing.assert_array_equal(a[4:-4, 4:-4], b[4:-4, 4:-4])


# WENO7-JS-RK4 rows of experiments/05_isentropic_vortex/tables/vortex_convergence.md: (L1, L2) of rho
VORTEX = {25: (1.48745803e-03, 7.10533170e-03), 50: (1.30815287e-04, 6.74983405e-04),
          100: (4.64194593e-06, 2.14910919e-05), 200: (1.06985939e-07, 6.36224117e-07)}


@pytest.mark.parametrize("n", [25, 50, 100, 200])
def test_vortex_table(n):
    r = A.vortex7_run(n, DEV)
    for got, ref in zip((r.l1, r.l2), VORTEX[n]):
        assert abs(got / ref - 1.0) <= 1e-8, (n, got, ref)


def test_sod_and_lax_tables():
    """weno7_js rows of experiments/02 (Sod: rho L1, L2, Linf) and 03 (Lax: rho, u, p)."""
    r = R.shock_tube_run(R.SOD, "w7_js", device=DEV)
    for got, ref in zip((r["rho_l1_mean"], r["rho_l2"], r["rho_linf"]),
                        (0.004933950990989144, 0.010405878939514045, 0.05208597567533657)):
        assert abs(got / ref - 1.0) <= 1e-9, (got, ref)
    r = R.shock_tube_run(R.LAX, "w7_js", device=DEV)
    lax = {"rho": (0.0059790562598758135, 0.03112867804980643, 0.3303178860042355),
           "velocity": (0.005698264470257289, 0.02511650899704151, 0.3210318145435665),
           "pressure": (0.006900526734718968, 0.024887536217841295, 0.22531532403641452)}
    for field, ref in lax.items():
        for got, rv in zip((r[f"{field}_l1_mean"], r[f"{field}_l2"], r[f"{field}_linf"]), ref):
            assert abs(got / rv - 1.0) <= 1e-9, (field, got, rv)


@pytest.mark.parametrize("name", ["vortex", "rough"])
@pytest.mark.parametrize("rev", [0, 1])
def test_z_rhs_matches_reference(name, rev):
    """weno7_point_rk4_z (weight_kind 1: p = 3, betas / 240, eps = h^3) right-hand sides."""
    g = _gold()
    p = _params(g, name)
    u = torch.as_tensor(g[f"{name}_initial"], device=DEV).contiguous()
    got = E7.rhs(u, p, str(g[f"{name}_bc"]), reverse=bool(rev), method="z").cpu().numpy()
    ref = g[f"z_{name}_rhs_rev{rev}"]
    assert np.abs(got - ref).max() <= RHS_TOL * np.abs(ref).max()


@pytest.mark.parametrize("name", ["vortex", "rough"])
def test_z_run_from_initial_matches_reference(name):
    g = _gold()
    p = _params(g, name)
    final, summary = E7.run_from_initial(g[f"{name}_initial"], p, device=DEV, boundary=str(g[f"{name}_bc"]),
                                         method="z")
    assert summary["steps"] == int(g[f"z_{name}_steps"]) and abs(summary["t"] - float(g[f"z_{name}_t"])) <= 1e-14
    assert _rel(final[4:-4, 4:-4], g[f"z_{name}_final"][4:-4, 4:-4]) <= RUN_TOL


@pytest.mark.parametrize("bc", ["periodic", "transmissive"])
def test_z_ragged_grid_against_oracle(bc):
    nx, ny = 29, 41
    p = E7.Params(nx=nx, ny=ny, cfl=0.4, t_end=0.5)
    init = problems.vortex_point_rk4(nx, ny, 0.0, 3)
    ref, rdts, rsteps, rt = O.w7_run(init, nx, ny, p.dx, p.dy, 0.4, 0.5, bc, method="z")
    u = torch.as_tensor(init, device=DEV).contiguous()
    res = E7.run(u, p, bc, method="z")
    assert res.steps == rsteps and res.t == pytest.approx(rt, abs=1e-15)
    np.testing.assert_allclose(res.dts, rdts, rtol=1e-12)
    assert _rel(u.cpu().numpy()[4:-4, 4:-4], ref[4:-4, 4:-4]) <= RUN_TOL


# WENO7-Z-RK4 rows of experiments/05_isentropic_vortex/tables/vortex_convergence.md: (L1, L2) of rho
VORTEX_Z = {25: (9.24722844e-04, 3.80751034e-03), 50: (8.30137623e-05, 4.47443425e-04),
            100: (2.38982847e-06, 1.31101155e-05), 200: (2.93282637e-08, 1.71997176e-07)}


@pytest.mark.parametrize("n", [25, 50, 100, 200])
def test_z_vortex_table(n):
    r = A.vortex7_run(n, DEV, method="z")
    for got, ref in zip((r.l1, r.l2), VORTEX_Z[n]):
        assert abs(got / ref - 1.0) <= 1e-8, (n, got, ref)


def test_z_sod_and_lax_tables():
    """weno7_z_p3 rows of experiments/02 (Sod: rho L1, L2, Linf) and 03 (Lax: rho, u, p)."""
    r = R.shock_tube_run(R.SOD, "w7_z", device=DEV)
    for got, ref in zip((r["rho_l1_mean"], r["rho_l2"], r["rho_linf"]),
                        (0.005067383382686812, 0.010572181673056028, 0.05182032580354834)):
        assert abs(got / ref - 1.0) <= 1e-9, (got, ref)
    r = R.shock_tube_run(R.LAX, "w7_z", device=DEV)
    lax = {"rho": (0.006104027658765422, 0.03149785277140588, 0.3313187561959483),
           "velocity": (0.006087585881834266, 0.027071085748154113, 0.3470615588986299),
           "pressure": (0.007345408696330224, 0.02675261391710653, 0.24739722211405157)}
    for field, ref in lax.items():
        for got, rv in zip((r[f"{field}_l1_mean"], r[f"{field}_l2"], r[f"{field}_linf"]), ref):
            assert abs(got / rv - 1.0) <= 1e-9, (field, got, rv)


def test_invalid_arguments_raise():
    p = E7.Params(nx=3, ny=8)
    with pytest.raises(ValueError):
        E7.workspace(3, 8, DEV)
    p = E7.Params(nx=8, ny=8)
    with pytest.raises(ValueError):
        E7.run(torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV), p, "reflective")
    with pytest.raises(NotImplementedError):
        E7.run_from_initial(np.zeros(p.padded_shape), p, device=DEV, riemann_solver="evilin")
    with pytest.raises(ValueError):
        E7.rhs(torch.zeros(p.padded_shape, dtype=torch.float64, device=DEV), p, method="sr_f32")
