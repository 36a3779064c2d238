"""Generate tests/golden/euler2d_w7.npz from the reference's WENO7 point-value Shu-RK4 solver.

Run in a container that holds the reference checkout (never needed at test time):

    python tests/golden/make_golden_w7.py --reference /path/to/WENO_SR_publishing

Through ``warp_shim`` (the reference's Warp kernels executed in Python) it records: the classical WENO7
face and Gauss reconstructions (warp_weno7_ader4_helpers_classical_only.weno7_lr_scalar /
weno7_gauss_lr_scalar) on seeded 7-point stencils; one right-hand side L and L~ (point_rk4.compute_rhs) of the
periodic vortex and of a rough transmissive state; and run_from_initial (HLLC, characteristic) of the vortex
on a 12 x 10 grid and of the rough state on 11 x 9.
"""
from __future__ import annotations

import argparse
import importlib
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import warp_shim  # noqa: E402


def rough_state(rng, nx, ny, g=4):
    shape = (ny + 2 * g, nx + 2 * g)
    rho = rng.uniform(0.8, 1.25, shape)
    u = rng.uniform(-0.3, 0.3, shape)
    v = rng.uniform(-0.3, 0.3, shape)
    p = rng.uniform(0.8, 1.25, shape)
    out = np.zeros(shape + (4,))
    out[..., 0], out[..., 1], out[..., 2] = rho, rho * u, rho * v
    out[..., 3] = p / 0.4 + 0.5 * rho * (u * u + v * v)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    warp_shim.install()
    snap = args.reference / "code" / "snapshot"
    for p in (snap, snap / "weno7_external_clean"):
        sys.path.insert(0, str(p))
    wh = importlib.import_module("weno7_external_clean.warp_weno7_ader4_helpers_classical_only")
    pr = importlib.import_module("weno7_point_rk4_shu.point_rk4")
    rng = np.random.default_rng(20261203)
    q = np.concatenate([rng.normal(size=(40, 7)), np.cumsum(rng.uniform(0, 1, (20, 7)), axis=1),
                        np.where(np.arange(7) < rng.integers(1, 7, (20, 1)), 2.0, 0.5)])
    out = {"q": q}
    for lr in (1, 2):
        out[f"face_lr{lr}"] = np.array([wh.weno7_lr_scalar(*map(float, r), lr, 1.0, 0) for r in q])
        out[f"gauss_lr{lr}"] = np.array([wh.weno7_gauss_lr_scalar(*map(float, r), lr, 1.0, 0) for r in q])
    cases = {
        "vortex": (pr.Params(nx=12, ny=10, t_end=1.0), None, "periodic"),
        "rough": (pr.Params(nx=11, ny=9, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=0.05), 7, "transmissive"),
    }
    for name, (params, seed, bc) in cases.items():
        init = pr.cell_average_state(params, 0.0, 5) if seed is None else rough_state(np.random.default_rng(seed),
                                                                                      params.nx, params.ny)
        out[f"{name}_initial"] = init
        out[f"{name}_meta"] = np.array([params.nx, params.ny, params.x_min, params.x_max, params.y_min, params.y_max,
                                        params.cfl, params.t_end])
        out[f"{name}_bc"] = bc
        for rev in (0, 1):
            arrays = pr.allocate_arrays(init, params, "cpu")
            pr.compute_rhs(arrays, params, "u", "rhs0", 0.01, "cpu", solver_kind=1, characteristic=True,
                           reverse_upwind=bool(rev), boundary=bc)
            g = params.ghost
            out[f"{name}_rhs_rev{rev}"] = np.asarray(arrays["rhs0"])[g:g + params.ny, g:g + params.nx]
        t0 = time.time()
        final, summary = pr.run_from_initial(init, params, device="cpu", riemann_solver="hllc", characteristic=True,
                                             boundary=bc)
        out[f"{name}_final"] = np.asarray(final)
        out[f"{name}_steps"] = summary["steps"]
        out[f"{name}_t"] = summary["t"]
        print(f"{name}: steps={summary['steps']} t={summary['t']:.6g} ({time.time() - t0:.1f}s)", flush=True)
    zh = importlib.import_module("weno_z_borges_p2_results.weno7_helpers_z")
    zr = importlib.import_module("weno_z_borges_p2_results.weno7_point_rk4_z")
    for hi, h in enumerate((0.1, 1.0)):
        for lr in (1, 2):
            out[f"z_face_lr{lr}_h{hi}"] = np.array([zh.weno7_lr_scalar_normalized(*map(float, r), lr, h, 0, 1)
                                                    for r in q])
            out[f"z_gauss_lr{lr}_h{hi}"] = np.array([zh.weno7_gauss_lr_scalar_normalized(*map(float, r), lr, h, 0, 1)
                                                     for r in q])
    out["z_h"] = np.array([0.1, 1.0])
    for name, (params, seed, bc) in cases.items():
        zp = zr.Params(nx=params.nx, ny=params.ny, x_min=params.x_min, x_max=params.x_max, y_min=params.y_min,
                       y_max=params.y_max, t_end=params.t_end)
        init = out[f"{name}_initial"]
        for rev in (0, 1):
            arrays = zr.allocate_arrays(init, zp, "cpu")
            zr.compute_rhs(arrays, zp, "u", "rhs0", 0.01, "cpu", solver_kind=1, characteristic=True,
                           reverse_upwind=bool(rev), boundary=bc, weight_kind=1)
            g = zp.ghost
            out[f"z_{name}_rhs_rev{rev}"] = np.asarray(arrays["rhs0"])[g:g + zp.ny, g:g + zp.nx]
        final, summary = zr.run_from_initial(init, zp, device="cpu", riemann_solver="hllc", characteristic=True,
                                             boundary=bc, weight_kind=1)
        out[f"z_{name}_final"] = np.asarray(final)
        out[f"z_{name}_steps"] = summary["steps"]
        out[f"z_{name}_t"] = summary["t"]
        print(f"z {name}: steps={summary['steps']} t={summary['t']:.6g}", flush=True)
    np.savez_compressed(HERE / "euler2d_w7.npz", **out)
    print("euler2d_w7.npz written")


if __name__ == "__main__":
    main()
