"""Generate tests/golden/euler2d_w7_sr.npz from the reference's 2D WENO7-SR (FP64 closure) Shu-RK4 solver.

Run in a container that holds the reference checkout (never needed at test time):

    python tests/golden/make_golden_w7_sr.py --reference /path/to/WENO_SR_publishing

The paper's WENO7-SR-RK4 method (for_paper_results/solvers/euler_methods.py:88-95) evaluates the closure
with torch (teacherfree_lab_weno7_rk4_distance_balanced_fast/warp_sod/beta_provider.py, checkpoint
model_step_016750.npz) and reconstructs in Warp (warp_sod/point_rk4_mlp.py,
warp_weno7_external_overwrite_fullall.py); the Warp kernels run in Python through ``warp_shim``. Recorded:
closure betas on seeded 7-point stencils in both orientations; the face and Gauss reconstructions from those
betas; one right-hand side L and L~ (compute_rhs_mlp) of the periodic vortex and of a rough transmissive
state; run_from_initial_mlp of both (the grids and end times of euler2d_w7.npz).
"""
from __future__ import annotations

import argparse
import importlib
import sys
import time
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import warp_shim  # noqa: E402
from make_golden_w7 import rough_state  # noqa: E402

CKPT = ("teacherfree_lab_weno7_rk4_distance_balanced_fast/runs/apost_weno7_rk4_distance_balanced_fast_4090_200k/"
        "checkpoints/model_step_016750.npz")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    warp_shim.install()
    snap = args.reference / "code" / "snapshot"
    for p in (snap, snap / "weno7_external_clean"):
        sys.path.insert(0, str(p))
    m = importlib.import_module("teacherfree_lab_weno7_rk4_distance_balanced_fast.warp_sod.point_rk4_mlp")
    ext = m.ext
    wp = warp_shim
    base = m.base
    beta = m.TorchWeno7PointBeta(snap / CKPT, "cpu", 1.4)
    rng = np.random.default_rng(20261204)
    q = np.concatenate([rng.normal(size=(40, 7)), np.cumsum(rng.uniform(0, 1, (20, 7)), axis=1),
                        np.where(np.arange(7) < rng.integers(1, 7, (20, 1)), 2.0, 0.5),
                        1.0 + 1e-15 * rng.normal(size=(6, 7)), np.full((2, 7), 0.75),
                        3.0 + 1e-9 * rng.normal(size=(6, 7))])
    qt = torch.as_tensor(q)
    with torch.no_grad():
        b1 = beta._mlp_beta(qt).numpy()
        b2 = torch.flip(beta._mlp_beta(torch.flip(qt, dims=(-1,))), dims=(-1,)).numpy()
    out = {"q": q, "beta_lr1": b1, "beta_lr2": b2}
    for lr, b in ((1, b1), (2, b2)):
        out[f"face_lr{lr}"] = np.array([ext._weno7_lr_scalar_external_beta(*map(float, r), lr, 1.0, 0,
                                                                            wp.vec4d(*map(float, bb)), 0)
                                        for r, bb in zip(q, b)])
        out[f"gauss_lr{lr}"] = np.array([ext._weno7_gauss_lr_scalar_external_beta(*map(float, r), lr, 1.0, 0,
                                                                                   wp.vec4d(*map(float, bb)), 0)
                                         for r, bb in zip(q, b)])
    cases = {
        "vortex": (base.Params(nx=12, ny=10, t_end=1.0), None, "periodic"),
        "rough": (base.Params(nx=11, ny=9, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, t_end=0.05), 7,
                  "transmissive"),
    }
    for name, (params, seed, bc) in cases.items():
        init = base.cell_average_state(params, 0.0, 5) if seed is None else rough_state(np.random.default_rng(seed),
                                                                                        params.nx, params.ny)
        out[f"{name}_initial"] = init
        out[f"{name}_meta"] = np.array([params.nx, params.ny, params.x_min, params.x_max, params.y_min, params.y_max,
                                        params.cfl, params.t_end])
        out[f"{name}_bc"] = bc
        for rev in (0, 1):
            arrays = m.allocate_arrays_mlp(init, params, "cpu")
            m.compute_rhs_mlp(arrays, params, "u", "rhs0", 0.01, "cpu", solver_kind=1, beta_model=beta,
                              reverse_upwind=bool(rev), boundary=bc)
            g = params.ghost
            out[f"{name}_rhs_rev{rev}"] = np.asarray(arrays["rhs0"])[g:g + params.ny, g:g + params.nx]
        t0 = time.time()
        final, summary = m.run_from_initial_mlp(init, params, device="cpu", riemann_solver="hllc", beta_model=beta,
                                                boundary=bc)
        out[f"{name}_final"] = np.asarray(final)
        out[f"{name}_steps"] = summary["steps"]
        out[f"{name}_t"] = summary["t"]
        print(f"{name}: steps={summary['steps']} t={summary['t']:.6g} ({time.time() - t0:.1f}s)", flush=True)
    np.savez_compressed(HERE / "euler2d_w7_sr.npz", **out)
    print("euler2d_w7_sr.npz written")


if __name__ == "__main__":
    main()
