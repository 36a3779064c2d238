"""Generate the golden fixtures of the 3D Euler path by running the reference's own Warp solver.

    python tests/golden/make_golden_3d.py --reference /path/to/WENO_SR_publishing [--only js,sr_f64,sr_f32,ic]

The reference's code/snapshot/warp_weno5_3d_rk3 package (Weno5Rk3Solver, its kernels and the MLP
kernels) is imported with warp_shim.py standing in for warp and executed on a 6 x 5 x 5 grid:

* ``ic``: the solver's own shock-bubble initialisation (3 x 3 x 3 Gauss cell averages) and one WENO5-JS
  step from it;
* ``js``, ``sr_f64``, ``sr_f32``: from a seeded smooth-plus-interface state, the first RK stage and one
  (JS: two) full steps, with the closure of the FP64 / FP32 reference checkpoints for SR;
* ``z``: the same two JS steps with the WENO-Z solver of code/snapshot/weno_z_borges_p2_results
  (Weno5ZRk3Solver, weno5_3d_kernels_z.py). That module replaces the base solver's kernel module when it is
  imported, so ``z`` runs last.

Each case stores the padded state before and after, and the dt of every step (3d_<case>.npz).
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
MODELS = HERE.parents[1] / "weno_sr_publishing_b200" / "models"


def seeded_state(nx, ny, nz, seed=5):
    """Padded conserved state: smooth variations plus an oblique density/pressure interface."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz, (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx,
                          indexing="ij")
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * (x + 0.3 * y)) + np.where(x + 0.5 * y - 0.2 * z > 0.55, 0.6, 0.0)
    u = 0.2 * np.cos(2 * np.pi * y) + 0.1 * rng.standard_normal(x.shape) * 0.1
    v = -0.15 * np.sin(2 * np.pi * z)
    w = 0.1 * np.sin(2 * np.pi * x)
    p = 1.0 + 0.2 * np.cos(2 * np.pi * z) + np.where(x + 0.5 * y - 0.2 * z > 0.55, 0.5, 0.0)
    E = p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)
    inner = np.stack([rho, rho * u, rho * v, rho * w, E], axis=-1)
    return np.pad(inner, ((3, 3), (3, 3), (3, 3), (0, 0)), mode="edge")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    ap.add_argument("--only", default="ic,js,sr_f64,sr_f32,z")
    args = ap.parse_args()
    sys.path.insert(0, str(HERE))
    import warp_shim  # noqa: PLC0415

    warp_shim.install()
    sys.path.insert(0, str(args.reference / "code" / "snapshot"))
    from warp_weno5_3d_rk3 import config as CF  # noqa: PLC0415
    from warp_weno5_3d_rk3 import kernels as K  # noqa: PLC0415
    from warp_weno5_3d_rk3 import solver as S  # noqa: PLC0415

    nx, ny, nz = 6, 5, 5
    models = {"sr_f64": MODELS / "weno5_sr_fp64_step012250.npz", "sr_f32": MODELS / "weno5_sr_fp32_step016500.npz"}
    cases = args.only.split(",")
    cases = [c for c in cases if c != "z"] + (["z"] if "z" in cases else [])
    for case in cases:
        t0 = time.time()
        cfg = CF.ShockBubbleConfig(nx=nx, ny=ny, nz=nz, t_end=1.0 if case != "ic" else 2.0e-5)
        model = models.get(case)
        solver_cls = S.Weno5Rk3Solver
        if case == "z":
            from weno_z_borges_p2_results import weno5_3d_solver_z as SZ  # noqa: PLC0415

            solver_cls = SZ.Weno5ZRk3Solver
            K = SZ.K
        sol = solver_cls(cfg, device="cpu", strict_sync=False, model=model)
        if case == "ic":
            sol.initialize()
        else:
            sol.q[...] = seeded_state(nx, ny, nz)
            sol.launch = None
            S.wp.launch(K.conserved_to_primitive_kernel, cfg.padded_shape[:3], [sol.q, sol.primitive])
        rec = {"q_init": np.array(sol.q, copy=True), "dx": cfg.dx, "dy": cfg.dy, "dz": cfg.dz, "cfl": cfg.cfl,
               "nx": nx, "ny": ny, "nz": nz}
        # first stage alone, on a copy of the solver state
        stage = solver_cls(cfg, device="cpu", strict_sync=False, model=model)
        stage.q[...] = sol.q
        stage.primitive[...] = sol.primitive
        m = stage.max_speed()
        dt = 1.0e10 if m < 1.0e-15 else cfg.cfl * min(cfg.dx, min(cfg.dy, cfg.dz)) / m
        dt = min(dt, cfg.t_end - 0.0)
        stage._rk_stage(1, dt)
        rec["stage1_dt"] = dt
        rec["q_stage1"] = np.array(stage.q, copy=True)
        steps = 2 if case in ("js", "z") else 1
        dts = []
        for _ in range(steps):
            sol.advance()
            dts.append(sol.dt_trace[-1]["dt"])
            rec[f"q_step{len(dts)}"] = np.array(sol.q, copy=True)
        rec["dts"] = np.array(dts)
        np.savez_compressed(HERE / f"3d_{case}.npz", **rec)
        print(case, "written", f"{time.time() - t0:.0f} s", "dts", dts, flush=True)


if __name__ == "__main__":
    main()
