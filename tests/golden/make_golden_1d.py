"""Generate the golden fixtures of the batched 1D advection path from the reference's torch code.

    python tests/golden/make_golden_1d.py --reference /path/to/WENO_SR_publishing

* gste.npz: for_paper_results/run_gste.py::run_torch_methods at N=200, t=10, CFL 0.6 for WENO5-JS,
  WENO5-SR (FP64, FP32) and WENO7-JS/SR (the paper's GSTE table), with initial, final and exact
  cell averages and the L1 errors;
* adv1d_steps.npz: a few seeded trajectories (several N, both velocity signs) advanced by the
  reference's ssprk3_step_signed / rollout_distance (WENO5) and shu_rk4_step_signed (WENO7);
* adv1d_z.npz: the WENO-Z GSTE rows of weno_z_borges_p2_results/run_gste.py (N=200, t=10, CFL 0.6:
  WENO5-Z with SSPRK3, WENO7-Z with Shu RK4, through its integrate()), and seeded trajectories advanced a
  few steps by torch_weno_z.ssprk3_step / shu_rk4_step (velocity +1, the only sign that module has).
"""
from __future__ import annotations

import argparse
import importlib
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
MODELS = HERE.parents[1] / "weno_sr_publishing_b200" / "models"


def seeded_profiles(rng, n):
    x = (np.arange(n) + 0.5) / n
    kind = rng.integers(0, 3)
    if kind == 0:
        u = 0.5 + 0.3 * np.sin(2 * np.pi * rng.integers(1, 5) * x + rng.uniform(0, 6.28))
    elif kind == 1:
        u = np.where((x > 0.3) & (x < 0.3 + rng.uniform(0.1, 0.4)), rng.uniform(0.5, 1.0), 0.0)
    else:
        u = np.exp(-((x - 0.5) / rng.uniform(0.03, 0.1)) ** 2) + np.where(x > 0.8, 0.5, 0.0)
    return u


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    ap.add_argument("--only", default="gste,steps,z")
    args = ap.parse_args()
    only = set(args.only.split(","))
    snap = args.reference / "code" / "snapshot"
    sys.path.insert(0, str(snap))
    import torch  # noqa: PLC0415

    torch.set_default_dtype(torch.float64)
    if "gste" in only:
        gste = importlib.import_module("for_paper_results.run_gste")
        methods = {"weno5_js", "weno5_sr_f64", "weno5_sr_f32", "weno7_js", "weno7_sr_f64"}
        with tempfile.TemporaryDirectory() as tmp:
            rows = gste.run_torch_methods(200, 10.0, torch.device("cpu"), Path(tmp), 15, methods, 0.6, 0.6)
            rec = {}
            for row in rows:
                d = np.load(Path(tmp) / f"{row['method']}.npz")
                rec[f"{row['method']}_final"] = d["final"]
                rec[f"{row['method']}_l1"] = row["l1"]
                rec[f"{row['method']}_steps"] = row["steps"]
                rec["initial"] = d["initial"]
                rec["exact"] = d["exact"]
        np.savez_compressed(HERE / "gste.npz", **rec)
        print("gste.npz written", {k: v for k, v in rec.items() if k.endswith("_l1")}, flush=True)
    if "steps" in only:
        fast = snap / "teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast"
        sys.path.insert(0, str(fast))
        rk3 = importlib.import_module("rk3_advection")
        model32 = importlib.import_module("model").load_checkpoint(MODELS / "weno5_sr_fp32_step016500.npz", "cpu")
        v12 = importlib.import_module("teacherfree_lab_weno5_v12_reflection_sym.v12_model")
        model64 = v12.load_checkpoint(MODELS / "weno5_sr_fp64_step012250.npz", "cpu")
        sys.path.remove(str(fast))
        w7dir = snap / "teacherfree_lab_weno7_rk4_distance_balanced_fast-2"
        sys.path.insert(0, str(w7dir))
        for name in ("weno7_core", "rk4_advection"):
            sys.modules.pop(name, None)
        w7 = importlib.import_module("weno7_core")
        rk4 = importlib.import_module("rk4_advection")
        model7 = w7.load_checkpoint(MODELS / "weno7_sr_fp64_step016750.npz", "cpu")
        rng = np.random.default_rng(104729)
        rec = {}
        for case, n in enumerate((37, 64, 100)):
            u0 = np.stack([seeded_profiles(rng, n) for _ in range(2)])
            vel = torch.tensor([1.0, -1.0])
            rec[f"c{case}_u0"] = u0
            dx = 1.0 / n
            for key, model in (("js", "classical"), ("sr_f64", model64), ("sr_f32", model32)):
                with torch.no_grad():
                    u = torch.tensor(u0)
                    for _ in range(3):
                        u = rk3.ssprk3_step_signed(model, u, 0.5 * dx, 1.0 / dx, vel)
                    rec[f"c{case}_w5_{key}_3steps"] = u.numpy()
                    rec[f"c{case}_w5_{key}_dist"] = rk3.rollout_distance(model, torch.tensor(u0), 2.3, 0.5,
                                                                         vel).numpy()
            for key, model in (("js", "classical"), ("sr_f64", model7)):
                with torch.no_grad():
                    u = torch.tensor(u0)
                    for _ in range(3):
                        u = rk4.shu_rk4_step_signed(model, u, 0.5 * dx, 1.0 / dx, vel)
                    rec[f"c{case}_w7_{key}_3steps"] = u.numpy()
        np.savez_compressed(HERE / "adv1d_steps.npz", **rec)
        print("adv1d_steps.npz written", flush=True)
    if "z" in only:
        zg = importlib.import_module("weno_z_borges_p2_results.run_gste")
        Z = importlib.import_module("weno_z_borges_p2_results.torch_weno_z")
        gste = importlib.import_module("for_paper_results.run_gste")
        Z.self_test()
        rec = {}
        x, initial = gste.cell_averages(200, 0.0, 15)
        _, exact = gste.cell_averages(200, 10.0, 15)
        rec["initial"], rec["exact"] = initial, exact
        for key, stepper in (("weno5_z", Z.ssprk3_step), ("weno7_z", Z.shu_rk4_step)):
            final, steps, dt, _ = zg.integrate(initial, 10.0, 0.6, stepper, "cpu")
            rec[f"{key}_final"] = final
            rec[f"{key}_steps"] = steps
            rec[f"{key}_dt"] = dt
            rec[f"{key}_l1"] = float(np.mean(np.abs(final - exact)))
        rng = np.random.default_rng(7919)
        for case, n in enumerate((37, 64, 100)):
            u0 = np.stack([seeded_profiles(rng, n) for _ in range(3)])
            rec[f"c{case}_u0"] = u0
            dx = 1.0 / n
            with torch.no_grad():
                for key, stepper in (("w5", Z.ssprk3_step), ("w7", Z.shu_rk4_step)):
                    u = torch.tensor(u0)
                    for _ in range(3):
                        u = stepper(u, 0.5 * dx, 1.0 / dx)
                    rec[f"c{case}_{key}_3steps"] = u.numpy()
        np.savez_compressed(HERE / "adv1d_z.npz", **rec)
        print("adv1d_z.npz written", {k: v for k, v in rec.items() if k.endswith("_l1")}, flush=True)


if __name__ == "__main__":
    main()
