"""Generate tests/golden/double_mach.npz from the reference's double-Mach boundary runs.

Run in a container that holds the reference checkout (never needed at test time):

    python tests/golden/make_golden_double_mach.py --reference /path/to/WENO_SR_publishing

Executes, through ``warp_shim`` (the reference's Warp kernels in Python), the reference's own initial
state (run_double_mach_compare.make_initial_state, 15-point Gauss averages) and run_to_time with
boundary="double-mach" of the FP64 SR adapter (weno5_hllc_refsym), the FP32 SR adapter
(for_paper_results/solvers/weno5_hllc_mixed) and the WENO5-Z solver (weno5_double_mach_z), on a coarse
32 x 8 grid of [0, 4] x [0, 1] for a few steps, plus the first stage of each. matplotlib, which the
initial-state module imports for plotting only, is replaced by an empty stand-in.
"""
from __future__ import annotations

import argparse
import importlib
import sys
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import warp_shim  # noqa: E402

NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")
MODELS = HERE.parents[1] / "weno_sr_publishing_b200" / "models"
NX, NY, T_END = 32, 8, 0.012


def _stub_matplotlib() -> None:
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    warp_shim.install()
    _stub_matplotlib()
    snap = args.reference / "code" / "snapshot"
    sys.path.insert(0, str(snap))
    dmc = importlib.import_module("run_double_mach_compare")
    wh = importlib.import_module("warp_weno5_helpers")
    refsym = importlib.import_module("teacherfree_lab_weno5_v20_distance_balanced.weno5_hllc_refsym")
    mixed = importlib.import_module("for_paper_results.solvers.weno5_hllc_mixed")
    zdm = importlib.import_module("weno_z_borges_p2_results.weno5_double_mach_z")
    zh = importlib.import_module("weno_z_borges_p2_results.weno5_helpers_z")
    params = wh.Params(nx=NX, ny=NY, x_length=4.0, y_length=1.0, cfl=0.4, t_end=T_END)
    init = dmc.make_initial_state(params, 15)
    out = {"initial": init, "nx": NX, "ny": NY, "t_end": T_END}
    m64 = {k: warp_shim.array(np.load(MODELS / "weno5_sr_fp64_step012250.npz")[k], dtype=warp_shim.float64)
           for k in NAMES}
    m32 = {k: warp_shim.array(np.load(MODELS / "weno5_sr_fp32_step016500.npz")[k], dtype=warp_shim.float32)
           for k in NAMES}
    zparams = zh.Params(nx=NX, ny=NY, x_length=4.0, y_length=1.0, cfl=0.4, t_end=T_END)
    runs = {
        "sr_f64": lambda: refsym.run_to_time(init, params, T_END, "cpu", m64, "double-mach", report_interval=0),
        "sr_f32": lambda: mixed.run_to_time(init, params, T_END, "cpu", m32, "double-mach"),
        "z": lambda: zdm.run_to_time(init, zparams, T_END, "cpu"),
    }
    for key, fn in runs.items():
        t0 = time.time()
        final, dts, steps, t = fn()
        out[f"{key}_final"], out[f"{key}_dts"], out[f"{key}_steps"], out[f"{key}_t"] = np.asarray(final), \
            np.asarray(dts), steps, t
        print(f"double-mach {key}: steps={steps} t={t:.6g} ({time.time() - t0:.1f}s)", flush=True)
    np.savez_compressed(HERE / "double_mach.npz", **out)
    print("double_mach.npz written")


if __name__ == "__main__":
    main()
