"""Generate the golden fixtures of the 2D path from the reference's own code.

Run in a container that holds the reference checkout (it is never needed at test time):

    python tests/golden/make_golden.py --reference /path/to/WENO_SR_publishing

What it does:

* installs ``warp_shim`` as ``warp`` and imports the reference's Warp modules unchanged
  (``warp_weno5_helpers``, the V20 deploy core, the FP32 core, and the three HLLC adapters);
* evaluates closure weights, JS/SR reconstructions and HLLC/FORCE fluxes on seeded inputs;
* runs the adapters' ``run_to_time`` on small non-square grids for WENO5-JS, WENO5-SR (FP64 MLP)
  and WENO5-SR (FP32 MLP), transmissive and periodic;
* runs ``scripts/verify_release.py::verify_reflection`` (which asserts the reference's own pinned
  MLP outputs) and stores the same fixed-feature outputs.

* runs the WENO5-Z helpers and minimal solver (weno_z_borges_p2_results) the same way (``--only z``).

Outputs: tests/golden/closure2d.npz, hllc2d.npz, euler2d_<case>.npz, mlp_golden.npz, euler2d_z.npz.
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

PARAM_NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")
MODEL64 = HERE.parents[1] / "weno_sr_publishing_b200" / "models" / "weno5_sr_fp64_step012250.npz"
MODEL32 = HERE.parents[1] / "weno_sr_publishing_b200" / "models" / "weno5_sr_fp32_step016500.npz"


def _load(path: Path, dtype) -> dict:
    data = np.load(path)
    return {k: warp_shim.array(data[k], dtype=dtype) for k in PARAM_NAMES}


def make_stencils(rng: np.random.Generator, n: int) -> np.ndarray:
    """Seeded 5-point stencils covering smooth, rough, discontinuous, plateau and near-plateau data."""
    rows = []
    x = np.arange(-2, 3, dtype=np.float64)
    for k in range(n):
        kind = k % 8
        if kind == 0:  # smooth polynomial
            c = rng.normal(size=4)
            q = c[0] + c[1] * x + c[2] * x * x + 0.1 * c[3] * x ** 3
        elif kind == 1:  # random rough
            q = rng.normal(size=5)
        elif kind == 2:  # jump at a random position
            pos = rng.integers(1, 5)
            q = np.where(np.arange(5) < pos, rng.uniform(0.5, 2.0), rng.uniform(-1.0, 1.0))
        elif kind == 3:  # exact plateau
            q = np.full(5, rng.uniform(-3, 3))
        elif kind == 4:  # near plateau (variation around 1e-13 of the scale)
            q = rng.uniform(0.5, 2.0) + rng.uniform(-1, 1, 5) * 10.0 ** rng.uniform(-15, -12)
        elif kind == 5:  # large amplitude
            q = rng.normal(size=5) * 10.0 ** rng.uniform(1, 4)
        elif kind == 6:  # tiny amplitude, small scale
            q = rng.normal(size=5) * 10.0 ** rng.uniform(-10, -4)
        else:  # kink
            q = np.abs(x - rng.uniform(-1, 1)) * rng.uniform(0.1, 3.0)
        rows.append(q)
    return np.asarray(rows, dtype=np.float64)


def gen_closure(wh, deploy, f32core) -> dict:
    rng = np.random.default_rng(20260803)
    q = make_stencils(rng, 96)
    m64 = _load(MODEL64, warp_shim.float64)
    m32 = _load(MODEL32, warp_shim.float32)
    p64 = [m64[k] for k in PARAM_NAMES]
    p32 = [m32[k] for k in PARAM_NAMES]
    out = {"q": q}
    for head in range(4):
        w64 = np.array([deploy.mlp_weights(*map(float, s), head, *p64, 0) for s in q])
        w32 = np.array([f32core.mlp_weights(*map(float, s), head, *p32, 0) for s in q])
        out[f"w_sr_f64_h{head}"] = w64
        out[f"w_sr_f32_h{head}"] = w32
    for lr in (1, 2):
        out[f"v_js_lr{lr}"] = np.array([wh.weno5_lr_value(*map(float, s), lr) for s in q])
        out[f"v_sr_f64_lr{lr}"] = np.array([deploy.weno5_lr_value_mlp(*map(float, s), lr, *p64, 0)[0] for s in q])
        out[f"v_sr_f32_lr{lr}"] = np.array([f32core.weno5_lr_value_mlp(*map(float, s), lr, *p32, 0)[0] for s in q])
    for loca in (1, 2):
        out[f"v_js_g{loca}"] = np.array([wh.weno5_gauss_lr_value(*map(float, s), loca) for s in q])
        out[f"v_sr_f64_g{loca}"] = np.array(
            [deploy.weno5_gauss_value_mlp(*map(float, s), loca, *p64, 0)[0] for s in q])
        out[f"v_sr_f32_g{loca}"] = np.array(
            [f32core.weno5_gauss_value_mlp(*map(float, s), loca, *p32, 0)[0] for s in q])
    out["features"] = np.array([list(deploy.weno5_nn_features(*map(float, s))) for s in q])
    return out


def _random_primitive_pairs(rng: np.random.Generator, n: int) -> tuple[np.ndarray, np.ndarray]:
    def state():
        rho = rng.uniform(0.05, 3.0, n)
        u = rng.uniform(-3.0, 3.0, n)
        v = rng.uniform(-3.0, 3.0, n)
        p = rng.uniform(0.01, 5.0, n)
        e = 0.5 * rho * (u * u + v * v) + p / 0.4
        return np.stack([rho, rho * u, rho * v, e], axis=1)
    left, right = state(), state()
    # degenerate rows: equal states, near vacuum, strongly supersonic both ways, zero velocity
    left[0] = right[0]
    left[1] = [1e-14, 0.0, 0.0, 1e-14]
    right[2] = [1.0, 10.0, 0.0, 0.5 * 100.0 + 1.0 / 0.4]
    left[2] = right[2]
    left[3] = [1.0, -10.0, 3.0, 0.5 * 109.0 + 1.0 / 0.4]
    right[3] = [0.5, -12.0, 0.0, 0.5 * 0.5 * 144.0 + 0.2 / 0.4]
    left[4] = [1.0, 0.0, 0.0, 2.5]
    right[4] = [0.125, 0.0, 0.0, 0.25]
    return left, right


def gen_hllc(hllc5, wh) -> dict:
    rng = np.random.default_rng(20260711)
    left, right = _random_primitive_pairs(rng, 512)
    out = {"left": left, "right": right}
    for d in (1, 2):
        out[f"hllc_d{d}"] = np.array([list(hllc5.hllc_flux(warp_shim.vec4d(a), warp_shim.vec4d(b), d, 1.4))
                                      for a, b in zip(left, right)])
        out[f"force_d{d}"] = np.array([list(wh.force_flux(warp_shim.vec4d(a), warp_shim.vec4d(b), d, 0.3, 1.4))
                                       for a, b in zip(left, right)])
    return out


def random_cell_state(rng, nx, ny, g=3):
    """Rough but physically mild per-cell data (every stencil non-smooth, no vacuum)."""
    shape = (ny + 2 * g, nx + 2 * g)
    rho = rng.uniform(0.8, 1.25, shape)
    u = rng.uniform(-0.3, 0.3, shape)
    v = rng.uniform(-0.3, 0.3, shape)
    p = rng.uniform(0.8, 1.25, shape)
    out = np.zeros(shape + (4,))
    out[..., 0] = rho
    out[..., 1] = rho * u
    out[..., 2] = rho * v
    out[..., 3] = p / 0.4 + 0.5 * rho * (u * u + v * v)
    return out


def smooth_state(nx, ny, g=3):
    jj, ii = np.indices((ny + 2 * g, nx + 2 * g))
    x = (ii - g + 0.5) / nx
    y = (jj - g + 0.5) / ny
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    u = 0.5 + 0.2 * np.cos(2 * np.pi * y)
    v = -0.3 + 0.1 * np.sin(2 * np.pi * x)
    p = 1.0 + 0.2 * np.sin(2 * np.pi * (x + y))
    out = np.zeros((ny + 2 * g, nx + 2 * g, 4))
    out[..., 0] = rho
    out[..., 1] = rho * u
    out[..., 2] = rho * v
    out[..., 3] = p / 0.4 + 0.5 * rho * (u * u + v * v)
    return out


def gen_euler2d(wh, adapters, out_dir: Path) -> None:
    m64 = _load(MODEL64, warp_shim.float64)
    m32 = _load(MODEL32, warp_shim.float32)
    sys.path.insert(0, str(HERE.parents[1]))
    from weno_sr_publishing_b200 import problems  # noqa: PLC0415

    cases = [
        ("rough_trans", 11, 9, "transmissive", "random", 0.1),
        ("quadrant_trans", 12, 10, "transmissive", "quadrant", 0.08),
        ("smooth_periodic", 12, 10, "periodic", "smooth", 0.05),
    ]
    for name, nx, ny, bc, kind, t_end in cases:
        rng = np.random.default_rng(7)
        if kind == "random":
            init = random_cell_state(rng, nx, ny)
        elif kind == "quadrant":
            init = problems.make_quadrant_state(nx, ny, problems.seeded_quadrant_states(0), 15)
        else:
            init = smooth_state(nx, ny)
        rec = {"initial": init, "nx": nx, "ny": ny, "t_end": t_end, "cfl": 0.4, "x_length": 1.0,
               "y_length": 1.0, "bc": bc}
        for key, ad, mlp in (("js", adapters["js"], None), ("sr_f64", adapters["sr_f64"], m64),
                             ("sr_f32", adapters["sr_f32"], m32)):
            params = wh.Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4, t_end=t_end)
            t0 = time.time()
            final, dts, steps, t = ad.run_to_time(init, params, t_end, "cpu", mlp, bc,
                                                  report_interval=0, report=None)
            rec[f"{key}_final"] = np.asarray(final)
            rec[f"{key}_dts"] = np.asarray(dts)
            rec[f"{key}_steps"] = steps
            rec[f"{key}_t"] = t
            # single first stage, for kernel-level checks
            arrays = ad.allocate_forward(init, params, "cpu")
            dt = dts[0]
            if key == "sr_f64":
                ad.launch_stage(arrays["u0"], arrays["u0"], arrays["u1"], arrays["s1"], params, dt, 1, "cpu", mlp,
                                bc, 0.0, False)
            else:
                ad.launch_stage(arrays["u0"], arrays["u0"], arrays["u1"], arrays["s1"], params, dt, 1, "cpu", mlp,
                                bc)
            rec[f"{key}_stage1"] = np.asarray(arrays["u1"])
            print(f"euler2d {name} {key}: steps={steps} t={t:.6g} ({time.time() - t0:.1f}s)", flush=True)
        np.savez_compressed(out_dir / f"euler2d_{name}.npz", **rec)


Z_CASES = [
    ("rough_trans", 11, 9, "transmissive", "random", 0.1),
    ("smooth_periodic", 12, 10, "periodic", "smooth", 0.05),
]


def gen_z(zh, zmin, out_dir: Path) -> None:
    """WENO5-Z (weno_z_borges_p2_results): reconstructions at two spacings, and the minimal solver's
    run_to_time / first stage on non-square grids (dx != dy, so the per-direction eps is exercised)."""
    rng = np.random.default_rng(20260803)
    q = make_stencils(rng, 96)
    rec = {"q": q, "h": np.array([0.05, 1.0e-3])}
    for hi, h in enumerate((0.05, 1.0e-3)):
        for lr in (1, 2):
            rec[f"v_lr{lr}_h{hi}"] = np.array([zh.weno5_lr_value(*map(float, s), lr, h) for s in q])
            rec[f"v_g{lr}_h{hi}"] = np.array([zh.weno5_gauss_lr_value(*map(float, s), lr, h) for s in q])
    for name, nx, ny, bc, kind, t_end in Z_CASES:
        init = random_cell_state(np.random.default_rng(7), nx, ny) if kind == "random" else smooth_state(nx, ny)
        params = zh.Params(nx=nx, ny=ny, x_length=1.0, y_length=1.0, cfl=0.4, t_end=t_end)
        t0 = time.time()
        final, dts, steps, t = zmin.run_to_time(init, params, t_end, "cpu", bc)
        arrays = {"u0": warp_shim.array(init, dtype=warp_shim.float64),
                  "u1": warp_shim.zeros(params.padded_shape, dtype=warp_shim.float64)}
        zmin._launch_stage(arrays["u0"], arrays["u0"], arrays["u1"], zmin._stage(params, "cpu"), params, dts[0], 1,
                           "cpu", bc)
        rec.update({f"{name}_initial": init, f"{name}_final": np.asarray(final), f"{name}_dts": np.asarray(dts),
                    f"{name}_steps": steps, f"{name}_t": t, f"{name}_stage1": np.asarray(arrays["u1"]),
                    f"{name}_nx": nx, f"{name}_ny": ny, f"{name}_t_end": t_end, f"{name}_bc": bc})
        print(f"euler2d z {name}: steps={steps} t={t:.6g} ({time.time() - t0:.1f}s)", flush=True)
    np.savez_compressed(out_dir / "euler2d_z.npz", **rec)


def gen_mlp_golden(reference: Path) -> dict:
    sys.path.insert(0, str(reference / "scripts"))
    vr = importlib.import_module("verify_release")
    messages = vr.verify_reflection()  # asserts the reference's own pinned outputs
    import torch  # noqa: PLC0415

    snapshot = reference / "code" / "snapshot"
    features5 = np.array([[0.12, 0.67, 1.0, 0.31, 0.82], [1.0, 0.28, 0.04, 0.73, 0.46]])
    features7 = np.array([[0.09, 0.36, 0.81, 1.0, 0.27, 0.73], [1.0, 0.71, 0.22, 0.03, 0.64, 0.41]])
    v12 = importlib.import_module("teacherfree_lab_weno5_v12_reflection_sym.v12_model")
    m5 = v12.load_checkpoint(MODEL64, "cpu").eval()
    fast_dir = snapshot / "teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast"
    sys.path.insert(0, str(fast_dir))
    mixed = importlib.import_module("model")
    m5f = mixed.load_checkpoint(MODEL32, "cpu").eval()
    sys.path.remove(str(fast_dir))
    w7 = importlib.import_module("teacherfree_lab_weno7_rk4_distance_balanced_fast.weno7_core")
    m7 = w7.load_checkpoint(HERE.parents[1] / "weno_sr_publishing_b200" / "models" / "weno7_sr_fp64_step016750.npz", "cpu").eval()
    with torch.no_grad():
        f5 = torch.tensor(features5)
        f7 = torch.tensor(features7)
        return {
            "features5_torch_scale": features5,
            "features7": features7,
            "out5_f64": m5(f5).numpy(),
            "out5_f32": m5f(f5).double().numpy(),
            "out7_f64": m7(f7).numpy(),
            "verify_messages": np.array(messages),
        }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    ap.add_argument("--only", default="closure,hllc,euler2d,mlp")
    args = ap.parse_args()
    only = set(args.only.split(","))
    warp_shim.install()
    snapshot = args.reference / "code" / "snapshot"
    sys.path.insert(0, str(snapshot))
    wh = importlib.import_module("warp_weno5_helpers")
    deploy = importlib.import_module("teacherfree_lab_weno5_v20_distance_balanced.weno5_rk3_diff_v20_deploy")
    f32core = importlib.import_module(
        "teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast.warp_mlp_f32.weno5_rk3_diff_mlp_f32")
    hllc5 = importlib.import_module("for_paper_results.solvers.weno5_hllc")
    refsym = importlib.import_module("teacherfree_lab_weno5_v20_distance_balanced.weno5_hllc_refsym")
    mixed = importlib.import_module("for_paper_results.solvers.weno5_hllc_mixed")
    if "closure" in only:
        np.savez_compressed(HERE / "closure2d.npz", **gen_closure(wh, deploy, f32core))
        print("closure2d.npz written", flush=True)
    if "hllc" in only:
        np.savez_compressed(HERE / "hllc2d.npz", **gen_hllc(hllc5, wh))
        print("hllc2d.npz written", flush=True)
    if "euler2d" in only:
        gen_euler2d(wh, {"js": hllc5, "sr_f64": refsym, "sr_f32": mixed}, HERE)
    if "mlp" in only:
        np.savez_compressed(HERE / "mlp_golden.npz", **gen_mlp_golden(args.reference))
        print("mlp_golden.npz written", flush=True)
    if "z" in only:
        zh = importlib.import_module("weno_z_borges_p2_results.weno5_helpers_z")
        zmin = importlib.import_module("weno_z_borges_p2_results.weno5_hllc_z_min")
        gen_z(zh, zmin, HERE)
        print("euler2d_z.npz written", flush=True)


if __name__ == "__main__":
    main()
