"""Generate the golden gradients of the closure-training objective from the reference's torch code.

    python tests/golden/make_golden_train.py --reference /path/to/WENO_SR_publishing

For a few small seeded problems (profiles from weno_sr_publishing_b200/profiles.py, balanced velocities,
N cells, S SSPRK3 steps at CFL 0.5), the reference's own modules (code/snapshot/teacherfree_lab_weno5_v20_
distance_balanced_mlp_f32_fast/rk3_advection.py ssprk3_step_signed with model.py's FP32 model, and
teacherfree_lab_weno5_v12_reflection_sym/v12_model.py's FP64 model) roll the trajectories out under
autograd; the loss is the mean |u_k - e_k| over trajectories, steps 1..S and cells, and its gradients
with respect to the MLP parameters and the initial state are written to train1d_grads.npz, together
with the reference's seeded initial parameters (weno5_core.py SharedBadnessMLP) for seed 83.
"""
from __future__ import annotations

import argparse
import importlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
MODELS = ROOT / "weno_sr_publishing_b200" / "models"
NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    snap = args.reference / "code" / "snapshot"
    fast = snap / "teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast"
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(snap))
    sys.path.insert(0, str(fast))
    import torch  # noqa: PLC0415

    from weno_sr_publishing_b200 import profiles as P  # noqa: PLC0415

    torch.set_default_dtype(torch.float64)
    rk3 = importlib.import_module("rk3_advection")
    fmodel = importlib.import_module("model")
    core = importlib.import_module("weno5_core")
    v12 = importlib.import_module("teacherfree_lab_weno5_v12_reflection_sym.v12_model")

    def ref_model(kind, packed, seed=None):
        if kind == "f32":
            m = fmodel.ReflectionSymmetricBadnessMLPFloat32(seed=0 if seed is None else seed)
        else:
            m = v12.ReflectionSymmetricBadnessMLP(seed=0 if seed is None else seed)
        if packed is not None:
            o = 0
            with torch.no_grad():
                for k in NAMES:
                    t = getattr(m, k)
                    t.copy_(torch.as_tensor(packed[o:o + t.numel()]).reshape(t.shape).to(t.dtype))
                    o += t.numel()
        return m

    def packed_of(m):
        return np.concatenate([getattr(m, k).detach().to(torch.float64).reshape(-1).numpy() for k in NAMES])

    def run(m, desc, n, steps, seed_case):
        B = desc.shape[0]
        vel = np.ones(B)
        vel[B // 2:] = -1.0
        cfl = 0.5
        dt = cfl / float(n)
        u0 = P.cell_averages(desc, n, 0.0)
        targets = np.stack([P.cell_averages(desc, n, vel * (float(k) * dt)) for k in range(1, steps + 1)], axis=1)
        u = torch.tensor(u0, requires_grad=True)
        velt = torch.tensor(vel)
        state = u
        total = torch.zeros(())
        for k in range(steps):
            state = rk3.ssprk3_step_signed(m, state, dt, float(n), velt)
            total = total + torch.sum(torch.abs(state - torch.as_tensor(targets[:, k])))
        loss = total / (B * steps * n)
        m.zero_grad()
        loss.backward()
        g = np.concatenate([getattr(m, k).grad.to(torch.float64).reshape(-1).numpy() for k in NAMES])
        return {"desc": desc, "vel": vel, "u0": u0, "targets": targets, "dt": dt, "n": n, "steps": steps,
                "params": packed_of(m), "loss": float(loss.detach()), "grad": g, "grad_u0": u.grad.numpy(),
                "final": state.detach().numpy()}

    rec = {}
    p64 = np.concatenate([np.load(MODELS / "weno5_sr_fp64_step012250.npz")[k].reshape(-1) for k in NAMES])
    p32 = np.concatenate([np.load(MODELS / "weno5_sr_fp32_step016500.npz")[k].reshape(-1).astype(np.float64)
                          for k in NAMES])
    rng = np.random.default_rng(20240611)
    cases = {
        "trained_f64": ("f64", p64, 32, 6, 6, None),
        "trained_f32": ("f32", p32, 32, 6, 6, None),
        "perturbed_f64": ("f64", p64 + 0.05 * rng.standard_normal(p64.size), 40, 8, 5, None),
        "init_f64": ("f64", None, 24, 4, 4, 83),
        "init_f32": ("f32", None, 24, 4, 4, 83),
    }
    for name, (kind, packed, n, B, steps, seed) in cases.items():
        desc, _ = P.make_profiles(rng, B, n)
        m = ref_model(kind, packed, seed)
        out = run(m, desc, n, steps, name)
        for k, v in out.items():
            rec[f"{name}_{k}"] = np.asarray(v)
        print(name, "loss", out["loss"], "|grad|", float(np.linalg.norm(out["grad"])), flush=True)
    np.savez_compressed(HERE / "train1d_grads.npz", **rec)
    print("train1d_grads.npz written", flush=True)


if __name__ == "__main__":
    main()
