"""WENO5-SR checkpoint I/O in the reference's .npz format.

Format (teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/weno5_core.py:62-126): arrays
w1 (1,5,10), b1 (1,10), w2 (1,10,6), b2 (1,6), w3 (1,6,6), b3 (1,6), w4 (1,6,3), b4 (1,3) plus a
0-d unicode ``meta_json``. Loaders follow run_weno5_circle_mlp_compare.py:49-81 (FP64) and
teacherfree_lab_weno5_mlp_f32/warp_mlp_f32/run_weno5_circle_mlp_compare_mlp_f32.py:52-84 (FP32): a
ValueError on missing arrays or wrong shapes, a printed warning when the architecture tag is absent.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

PARAM_NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")
ARCH_TAG = "shared_direct_beta_ratio_5_10_6_6_3"
EXPECTED_SHAPES = {
    "w1": (1, 5, 10), "b1": (1, 10), "w2": (1, 10, 6), "b2": (1, 6),
    "w3": (1, 6, 6), "b3": (1, 6), "w4": (1, 6, 3), "b4": (1, 3),
}
MODELS_DIR = Path(__file__).resolve().parent / "models"


def _read(model_path) -> dict[str, np.ndarray]:
    data = np.load(model_path, allow_pickle=True)
    missing = [name for name in PARAM_NAMES if name not in data.files]
    if missing:
        raise ValueError(f"Model {model_path} is missing arrays: {missing}")
    wrong = {name: data[name].shape for name, shape in EXPECTED_SHAPES.items() if data[name].shape != shape}
    if wrong:
        raise ValueError(
            f"Model {model_path} uses old/incompatible MLP shapes: {wrong}. "
            "Retrain with the shared direct beta-ratio 5->10->6->6->3 WENO5-NN architecture.")
    if "meta_json" in data.files:
        meta = str(data["meta_json"])
        if ARCH_TAG not in meta:
            print("warning: model metadata does not say it was trained with the "
                  "shared direct beta-ratio 5->10->6->6->3 WENO5-NN architecture; retrain before trusting "
                  "this comparison.")
    return {name: np.asarray(data[name]) for name in PARAM_NAMES}


def _to_device(arrays: dict[str, np.ndarray], device: str, dtype):
    import torch  # noqa: PLC0415

    tdtype = torch.float64 if dtype == np.float64 else torch.float32
    return {k: torch.as_tensor(v.astype(dtype), device=device, dtype=tdtype) for k, v in arrays.items()}


def load_mlp_params(model_path, device: str = "cuda") -> dict:
    """FP64 loader: {w1..b4} as float64 tensors on `device`."""
    return _to_device(_read(model_path), device, np.float64)


def load_mlp_params_f32(model_path, device: str = "cuda") -> dict:
    """FP32 loader: {w1..b4} as float32 tensors on `device`."""
    return _to_device(_read(model_path), device, np.float32)


def checkpoint_payload(params: dict, meta: dict) -> dict[str, np.ndarray]:
    """Arrays and meta_json as the reference writes them (weno5_core.py:75-99)."""
    payload = {}
    for k in PARAM_NAMES:
        v = params[k]
        if hasattr(v, "detach"):
            v = v.detach().cpu().numpy()
        v = np.asarray(v)
        payload[k] = v.reshape(EXPECTED_SHAPES[k])
    full_meta = {
        "mlp_architecture": f"{ARCH_TAG}_power2_normdelta_scale",
        "mlp_features": ("[delta0/max_delta, delta1/max_delta, delta2/max_delta, gamma_s, "
                         "clipped((log10(max_delta/q_scale)+16)/16)]"),
        "mlp_weight_formula": ("shared hidden MLP direct beta-like badness logits: 5->10->6->6->3; "
                               "r=softmax(6*tanh(raw/6)); beta=3*r; omega=normalize(d/(beta+1e-12)^2)"),
    }
    full_meta.update(meta)
    payload["meta_json"] = np.array(json.dumps(full_meta, sort_keys=True), dtype=np.str_)
    return payload


def save_checkpoint(path, params: dict, meta: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez(path, **checkpoint_payload(params, meta))
