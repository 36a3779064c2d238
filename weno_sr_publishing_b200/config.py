"""Method registry (for_paper_results/config.py:30-78 of the reference), WENO5 rows of the 2D path."""
from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

from .checkpoint import MODELS_DIR


@dataclass(frozen=True)
class Method:
    key: str
    label: str
    family: str
    time_integrator: str
    model: Path | None
    mlp_precision: str | None
    color: str
    linestyle: str


METHODS = {
    "weno5_js": Method("weno5_js", "WENO5-JS-RK3", "weno5", "SSPRK3", None, None, "#4D4D4D", "--"),
    "weno5_sr_f64": Method("weno5_sr_f64", "WENO5-SR-RK3", "weno5", "SSPRK3",
                           MODELS_DIR / "weno5_sr_fp64_step012250.npz", "float64", "#0072B2", "-"),
    "weno5_sr_f32": Method("weno5_sr_f32", "WENO5-SR-FP32-RK3", "weno5_mixed", "SSPRK3",
                           MODELS_DIR / "weno5_sr_fp32_step016500.npz", "float32", "#009E73", "-."),
}


def validate_models() -> None:
    missing = [str(m.model) for m in METHODS.values() if m.model is not None and not m.model.is_file()]
    if missing:
        raise FileNotFoundError("missing selected checkpoint(s):\n" + "\n".join(missing))
