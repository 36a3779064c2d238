"""Method registry (for_paper_results/config.py:30-78 of the reference): the five Euler methods of the paper,
three WENO5 rows (SSPRK3) and two WENO7 rows (Shu RK4)."""
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
    "weno7_js": Method("weno7_js", "WENO7-JS-RK4", "weno7", "SSP-RK4", None, None, "#D55E00", "--"),
    "weno7_sr_f64": Method("weno7_sr_f64", "WENO7-SR-RK4", "weno7", "SSP-RK4",
                           MODELS_DIR / "weno7_sr_fp64_step016750.npz", "float64", "#CC79A7", "-"),
}

EULER_METHODS = tuple(METHODS)


def validate_models() -> None:
    missing = [str(m.model) for m in METHODS.values() if m.model is not None and not m.model.is_file()]
    if missing:
        raise FileNotFoundError("missing selected checkpoint(s):\n" + "\n".join(missing))
