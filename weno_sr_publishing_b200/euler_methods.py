"""Unified entry points of the five Euler methods (for_paper_results/solvers/euler_methods.py:27-96 of the
reference): run_weno5 for the WENO5 rows of config.METHODS, run_weno7 for the WENO7 rows."""
from __future__ import annotations

from typing import Any

import numpy as np

from . import config
from . import euler2d_w7
from .checkpoint import load_mlp_params, load_mlp_params_f32
from .params import Params
from .solvers import weno5_hllc, weno5_hllc_mixed, weno5_hllc_refsym


def make_weno5_params(nx: int, ny: int, x_length: float, y_length: float, cfl: float, t_end: float,
                      mixed: bool = False) -> Params:
    del mixed  # one Params class serves both precisions
    return Params(nx=nx, ny=ny, x_length=x_length, y_length=y_length, cfl=cfl, t_end=t_end)


def make_weno7_params(nx: int, ny: int, x_min: float, x_max: float, y_min: float, y_max: float, cfl: float,
                      t_end: float) -> euler2d_w7.Params:
    """Params of the WENO7 path on [x_min, x_max] x [y_min, y_max] (euler_methods.py:33-38)."""
    return euler2d_w7.Params(nx=nx, ny=ny, x_min=x_min, x_max=x_max, y_min=y_min, y_max=y_max, cfl=cfl, t_end=t_end)


def run_weno5(method_key: str, initial: np.ndarray, params: Params, *, device: str, boundary: str,
              report_interval: int = 0) -> tuple[np.ndarray, dict[str, Any]]:
    method = config.METHODS.get(method_key)
    if method_key == "weno5_js":
        adapter, mlp_params = weno5_hllc, None
    elif method_key == "weno5_sr_f64":
        adapter, mlp_params = weno5_hllc_refsym, load_mlp_params(method.model, device)
    elif method_key == "weno5_sr_f32":
        adapter, mlp_params = weno5_hllc_mixed, load_mlp_params_f32(method.model, device)
    else:
        raise ValueError(f"not a WENO5 paper method: {method_key}")

    def report(step: int, t: float, dt: float, stats: dict[str, float]) -> None:
        print(f"{method_key} step={step:05d} t={t:.8e} dt={dt:.4e} "
              f"rho=[{stats['rho_min']:.5e},{stats['rho_max']:.5e}] "
              f"p=[{stats['p_min']:.5e},{stats['p_max']:.5e}] nan={int(stats['nan_count'])}", flush=True)

    final, dts, steps, t = adapter.run_to_time(initial, params, params.t_end, device, mlp_params, boundary,
                                               report_interval=report_interval,
                                               report=report if report_interval else None)
    return final, {
        "method": method_key, "riemann_solver": "hllc", "weno_space": "characteristic", "eno_cutoff": False,
        "steps": steps, "t": t,
        "dt_min": min(dts) if dts else 0.0, "dt_max": max(dts) if dts else 0.0,
        "dt_mean": float(np.mean(dts)) if dts else 0.0,
    }


def run_weno7(method_key: str, initial: np.ndarray, params: euler2d_w7.Params, *, device: str, boundary: str,
              report_interval: int = 0) -> tuple[np.ndarray, dict[str, Any]]:
    """WENO7-JS or WENO7-SR (FP64 closure) with Shu RK4 and HLLC, characteristic normal reconstruction
    (euler_methods.py:81-96): (final padded state, summary) of euler2d_w7.run_from_initial(_mlp)."""
    if method_key == "weno7_js":
        return euler2d_w7.run_from_initial(initial, params, device=device, riemann_solver="hllc", characteristic=True,
                                           boundary=boundary, report_interval=report_interval)
    if method_key == "weno7_sr_f64":
        beta = euler2d_w7.Weno7PointBeta(config.METHODS[method_key].model, device, params.gamma)
        return euler2d_w7.run_from_initial_mlp(initial, params, device=device, riemann_solver="hllc",
                                               beta_model=beta, boundary=boundary, eno_cutoff=False,
                                               report_interval=report_interval)
    raise ValueError(f"not a WENO7 paper method: {method_key}")
