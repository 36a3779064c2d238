"""Sod checkpoint monitor: every saved closure checkpoint of a training run, evaluated on the Sod shock tube.

The reference watches a training run directory and, for every checkpoint whose step is a multiple of an interval,
runs a Sod problem with WENO5-JS and with the checkpoint's closure and records their density errors against the
exact solution (teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/sod_checkpoint_monitor.py:27-101 driving
warp_sod_validation.py:339-548). Here the runs go through this package's 2D kernels (euler2d.run, device-resident
time loop with the per-step health check) and the exact solution through riemann.py:

* problem: Sod on [-0.5, 0.5] x [0, ny/nx] (axis "x", the reference's monitor) or its transpose (axis "y":
  a unit-length tube along y with square cells), left (1, 0, 1), right (0.125, 0, 0.1), interface at 0,
  gamma 1.4, transmissive, CFL 0.4 to t = 0.25, 100 x 10 cells; initial and exact states are 15-point Gauss
  averages of the exact solution over each cell (warp_sod_validation.py:183-210);
* runs: WENO5-JS ("classical") and WENO5-SR with the checkpoint's closure in FP32 (the reference's
  "mlp_float32_state_float64") or FP64, characteristic reconstruction, HLLC (the reference's monitor uses its 2D
  EVILIN interface state, which this package's 2D path does not provide; the flux is a parameter);
* record: the reference's metric keys (density rows averaged over the transverse direction; L1 = mean |e|,
  L2 = rms, Linf = max; gains of the closure over JS against the exact solution, absolute and relative; failure
  flags), written to circle_validation_metrics.csv / .npz in the run directory (the reference's file names).

`monitor` is the sidecar loop (poll the run directory, evaluate new checkpoints, stop at max_step);
`train1d.train(..., TrainConfig(sod_monitor_interval=K))` evaluates inline every K training steps.
"""
from __future__ import annotations

import csv
import re
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import euler2d as E
from . import riemann as R
from .checkpoint import load_mlp_params
from .params import Params

STEP_PATTERN = re.compile(r"model_step_(\d+)\.npz$")
SOD_LEFT = (1.0, 0.0, 1.0)
SOD_RIGHT = (0.125, 0.0, 0.1)
METRICS_STEM = "circle_validation_metrics"


@dataclass(frozen=True)
class SodMonitorConfig:
    nx: int = 100
    ny: int = 10
    cfl: float = 0.4
    t_end: float = 0.25
    axis: str = "x"
    flux: str = "hllc"
    precision: str = "sr_f32"  # closure precision of the MLP run: "sr_f32" or "sr_f64"
    gamma: float = 1.4

    def params(self) -> Params:
        """The tube has unit length along `axis` and square cells (for axis "y" the transpose of the x tube)."""
        if self.axis == "y":
            return Params(nx=self.nx, ny=self.ny, x_length=self.nx / float(self.ny), y_length=1.0, cfl=self.cfl,
                          t_end=self.t_end, gamma=self.gamma)
        return Params(nx=self.nx, ny=self.ny, x_length=1.0, y_length=self.ny / float(self.nx), cfl=self.cfl,
                      t_end=self.t_end, gamma=self.gamma)


def exact_state(cfg: SodMonitorConfig, t: float) -> np.ndarray:
    """Padded [ny+6][nx+6][4] cell averages of the exact Sod solution at time t (ghost cells included)."""
    p = cfg.params()
    g = p.ghost
    if cfg.axis == "y":
        h, n_along, n_across = p.dy, p.ny, p.nx
        start = -0.5 * p.y_length
    else:
        h, n_along, n_across = p.dx, p.nx, p.ny
        start = -0.5 * p.x_length
    centers = start + (np.arange(n_along + 2 * g) - g + 0.5) * h
    line = R.cell_averages(centers, h, t, 0.0, SOD_LEFT, SOD_RIGHT, cfg.gamma, quadrature=15, split=False)
    if cfg.axis == "y":  # the momentum of the tube goes in the y slot
        line = line[:, [0, 2, 1, 3]]
        return np.ascontiguousarray(np.broadcast_to(line[:, None, :], (n_along + 2 * g, n_across + 2 * g, 4)))
    return np.ascontiguousarray(np.broadcast_to(line[None, :, :], (n_across + 2 * g, n_along + 2 * g, 4)))


def density_row(u: np.ndarray, cfg: SodMonitorConfig) -> np.ndarray:
    """Interior density averaged over the direction across the tube."""
    p = cfg.params()
    g = p.ghost
    rho = np.asarray(u)[g:g + p.ny, g:g + p.nx, 0]
    return rho.mean(axis=1) if cfg.axis == "y" else rho.mean(axis=0)


def row_metrics(row: np.ndarray, reference: np.ndarray) -> tuple[float, float, float]:
    diff = np.asarray(row) - np.asarray(reference)
    if not np.all(np.isfinite(diff)):
        return float("nan"), float("nan"), float("nan")
    return float(np.mean(np.abs(diff))), float(np.sqrt(np.mean(diff * diff))), float(np.max(np.abs(diff)))


def _interior_stats(u: np.ndarray, p: Params) -> dict:
    g = p.ghost
    q = np.asarray(u)[g:g + p.ny, g:g + p.nx]
    rho = q[..., 0]
    with np.errstate(all="ignore"):
        vel2 = (q[..., 1] ** 2 + q[..., 2] ** 2) / rho ** 2
        prs = (p.gamma - 1.0) * (q[..., 3] - 0.5 * rho * vel2)
    return {"rho_min": float(np.nanmin(rho)), "rho_max": float(np.nanmax(rho)), "p_min": float(np.nanmin(prs)),
            "nan_count": float(np.isnan(q).sum()), "rho_neg": float(np.sum(rho <= 0.0)),
            "p_neg": float(np.sum(prs <= 0.0))}


def _advance(u0: np.ndarray, cfg: SodMonitorConfig, method: str, mlp, device) -> tuple:
    """(final state, t, steps, dts, failed): the device time loop to t_end with the health check after every
    step (a non-finite or non-positive dt, NaN or non-positive density/pressure stops the run)."""
    p = cfg.params()
    dev = torch.device(device)
    bufs = [torch.as_tensor(u0, device=dev).clone()] + [torch.zeros(p.padded_shape, dtype=torch.float64,
                                                                    device=dev) for _ in range(3)]
    res = E.run(bufs, p, cfg.t_end, method, "transmissive", mlp_params=mlp, flux=cfg.flux, check_health=True,
                check_interval=1)
    u = bufs[res.final_slot].cpu().numpy()
    st = _interior_stats(u, p)
    failed = (abs(res.t - cfg.t_end) > 1.0e-12) or bool(st["nan_count"] or st["rho_neg"] or st["p_neg"])
    return u, res.t, res.steps, res.dts, failed


def _dt_stats(dts, prefix: str) -> dict:
    d = np.asarray(dts, dtype=np.float64)
    return {f"{prefix}dt_min": float(d.min()) if d.size else 0.0, f"{prefix}dt_max": float(d.max()) if d.size else 0.0,
            f"{prefix}dt_mean": float(d.mean()) if d.size else 0.0}


def evaluate_checkpoint(checkpoint, step: int, cfg: SodMonitorConfig = SodMonitorConfig(), device="cuda",
                        out_dir: Path | None = None) -> dict:
    """One monitor record for a checkpoint (a reference-format .npz path or a {w1..b4} dict of arrays)."""
    if cfg.precision not in ("sr_f32", "sr_f64"):
        raise ValueError(f"monitor precision must be 'sr_f32' or 'sr_f64', got {cfg.precision!r}")
    if cfg.axis not in ("x", "y"):
        raise ValueError(f"axis must be 'x' or 'y', got {cfg.axis!r}")
    mlp = load_mlp_params(checkpoint, "cpu") if isinstance(checkpoint, (str, Path)) else checkpoint
    mlp = {k: np.asarray(v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else v, dtype=np.float64)
           for k, v in mlp.items() if k != "meta_json"}
    p = cfg.params()
    u0 = exact_state(cfg, 0.0)
    ref_row = density_row(exact_state(cfg, cfg.t_end), cfg)
    u_c, t_c, n_c, dts_c, fail_c = _advance(u0, cfg, "js", None, device)
    u_m, t_m, n_m, dts_m, fail_m = _advance(u0, cfg, cfg.precision, mlp, device)
    rho_c, rho_m = density_row(u_c, cfg), density_row(u_m, cfg)
    full_mlp = (not fail_m) and abs(t_m - cfg.t_end) < 1.0e-12
    same_time = full_mlp and (not fail_c) and abs(t_c - t_m) < 1.0e-12
    d_l1, d_l2, d_linf = row_metrics(rho_m, rho_c) if same_time else (float("nan"),) * 3
    c_l1, c_l2, c_linf = row_metrics(rho_c, ref_row)
    m_l1, m_l2, m_linf = row_metrics(rho_m, ref_row) if full_mlp else (float("nan"),) * 3
    gains = {}
    for name, c, m in (("l1", c_l1, m_l1), ("l2", c_l2, m_l2), ("linf", c_linf, m_linf)):
        gains[f"gain_vs_reference_{name}"] = c - m
        gains[f"rel_gain_vs_reference_{name}"] = (c - m) / max(c, 1.0e-300)
    sc, sm = _interior_stats(u_c, p), _interior_stats(u_m, p)
    half = 0.5 * (p.y_length if cfg.axis == "y" else p.x_length)
    record = {
        "raw_step": int(step), "step": int(step),
        "validation_kind": "weno5-sod-2d-b200-" + ("sr-float32" if cfg.precision == "sr_f32" else "sr-float64"),
        "mlp_forward": "0.5*(M(x)+P*M(Px))",
        "precision": "mlp_float32_state_float64" if cfg.precision == "sr_f32" else "mlp_float64_state_float64",
        "axis": cfg.axis, "riemann_solver": cfg.flux, "weno_space": "characteristic",
        "x_min": -half, "x_max": half, "dx": p.dx, "dy": p.dy,
        "t": t_m, "steps": n_m, "classical_t": t_c, "classical_steps": n_c, "mlp_t": t_m, "mlp_steps": n_m,
        **_dt_stats(dts_m, ""), **_dt_stats(dts_c, "classical_"),
        "rho_diff_l1": d_l1, "rho_diff_l2": d_l2, "rho_diff_linf": d_linf,
        "reference_nx": float(p.nx), "reference_ny": float(p.ny), "reference_steps": 0.0,
        "classical_vs_reference_l1": c_l1, "classical_vs_reference_l2": c_l2, "classical_vs_reference_linf": c_linf,
        "mlp_vs_reference_l1": m_l1, "mlp_vs_reference_l2": m_l2, "mlp_vs_reference_linf": m_linf, **gains,
        "classical_rho_min": sc["rho_min"], "classical_rho_max": sc["rho_max"], "classical_p_min": sc["p_min"],
        "mlp_rho_min": sm["rho_min"], "mlp_rho_max": sm["rho_max"], "mlp_p_min": sm["p_min"],
        "mlp_nan_count": sm["nan_count"], "mlp_rho_neg": sm["rho_neg"], "mlp_p_neg": sm["p_neg"],
        "failed": float(fail_c or fail_m),
    }
    if out_dir is not None:  # the density rows of this checkpoint (the reference plots them)
        step_dir = Path(out_dir) / "circle_validation" / f"step_{int(step):06d}"
        step_dir.mkdir(parents=True, exist_ok=True)
        h = p.dy if cfg.axis == "y" else p.dx
        n = p.ny if cfg.axis == "y" else p.nx
        np.savez(step_dir / "sod_density.npz", x=-half + (np.arange(n) + 0.5) * h, exact=ref_row, classical=rho_c,
                 mlp=rho_m)
        record["plot_dir"] = str(step_dir)
    return record


def ready_checkpoints(run_dir: Path, interval: int) -> list[tuple[int, Path]]:
    """(step, path) of the run's checkpoints whose step is a positive multiple of `interval`, by step."""
    ready = []
    for path in (Path(run_dir) / "checkpoints").glob("model_step_*.npz"):
        m = STEP_PATTERN.match(path.name)
        if m is None:
            continue
        step = int(m.group(1))
        if step > 0 and step % interval == 0:
            ready.append((step, path))
    return sorted(ready)


def load_records(run_dir: Path) -> dict[int, dict]:
    path = Path(run_dir) / f"{METRICS_STEM}.npz"
    if not path.is_file():
        return {}
    with np.load(path, allow_pickle=True) as data:
        return {int(r["raw_step"]): r for r in data["records"].tolist()}


def write_records(run_dir: Path, records: list[dict]) -> None:
    """The records, by step, as CSV and as an object array in .npz (rewritten whole each time)."""
    if not records:
        return
    run_dir = Path(run_dir)
    run_dir.mkdir(parents=True, exist_ok=True)
    fields = []
    for r in records:
        fields += [k for k in r if k not in fields]
    with (run_dir / f"{METRICS_STEM}.csv").open("w", newline="", encoding="utf-8") as f:
        w = csv.DictWriter(f, fieldnames=fields, extrasaction="ignore")
        w.writeheader()
        w.writerows(records)
    np.savez(run_dir / f"{METRICS_STEM}.npz", records=np.array(records, dtype=object))


def record_checkpoint(run_dir: Path, checkpoint: Path, step: int, cfg: SodMonitorConfig, device="cuda") -> dict:
    """Evaluate one checkpoint and add its record to the run directory's metrics (replacing a record of the
    same step)."""
    records = load_records(run_dir)
    rec = evaluate_checkpoint(checkpoint, step, cfg, device, out_dir=run_dir)
    records[int(step)] = rec
    write_records(run_dir, [records[k] for k in sorted(records)])
    return rec


def monitor(run_dir: Path, interval: int = 250, max_step: int = 200000, poll_seconds: float = 10.0,
            cfg: SodMonitorConfig = SodMonitorConfig(), device="cuda", once: bool = False) -> dict[int, dict]:
    """The sidecar loop: evaluate every ready checkpoint not yet recorded, then poll; returns the records when
    the checkpoint of max_step has been recorded (or after one pass with once=True). A checkpoint that fails to
    load or run is retried on the next poll."""
    if interval <= 0 or poll_seconds <= 0:
        raise ValueError("interval and poll_seconds must be positive")
    run_dir = Path(run_dir)
    if not run_dir.is_dir():
        raise FileNotFoundError(run_dir)
    records = load_records(run_dir)
    print(f"sod_monitor_start run={run_dir} interval={interval} grid={cfg.nx}x{cfg.ny} cfl={cfg.cfl} "
          f"t_end={cfg.t_end} space=characteristic solver={cfg.flux} existing={len(records)} "
          f"precision={cfg.precision}", flush=True)
    while True:
        for step, path in [x for x in ready_checkpoints(run_dir, interval) if x[0] not in records]:
            print(f"SOD_START step={step:06d} checkpoint={path}", flush=True)
            try:
                rec = evaluate_checkpoint(path, step, cfg, device, out_dir=run_dir)
            except (OSError, ValueError, RuntimeError) as err:
                print(f"SOD_RETRY step={step:06d} error={type(err).__name__}: {err}", flush=True)
                break
            records[step] = rec
            write_records(run_dir, [records[k] for k in sorted(records)])
            print(f"SOD_DONE step={step:06d} gain_L2={100.0 * rec['rel_gain_vs_reference_l2']:.2f}% "
                  f"failed={int(rec['failed'])}", flush=True)
        if once:
            return records
        if max_step in records:
            print(f"sod_monitor_complete step={max_step:06d}", flush=True)
            return records
        time.sleep(poll_seconds)
