"""GPU: the Sod checkpoint monitor (sod_monitor.py) through this package's 2D kernels: records written during a
short training run equal a direct evaluation of the same checkpoints, the sidecar loop reproduces them, the shipped
FP32 closure beats WENO5-JS on the monitor's Sod problem (as in the reference's Sod table), and the x and y
orientations of the tube agree."""
from __future__ import annotations

import math

import pytest

from weno_sr_publishing_b200 import sod_monitor as SM
from weno_sr_publishing_b200 import train1d as T
from weno_sr_publishing_b200.checkpoint import MODELS_DIR

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _same(a: dict, b: dict) -> None:
    assert set(a) == set(b)
    for k in a:
        if isinstance(a[k], float) and math.isnan(a[k]):
            assert math.isnan(b[k]), k
        else:
            assert a[k] == b[k], (k, a[k], b[k])


def test_training_run_records_match_direct_evaluation(tmp_path):
    cfg = T.TrainConfig(out_dir=tmp_path / "run", steps=20, grid=32, batch=16, distances=(2, 8), precision="f32",
                        lr=1e-3, lr_final=2e-4, log_interval=10, checkpoint_interval=20, state_interval=1000,
                        device=DEV, sod_monitor_interval=10)
    T.train(cfg)
    run = tmp_path / "run"
    recs = SM.load_records(run)
    assert sorted(recs) == [10, 20]
    assert (run / "circle_validation_metrics.csv").read_text().count("\n") == 3
    for step in (10, 20):
        ck = run / "checkpoints" / f"model_step_{step:06d}.npz"
        direct = SM.evaluate_checkpoint(ck, step, SM.SodMonitorConfig(), DEV, out_dir=run)
        _same(recs[step], direct)
        # a closure after a few training steps may fail on Sod (the record says so, as the reference's does)
        assert recs[step]["classical_t"] == pytest.approx(0.25, abs=1e-12) and recs[step]["classical_steps"] > 0
    # the sidecar loop finds nothing new, and recomputes the same records from scratch
    again = SM.monitor(run, interval=10, cfg=SM.SodMonitorConfig(), device=DEV, once=True)
    for step in (10, 20):
        _same(again[step], recs[step])
    (run / "circle_validation_metrics.npz").unlink()
    fresh = SM.monitor(run, interval=10, cfg=SM.SodMonitorConfig(), device=DEV, once=True)
    assert sorted(fresh) == [10, 20]
    for step in (10, 20):
        _same(fresh[step], recs[step])


def test_shipped_fp32_closure_beats_js_on_the_monitor_problem():
    rec = SM.evaluate_checkpoint(MODELS_DIR / "weno5_sr_fp32_step016500.npz", 16500, SM.SodMonitorConfig(), DEV)
    assert rec["failed"] == 0.0
    assert 1e-3 < rec["classical_vs_reference_l1"] < 1e-2
    assert rec["rel_gain_vs_reference_l1"] > 0.0 and rec["rel_gain_vs_reference_l2"] > 0.0
    assert rec["rho_diff_l1"] > 0.0 and rec["mlp_steps"] > 0 and rec["classical_steps"] > 0


def test_x_and_y_tubes_agree():
    ck = MODELS_DIR / "weno5_sr_fp32_step016500.npz"
    rx = SM.evaluate_checkpoint(ck, 1, SM.SodMonitorConfig(axis="x"), DEV)
    ry = SM.evaluate_checkpoint(ck, 1, SM.SodMonitorConfig(axis="y", nx=10, ny=100), DEV)
    for k in ("classical_vs_reference_l1", "mlp_vs_reference_l1", "rho_diff_l2"):
        assert rx[k] == pytest.approx(ry[k], rel=1e-9, abs=1e-14), k
    assert rx["mlp_steps"] == ry["mlp_steps"]
