"""CPU: the Sod monitor's host logic (exact initial/final states, checkpoint discovery, record files, argument
errors); the GPU runs are in test_gpu_sod_monitor.py."""
from __future__ import annotations

import numpy as np
import pytest

from weno_sr_publishing_b200 import sod_monitor as SM


def test_exact_states_follow_the_tube():
    cfg = SM.SodMonitorConfig()
    u0 = SM.exact_state(cfg, 0.0)
    assert u0.shape == (cfg.ny + 6, cfg.nx + 6, 4)
    row = SM.density_row(u0, cfg)
    assert row[: cfg.nx // 2].max() == 1.0 and row[cfg.nx // 2:].max() == 0.125  # interface on a cell edge
    uy = SM.exact_state(SM.SodMonitorConfig(axis="y", nx=10, ny=100), 0.1)
    ux = SM.exact_state(cfg, 0.1)
    np.testing.assert_array_equal(uy[:, :, 0].T, ux[:, :, 0])
    np.testing.assert_array_equal(uy[:, :, 2].T, ux[:, :, 1])  # the tube's momentum in the y slot
    mass = SM.density_row(ux, cfg).sum() * cfg.params().dx
    # the waves stay inside the tube at t = 0.1 (15-point averages of discontinuous cells are not exactly conservative)
    assert mass == pytest.approx(0.5 * (1.0 + 0.125), rel=1e-4)


def test_ready_checkpoints_and_record_files(tmp_path):
    (tmp_path / "checkpoints").mkdir()
    for s in (0, 5, 10, 15, 20):
        (tmp_path / "checkpoints" / f"model_step_{s:06d}.npz").write_bytes(b"")
    (tmp_path / "checkpoints" / "other.npz").write_bytes(b"")
    assert [s for s, _ in SM.ready_checkpoints(tmp_path, 10)] == [10, 20]
    recs = [{"raw_step": 10, "step": 10, "gain": 0.5}, {"raw_step": 20, "step": 20, "gain": float("nan"),
                                                        "extra": 1.0}]
    SM.write_records(tmp_path, recs)
    back = SM.load_records(tmp_path)
    assert sorted(back) == [10, 20] and back[10]["gain"] == 0.5 and np.isnan(back[20]["gain"])
    header = (tmp_path / "circle_validation_metrics.csv").read_text().splitlines()[0]
    assert header == "raw_step,step,gain,extra"


def test_argument_errors(tmp_path):
    with pytest.raises(ValueError):
        SM.monitor(tmp_path, interval=0)
    with pytest.raises(FileNotFoundError):
        SM.monitor(tmp_path / "missing", interval=10)
    with pytest.raises(ValueError):
        SM.evaluate_checkpoint({}, 1, SM.SodMonitorConfig(precision="sr_bf16"))
