"""Pin the numpy 1D oracle to the reference's torch steppers (fixtures from tests/golden/make_golden_1d.py)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import adv1d_oracle as A
from oracle.oracle import pack_params

G = Path(__file__).resolve().parent / "golden"
M = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
P64 = pack_params(dict(np.load(M / "weno5_sr_fp64_step012250.npz")))
P32 = pack_params(dict(np.load(M / "weno5_sr_fp32_step016500.npz")))
P7 = pack_params(dict(np.load(M / "weno7_sr_fp64_step016750.npz")))
W5 = {"js": None, "sr_f64": (5, "f64", P64), "sr_f32": (5, "f32", P32)}
W7 = {"js": None, "sr_f64": (7, "f64", P7)}
TOL = {"js": 0.0, "sr_f64": 2e-15, "sr_f32": 1e-8}
PUBLISHED_GSTE_L1 = {  # experiments/01_gste_long_time_advection/tables/gste_metrics.csv
    "weno5_js": 0.04976537479001931, "weno5_sr_f64": 0.03756399031896309,
    "weno7_js": 0.029739185322686722, "weno7_sr_f64": 0.02341602561621716,
}


@pytest.mark.parametrize("case,n", [(0, 37), (1, 64), (2, 100)])
@pytest.mark.parametrize("key", ["js", "sr_f64", "sr_f32"])
def test_weno5_ssprk3_matches_reference(case, n, key):
    g = np.load(G / "adv1d_steps.npz")
    u0, dx = g[f"c{case}_u0"], 1.0 / n
    for b, a in enumerate((1.0, -1.0)):
        out = A.run(u0[b], a, dx, [0.5 * dx] * 3, 5, W5[key], "ssprk3")
        assert np.abs(out - g[f"c{case}_w5_{key}_3steps"][b]).max() <= TOL[key]
        out = A.run(u0[b], a, dx, [s * dx for s in A.cfl_schedule(2.3, 0.5)], 5, W5[key], "ssprk3")
        assert np.abs(out - g[f"c{case}_w5_{key}_dist"][b]).max() <= TOL[key]


@pytest.mark.parametrize("case,n", [(0, 37), (1, 64), (2, 100)])
@pytest.mark.parametrize("key", ["js", "sr_f64"])
def test_weno7_shu_rk4_matches_reference(case, n, key):
    g = np.load(G / "adv1d_steps.npz")
    u0, dx = g[f"c{case}_u0"], 1.0 / n
    for b, a in enumerate((1.0, -1.0)):
        out = A.run(u0[b], a, dx, [0.5 * dx] * 3, 7, W7[key], "shu_rk4")
        assert np.abs(out - g[f"c{case}_w7_{key}_3steps"][b]).max() <= TOL[key]


def test_gste_fixture_reproduces_published_table():
    g = np.load(G / "gste.npz")
    for key, l1 in PUBLISHED_GSTE_L1.items():
        assert abs(float(g[f"{key}_l1"]) - l1) <= 1e-14
        assert abs(np.mean(np.abs(g[f"{key}_final"] - g["exact"])) - l1) <= 1e-14


def test_gste_weno5_js_oracle_matches_reference_final_state():
    g = np.load(G / "gste.npz")
    steps = int(g["weno5_js_steps"])
    dx = 2.0 / 200
    dt = 10.0 / steps
    out = A.run(g["initial"], 1.0, dx, [dt] * steps, 5, None, "ssprk3")
    assert np.abs(out - g["weno5_js_final"]).max() <= 1e-12


def test_shard_by_cost_partitions_and_balances():
    from weno_sr_publishing_b200 import adv1d as A1

    rng = np.random.default_rng(4)
    cost = rng.integers(100, 1001, 4096 * 3) * 2 * rng.choice([2, 8, 64, 128, 256, 512, 1024], 4096 * 3)
    for world in (1, 2, 3, 8):
        parts = [A1.shard_by_cost(cost, world, r) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        np.testing.assert_array_equal(allidx, np.arange(cost.size))
        loads = np.array([cost[p].sum() for p in parts])
        assert loads.max() - loads.min() <= cost.max()
        np.testing.assert_array_equal(parts[0], A1.shard_by_cost(cost, world, 0))  # deterministic
    with pytest.raises(ValueError):
        A1.shard_by_cost(cost, 2, 2)


# WENO-Z rows of the paper's GSTE table (N=200, t=10, CFL 0.6), weno_z_borges_p2_results/README.md
PUBLISHED_GSTE_Z_L1 = {"weno5_z": 4.198206e-2, "weno7_z": 2.928891e-2}


def test_gste_z_fixture_reproduces_published_table():
    g = np.load(G / "adv1d_z.npz")
    for key, l1 in PUBLISHED_GSTE_Z_L1.items():
        assert abs(float(g[f"{key}_l1"]) - l1) <= 5e-9  # the table prints 7 significant digits
        assert abs(np.mean(np.abs(g[f"{key}_final"] - g["exact"])) - float(g[f"{key}_l1"])) <= 1e-15


@pytest.mark.parametrize("case,n", [(0, 37), (1, 64), (2, 100)])
@pytest.mark.parametrize("scheme,integ,key", [(5, "ssprk3", "w5"), (7, "shu_rk4", "w7")])
def test_weno_z_matches_reference(case, n, scheme, integ, key):
    g = np.load(G / "adv1d_z.npz")
    u0, dx = g[f"c{case}_u0"], 1.0 / n
    for b in range(u0.shape[0]):
        out = A.run(u0[b], 1.0, dx, [0.5 * dx] * 3, scheme, "z", integ)
        ref = g[f"c{case}_{key}_3steps"][b]
        # the reference sums the three or four alphas with torch.sum and takes h = 1 / (1 / dx)
        assert np.abs(out - ref).max() <= 1e-14 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("scheme,integ", [(5, "ssprk3"), (7, "shu_rk4")])
def test_gste_z_oracle_matches_reference_final_state(scheme, integ):
    g = np.load(G / "adv1d_z.npz")
    key = f"weno{scheme}_z"
    steps, dt = int(g[f"{key}_steps"]), float(g[f"{key}_dt"])
    out = A.run(g["initial"], 1.0, 2.0 / 200, [dt] * steps, scheme, "z", integ)
    assert np.abs(out - g[f"{key}_final"]).max() <= 1e-11
