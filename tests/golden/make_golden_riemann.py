"""Generate tests/golden/riemann_exact.npz from the reference's exact Riemann code and shock-tube setups.

Run in a container that holds the reference checkout (never needed at test time):

    python tests/golden/make_golden_riemann.py --reference /path/to/WENO_SR_publishing

Stores: the star states and wave speeds of Sod and Lax (for_paper_results/exact_riemann.py), pointwise
samples, the exact cell averages used by the published Sod (unsplit 15-point Gauss,
weno_z_borges_p2_results/run_riemann_1d.py:45-63, whose pointwise sampler lives in a module the reference
does not ship, so the shipped exact sampler stands in) and Lax (split, for_paper_results/exact_riemann.py) error
tables, and the initial states of the Sod (teacherfree_lab_weno5/warp_sod_validation.py), Lax
(for_paper_results/run_shock_tube_benchmark.py) and Titarev-Toro (for_paper_results/run_weno5_titarev_toro.py)
runs.
"""
from __future__ import annotations

import argparse
import importlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import warp_shim  # noqa: E402

SOD = ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
LAX = ((0.445, 0.698, 3.528), (0.5, 0.0, 0.571))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    warp_shim.install()
    snap = args.reference / "code" / "snapshot"
    sys.path.insert(0, str(snap))
    er = importlib.import_module("for_paper_results.exact_riemann")
    stb = importlib.import_module("for_paper_results.run_shock_tube_benchmark")
    ttr = importlib.import_module("for_paper_results.run_weno5_titarev_toro")
    sod5 = importlib.import_module("teacherfree_lab_weno5.warp_sod_validation")
    wh = importlib.import_module("warp_weno5_helpers")
    out = {}
    for name, (left, right) in (("sod", SOD), ("lax", LAX)):
        out[f"{name}_star"] = np.array(er.solve_star(left, right, 1.4))
        out[f"{name}_speeds"] = np.array(er.wave_speeds(left, right, 1.4))
        xi = np.linspace(-3.0, 3.0, 241)
        out[f"{name}_xi"] = xi
        out[f"{name}_sample"] = np.array([er.sample_similarity(float(v), left, right, 1.4) for v in xi])
    # Sod table: N = 100 on [0, 1], x0 = 0.5, t = 0.2, unsplit Gauss-15
    dx = 0.01
    x = (np.arange(100) + 0.5) * dx
    # run_riemann_1d.sod_cell_average_conserved samples train_weno5_mlp.sample_riemann_primitive, a module the
    # reference does not ship; the same unsplit Gauss-15 average is formed here with the shipped exact sampler
    nodes, weights = np.polynomial.legendre.leggauss(15)
    acc = np.zeros((x.size, 4))
    for node, weight in zip(nodes, weights):
        for i, xq in enumerate(x + 0.5 * dx * float(node) - 0.5):
            rho, vel, prs = er.sample_similarity(float(xq) / 0.2, SOD[0], SOD[1], 1.4)
            acc[i] += 0.5 * float(weight) * np.array([rho, rho * vel, 0.0, prs / 0.4 + 0.5 * rho * vel * vel])
    out["sod_exact_t02"] = acc
    # Lax table: N = 200 on [-5, 5], x0 = 0, t = 1.3, split (default 20-point and 15-point rules)
    dx = 0.05
    x = -5.0 + (np.arange(200) + 0.5) * dx
    out["lax_exact_t13_q20"] = er.cell_average_conserved(x, dx, 1.3, 0.0, LAX[0], LAX[1])
    out["lax_exact_t13_q15"] = er.cell_average_conserved(x, dx, 1.3, 0.0, LAX[0], LAX[1], quadrature=15)
    # initial states
    p = wh.Params(nx=100, ny=10, x_length=1.0, y_length=0.1, cfl=0.8, t_end=0.2)
    out["sod_initial"] = sod5.make_exact_sod_state(p, 0.0, "x")
    p = wh.Params(nx=200, ny=10, x_length=10.0, y_length=0.5, cfl=0.8, t_end=1.3)
    out["lax_initial"] = stb.make_initial_state(p, stb.BENCHMARKS["lax"])
    for n in (1001, 2000):
        p = wh.Params(nx=n, ny=10, x_length=10.0, y_length=10 * 10.0 / n, cfl=0.8, t_end=5.0)
        out[f"tt_initial_{n}"] = ttr.make_initial_state(p, -5.0, 5.0)
    np.savez_compressed(HERE / "riemann_exact.npz", **out)
    print("riemann_exact.npz written", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
