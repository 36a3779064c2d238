"""Shock tubes through the CUDA 2D path (nx x 10 grids, transmissive) against exact Riemann solutions:
the reference's published Sod and Lax error tables (experiments/02_sod_shock_tube/tables/sod_metrics.csv,
experiments/03_lax_shock_tube/tables/lax_metrics.csv) reproduced digit for digit."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from weno_sr_publishing_b200 import riemann as R

pytestmark = pytest.mark.gpu

M = Path(__file__).resolve().parents[1] / "weno_sr_publishing_b200" / "models"
P64 = {k: v for k, v in np.load(M / "weno5_sr_fp64_step012250.npz").items() if k != "meta_json"}
P32 = {k: v for k, v in np.load(M / "weno5_sr_fp32_step016500.npz").items() if k != "meta_json"}
PARAMS = {"js": None, "z": None, "sr_f64": P64, "sr_f32": P32}
DEV = "cuda:0"
# relative tolerance against the published 16-digit values: the FP64 paths reproduce the reference's GPU
# run to rounding; the FP32 closure differs from it in the last float bits of exp/tanh
TOL = {"js": 1e-9, "z": 1e-9, "sr_f64": 1e-9, "sr_f32": 1e-4}

# (rho L1, rho L2, rho Linf) at N = 100, CFL 0.8, t = 0.2
SOD = {
    "js": (0.004969788355086182, 0.010231427744136113, 0.051714576051554495),
    "z": (0.004495033825294024, 0.009396942104484428, 0.04742549657693956),
    "sr_f64": (0.0038059560464159797, 0.007958549368864762, 0.03940045209093579),
    "sr_f32": (0.0038867036160611253, 0.008127901599424399, 0.039988391625698116),
}
# (L1, L2, Linf) of rho, velocity and pressure at N = 200, CFL 0.8, t = 1.3
LAX = {
    "js": ((0.00677337105849069, 0.033646180475622185, 0.3461942611056521),
           (0.005427914253574433, 0.02396824363986733, 0.30784890245086466),
           (0.006548192025839354, 0.02328848571962226, 0.21385620898704893)),
    "z": ((0.005399423435389255, 0.028742561613860573, 0.3155316586396848),
          (0.004801859511601044, 0.019020827456441274, 0.23474731756157174),
          (0.005848033894982103, 0.018161069642420966, 0.158749460783004)),
    "sr_f64": ((0.004854836515529101, 0.027114703386362016, 0.31171828742193375),
               (0.0033738175773912727, 0.014235096584539465, 0.18399202496698255),
               (0.004221069331847009, 0.013449019807735952, 0.12206487964216739)),
    "sr_f32": ((0.004855994352603844, 0.026922867941882953, 0.3083570523713782),
               (0.0035875358647294163, 0.014833925658601366, 0.19006372493245763),
               (0.004465134225500693, 0.014237412810373724, 0.12564315641828572)),
}


def _close(got, ref, tol):
    return abs(got / ref - 1.0) <= tol


@pytest.mark.parametrize("method", ["js", "z", "sr_f64", "sr_f32"])
def test_sod_table(method):
    r = R.shock_tube_run(R.SOD, method, PARAMS[method], DEV)
    assert r["t"] == pytest.approx(0.2, abs=1e-14)
    got = (r["rho_l1_mean"], r["rho_l2"], r["rho_linf"])
    for g, ref in zip(got, SOD[method]):
        assert _close(g, ref, TOL[method]), (method, got, SOD[method])


@pytest.mark.parametrize("method", ["js", "z", "sr_f64", "sr_f32"])
def test_lax_table(method):
    r = R.shock_tube_run(R.LAX, method, PARAMS[method], DEV)
    assert r["t"] == pytest.approx(1.3, abs=1e-14)
    for field, ref in zip(("rho", "velocity", "pressure"), LAX[method]):
        got = (r[f"{field}_l1_mean"], r[f"{field}_l2"], r[f"{field}_linf"])
        for g, rv in zip(got, ref):
            assert _close(g, rv, TOL[method]), (method, field, got, ref)
        assert r[f"{field}_l1_integral"] == pytest.approx(10.0 * r[f"{field}_l1_mean"], rel=1e-12)


# rho L1 at N = 1001 (experiments/04_titarev_toro/tables/titarev_toro_N1001_metrics.csv)
TT1001 = {"js": 0.045817915309323325, "z": 0.03666952543273437, "sr_f64": 0.016817740885314403,
          "sr_f32": 0.01960565024853782}


def test_titarev_toro_against_fine_js_run():
    """Titarev-Toro at N = 1001 against a WENO5-JS N = 10001 run interpolated to the mesh. Every method
    finishes, the ordering of the reference's table holds, and the errors agree with the table to within
    the uncertainty of its fine-grid run (whose script and settings the reference does not ship: the FP64
    methods land 0.3% below the table, consistently across methods)."""
    ref = R.titarev_toro_run(10001, "js", device=DEV)
    assert ref["t"] == pytest.approx(5.0, abs=1e-12)
    err = {m: R.titarev_toro_errors(R.titarev_toro_run(1001, m, PARAMS[m], DEV), ref)["rho_l1"]
           for m in ("js", "z", "sr_f64", "sr_f32")}
    assert all(np.isfinite(v) for v in err.values())
    assert err["sr_f64"] < err["sr_f32"] < err["z"] < err["js"], err
    for m, v in err.items():
        assert _close(v, TT1001[m], 0.01 if m != "sr_f32" else 0.03), (m, v, TT1001[m])
