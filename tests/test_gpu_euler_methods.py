"""GPU: the method registry's WENO7 entries (euler_methods.run_weno7 with the weno7_js / weno7_sr_f64 rows of
config.METHODS, for_paper_results/solvers/euler_methods.py:81-96 and config.py:65-78 of the reference) against
the reference's own WENO7-JS and WENO7-SR solver fixtures, and run_weno5 against the WENO5 adapters."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from weno_sr_publishing_b200 import config
from weno_sr_publishing_b200 import euler_methods as M
from weno_sr_publishing_b200 import problems
from weno_sr_publishing_b200.params import Params
from weno_sr_publishing_b200.solvers import weno5_hllc_mixed

pytestmark = pytest.mark.gpu
G = Path(__file__).resolve().parent / "golden"
DEV = "cuda:0"
# the tolerances of the direct WENO7 solver tests (a few times the reference's own measured conditioning)
TOL = {("weno7_js", "vortex"): 1e-11, ("weno7_js", "rough"): 1e-11,
       ("weno7_sr_f64", "vortex"): 1e-10, ("weno7_sr_f64", "rough"): 1e-12}


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("key,fixture", [("weno7_js", "euler2d_w7.npz"), ("weno7_sr_f64", "euler2d_w7_sr.npz")])
@pytest.mark.parametrize("name", ["vortex", "rough"])
def test_run_weno7_matches_reference_fixtures(key, fixture, name):
    g = np.load(G / fixture)
    nx, ny, x0, x1, y0, y1, cfl, t_end = g[f"{name}_meta"]
    p = M.make_weno7_params(int(nx), int(ny), x0, x1, y0, y1, cfl, t_end)
    final, summary = M.run_weno7(key, g[f"{name}_initial"], p, device=DEV, boundary=str(g[f"{name}_bc"]))
    assert summary["steps"] == int(g[f"{name}_steps"]) and abs(summary["t"] - float(g[f"{name}_t"])) <= 1e-14
    assert _rel(final[4:-4, 4:-4], g[f"{name}_final"][4:-4, 4:-4]) <= TOL[(key, name)]


def test_run_weno7_rejects_other_keys():
    p = M.make_weno7_params(8, 8, -1.0, 1.0, -1.0, 1.0, 0.4, 0.1)
    with pytest.raises(ValueError):
        M.run_weno7("weno5_js", np.zeros(p.padded_shape), p, device=DEV, boundary="periodic")


def test_run_weno5_equals_its_adapter():
    n = 40
    p = Params(nx=n, ny=n, x_length=1.0, y_length=1.0, cfl=0.4, t_end=0.05)
    init = problems.make_quadrant_state(n, n, problems.seeded_quadrant_states(2), 3)
    final, summary = M.run_weno5("weno5_sr_f32", init, p, device=DEV, boundary="transmissive")
    mlp = M.load_mlp_params_f32(config.METHODS["weno5_sr_f32"].model, DEV)
    ref, dts, steps, t = weno5_hllc_mixed.run_to_time(init, p, p.t_end, DEV, mlp, "transmissive")
    assert summary["steps"] == steps and summary["t"] == t
    np.testing.assert_array_equal(final, ref)
