"""CPU: the WENO7 2D oracle (Shu RK4, characteristic WENO7, HLLC) against the reference's own solver, bit for bit
(tests/golden/euler2d_w7.npz, written by tests/golden/make_golden_w7.py)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

G = Path(__file__).resolve().parent / "golden" / "euler2d_w7.npz"


@pytest.fixture(scope="module")
def gold():
    if not G.exists():
        pytest.skip("euler2d_w7.npz not generated")
    return np.load(G)


@pytest.mark.parametrize("lr", [1, 2])
def test_face_and_gauss_reconstructions_bitwise(gold, lr):
    np.testing.assert_array_equal(O.w7_face(gold["q"], lr), gold[f"face_lr{lr}"])
    np.testing.assert_array_equal(O.w7_gauss(gold["q"], lr), gold[f"gauss_lr{lr}"])


def _meta(gold, name):
    nx, ny, x0, x1, y0, y1, cfl, t_end = gold[f"{name}_meta"]
    return int(nx), int(ny), (x1 - x0) / nx, (y1 - y0) / ny, float(cfl), float(t_end), str(gold[f"{name}_bc"])


@pytest.mark.parametrize("name", ["vortex", "rough"])
@pytest.mark.parametrize("rev", [0, 1])
def test_rhs_matches_reference(gold, name, rev):
    nx, ny, dx, dy, _, _, bc = _meta(gold, name)
    got = O.w7_rhs(gold[f"{name}_initial"], nx, ny, dx, dy, bc, reverse=rev)
    np.testing.assert_array_equal(got, gold[f"{name}_rhs_rev{rev}"])


@pytest.mark.parametrize("name", ["vortex", "rough"])
def test_run_matches_reference(gold, name):
    nx, ny, dx, dy, cfl, t_end, bc = _meta(gold, name)
    fin, dts, steps, t = O.w7_run(gold[f"{name}_initial"], nx, ny, dx, dy, cfl, t_end, bc)
    assert steps == int(gold[f"{name}_steps"]) and t == float(gold[f"{name}_t"])
    g = 4
    np.testing.assert_array_equal(fin[g:g + ny, g:g + nx], gold[f"{name}_final"][g:g + ny, g:g + nx])


def test_vortex_initial_state_matches_reference(gold):
    from weno_sr_publishing_b200 import problems  # noqa: PLC0415
    np.testing.assert_array_equal(problems.vortex_point_rk4(12, 10, 0.0, 5), gold["vortex_initial"])


# WENO-Z variant of the same path (weno_z_borges_p2_results/weno7_point_rk4_z.py, weight_kind 1)
@pytest.mark.parametrize("hi", [0, 1])
@pytest.mark.parametrize("lr", [1, 2])
def test_z_reconstructions_bitwise(gold, lr, hi):
    h = float(gold["z_h"][hi])
    np.testing.assert_array_equal(O.w7z_face(gold["q"], lr, h), gold[f"z_face_lr{lr}_h{hi}"])
    np.testing.assert_array_equal(O.w7z_gauss(gold["q"], lr, h), gold[f"z_gauss_lr{lr}_h{hi}"])


@pytest.mark.parametrize("name", ["vortex", "rough"])
@pytest.mark.parametrize("rev", [0, 1])
def test_z_rhs_matches_reference(gold, name, rev):
    nx, ny, dx, dy, _, _, bc = _meta(gold, name)
    got = O.w7_rhs(gold[f"{name}_initial"], nx, ny, dx, dy, bc, reverse=rev, method="z")
    np.testing.assert_array_equal(got, gold[f"z_{name}_rhs_rev{rev}"])


@pytest.mark.parametrize("name", ["vortex", "rough"])
def test_z_run_matches_reference(gold, name):
    nx, ny, dx, dy, cfl, t_end, bc = _meta(gold, name)
    fin, dts, steps, t = O.w7_run(gold[f"{name}_initial"], nx, ny, dx, dy, cfl, t_end, bc, method="z")
    assert steps == int(gold[f"z_{name}_steps"]) and t == float(gold[f"z_{name}_t"])
    g = 4
    np.testing.assert_array_equal(fin[g:g + ny, g:g + nx], gold[f"z_{name}_final"][g:g + ny, g:g + nx])
