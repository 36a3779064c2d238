"""CPU: 3D step files against the reference's own writer (tests/golden/step_ref.bin, written by
tests/golden/make_golden_binary_io.py) and the comparison report."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from weno_sr_publishing_b200 import binary_io as B

G = Path(__file__).resolve().parent / "golden"


def _prim():
    return np.random.default_rng(20261203).uniform(0.1, 2.0, (3, 4, 5, 5))


def test_writer_is_byte_identical_to_reference(tmp_path):
    B.write_step(tmp_path / "s.bin", 0.125, _prim())
    assert (tmp_path / "s.bin").read_bytes() == (G / "step_ref.bin").read_bytes()


def test_read_round_trip():
    t, prim = B.read_step(G / "step_ref.bin")
    assert t == 0.125 and prim.shape == (3, 4, 5, 5)
    np.testing.assert_array_equal(prim, _prim())


def test_truncated_and_trailing_files_raise(tmp_path):
    raw = (G / "step_ref.bin").read_bytes()
    for name, data in (("head", raw[:10]), ("body", raw[:-8]), ("tail", raw + b"\0")):
        (tmp_path / name).write_bytes(data)
        with pytest.raises(ValueError):
            B.read_step(tmp_path / name)
    with pytest.raises(ValueError):
        B.write_step(tmp_path / "bad.bin", 0.0, np.zeros((2, 2, 5)))


def test_compare_report_matches_reference(tmp_path):
    moved = _prim()
    moved[1, 2, 3, 4] = np.nextafter(moved[1, 2, 3, 4], 10.0)
    B.write_step(tmp_path / "m.bin", 0.125, moved)
    rep = B.compare_steps(tmp_path / "m.bin", G / "step_ref.bin")
    ref = json.loads((G / "step_ref_compare.json").read_text())
    for k in ("candidate", "reference", "candidate_sha256"):
        rep.pop(k)
    assert json.loads(json.dumps(rep, sort_keys=True)) == ref


def test_primitive_of_padded_state():
    nx, ny, nz = 5, 4, 3
    rng = np.random.default_rng(1)
    rho = rng.uniform(0.5, 2.0, (nz + 6, ny + 6, nx + 6))
    vel = rng.uniform(-1.0, 1.0, (nz + 6, ny + 6, nx + 6, 3))
    p = rng.uniform(0.5, 2.0, (nz + 6, ny + 6, nx + 6))
    q = np.concatenate([rho[..., None], rho[..., None] * vel,
                        (p / 0.4 + 0.5 * rho * (vel * vel).sum(-1))[..., None]], axis=-1)
    prim = B.primitive_interior(q, nx, ny, nz)
    sl = (slice(3, -3),) * 3
    np.testing.assert_allclose(prim[..., 0], rho[sl], rtol=0)
    np.testing.assert_allclose(prim[..., 1:4], vel[sl], rtol=1e-14)
    np.testing.assert_allclose(prim[..., 4], p[sl], rtol=1e-13)
