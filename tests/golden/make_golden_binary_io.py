"""Generate tests/golden/step_ref.bin and step_ref_compare.json with the reference's own 3D step writer.

Run in a container that holds the reference checkout (never needed at test time):

    python tests/golden/make_golden_binary_io.py --reference /path/to/WENO_SR_publishing

Writes a seeded primitive array (3 x 4 x 5 cells, time 0.125) with warp_weno5_3d_rk3/binary_io.py::write_step,
and the reference's compare_steps report of that file against a copy with one value moved by one ulp.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    src = args.reference / "code" / "snapshot" / "warp_weno5_3d_rk3" / "binary_io.py"
    spec = importlib.util.spec_from_file_location("ref_binary_io", src)
    bio = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bio)
    rng = np.random.default_rng(20261203)
    prim = rng.uniform(0.1, 2.0, (3, 4, 5, 5))
    bio.write_step(HERE / "step_ref.bin", 0.125, prim)
    moved = prim.copy()
    moved[1, 2, 3, 4] = np.nextafter(moved[1, 2, 3, 4], 10.0)
    tmp = HERE / "_step_moved.bin"
    bio.write_step(tmp, 0.125, moved)
    rep = bio.compare_steps(tmp, HERE / "step_ref.bin")
    tmp.unlink()
    for k in ("candidate", "reference", "candidate_sha256"):
        rep.pop(k)
    (HERE / "step_ref_compare.json").write_text(json.dumps(rep, indent=1, sort_keys=True) + "\n")
    print("step_ref.bin and step_ref_compare.json written")


if __name__ == "__main__":
    main()
