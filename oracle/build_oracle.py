"""Build the CPU oracle shared library (test infrastructure; see euler2d_oracle.c and euler3d_oracle.c).

Two builds are produced from the same sources:

* ``liboracle.so``        -O2 -ffp-contract=off: deterministic IEEE evaluation, used as the checker.
* ``liboracle_fast.so``   -O3 (portable x86-64, runs on any host that loads it), OpenMP: the timed CPU baseline in bench.py.

Usage: python oracle/build_oracle.py
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = ["euler2d_oracle.c", "euler3d_oracle.c"]


def _cc(out: Path, flags: list[str]) -> None:
    srcs = [str(HERE / s) for s in SOURCES]
    cmd = ["gcc", "-std=c11", "-shared", "-fPIC", "-fopenmp", *flags, "-o", str(out), *srcs, "-lm"]
    subprocess.run(cmd, check=True)


def build(force: bool = False) -> list[Path]:
    outs = [(HERE / "liboracle.so", ["-O2", "-ffp-contract=off"]),
            (HERE / "liboracle_fast.so", ["-O3", "-fno-math-errno"])]
    built = []
    newest_src = max(os.path.getmtime(HERE / s) for s in SOURCES)
    for out, flags in outs:
        if force or not out.exists() or os.path.getmtime(out) < newest_src:
            _cc(out, flags)
        built.append(out)
    return built


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv):
        print(p)
