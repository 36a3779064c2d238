"""Build libwsr.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

Usage: python -m weno_sr_publishing_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libwsr.so"
SOURCES = [CSRC / "wsr_api.cu", CSRC / "wsr_api_1d.cu", CSRC / "wsr_api_w7.cu", CSRC / "euler3d.cu"]
# euler3d.cu's main object reproduces the reference's 3D Warp module for WENO5-JS, which is compiled without
# contraction; the same file with WSR_EULER3D_SR_UNIT gives the SR stages, with contraction
EXTRA_FLAGS = {"euler3d.cu": ["-fmad=false"]}
EXTRA_OBJECTS = {"euler3d.cu": [("_euler3d_sr", ["-DWSR_EULER3D_SR_UNIT", "-diag-suppress=177"])]}
HEADERS = sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "wsr.h"]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    raise RuntimeError("nvcc not found")


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile each translation unit (in parallel) and link libwsr.so."""
    if force or stale():
        compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
        objs, procs = [], []
        jobs = []
        for src in SOURCES:
            jobs.append((src, PKG / ("_" + src.stem + ".o"), EXTRA_FLAGS.get(src.name, [])))
            for stem, flags in EXTRA_OBJECTS.get(src.name, []):
                jobs.append((src, PKG / (stem + ".o"), flags))
        for src, obj, flags in jobs:
            cmd = [nvcc(), *compile_flags, *flags, "-c", "-o", str(obj), str(src)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            procs.append(subprocess.Popen(cmd))
            objs.append(obj)
        codes = [p.wait() for p in procs]
        if any(codes):
            raise subprocess.CalledProcessError(max(codes), "nvcc")
        subprocess.run([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(LIB),
                        *map(str, objs)], check=True)
        for obj in objs:
            obj.unlink(missing_ok=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
