"""Algorithmic work of the 2D WENO5 step, per kernel class, for roofline accounting.

Counting convention: a fused multiply-add is 2 flops; an add, multiply, divide, square root, exp, log or
tanh is 1 flop; comparisons, min/max and abs are 1 flop. The counts are taken from the operation
sequence of the kernels in csrc/ (the reference's arithmetic, with the closure evaluated once per
stencil). The amount of closure work depends on the data: plateau stencils take the linear weights
and skip the MLP, so bench.py counts MLP evaluations and plateau stencils per kernel class on the
device (WSR_OPT_COUNT) and multiplies them by the per-evaluation constants below.

Bytes are the unique HBM bytes each kernel must move (state, face values, fluxes), FP64.
"""
from __future__ import annotations

# MLP 5->10->6->6->3 pair (direct + reflected): per pass 164 FMA (328) + 22 swish x (exp, add, div)
# (66) + 3 x (div, tanh, mul) (9) + softmax (max 2, sub 3, exp 3, add 2, div 1, mul 3 = 14) = 417.
MLP_PAIR_FLOPS = 2 * 417

# FP64 per stencil: sensors 67; features/ratio/beta 28 when the MLP runs; per head: weights 13,
# candidates 15, combination 5 (plateau heads skip the weights).
SENSORS64 = 67
FEATURES64 = 28
HEAD64 = 33
HEAD64_PLATEAU = 20
# JS per stencil: betas and reciprocals 30; per head: weights 11, candidates 15, combination 5.
JS_STENCIL64 = 30
JS_HEAD64 = 31

# Non-closure FP64 per normal-reconstruction face (Roe 60, eigenvectors 24, 6 cells x 4 fields of
# projections 168, two back-projections 50) and per flux face (two HLLC 2 x 90, scaling 12).
NORMAL_FACE64 = 60 + 24 + 168 + 50
FLUX_FACE64 = 2 * 90 + 12
UPDATE_CELL64 = 24

BYTES_PER_CELL = {"normal_x": 96, "normal_y": 96, "flux_x": 96, "flux_y": 96, "update": 160}


def faces(kind: str, nx: int, ny: int) -> int:
    return {"normal_x": (ny + 4) * (nx + 1), "normal_y": (ny + 1) * (nx + 4),
            "flux_x": (nx + 1) * ny, "flux_y": nx * (ny + 1)}[kind]


def kernel_work(kind: str, method: str, nx: int, ny: int, mlp: float = 0, plateau: float = 0) -> dict:
    """Work of ONE launch of kernel class `kind` on an nx x ny grid.

    mlp / plateau: closure tallies of that launch (device counters; 0 for JS)."""
    if kind == "update":
        return {"w32": 0.0, "w64": float(nx * ny * UPDATE_CELL64), "bytes": float(nx * ny * BYTES_PER_CELL[kind])}
    work_faces = faces(kind, nx, ny)
    w32 = w64 = 0.0
    heads = 1 if kind.startswith("normal") else 2
    w64 += work_faces * (NORMAL_FACE64 if kind.startswith("normal") else FLUX_FACE64)
    if method == "js":
        w64 += 8 * work_faces * (JS_STENCIL64 + heads * JS_HEAD64)
    else:
        pairs = mlp * MLP_PAIR_FLOPS
        if method == "sr_f64":
            w64 += pairs
        else:
            w32 += pairs
        w64 += mlp * (SENSORS64 + FEATURES64 + heads * HEAD64) + plateau * (SENSORS64 + heads * HEAD64_PLATEAU)
    return {"w32": float(w32), "w64": float(w64), "bytes": float(nx * ny * BYTES_PER_CELL[kind])}


def bound(work: dict, seconds: float, peak32_tflops: float, peak64_tflops: float, hbm_gbs: float) -> dict:
    """Roofline time = max(W32/peak32, W64/peak64, bytes/BW); frac = roofline time / measured time."""
    t32 = work["w32"] / (peak32_tflops * 1e12)
    t64 = work["w64"] / (peak64_tflops * 1e12)
    tb = work["bytes"] / (hbm_gbs * 1e9)
    kind, t_roof = max((("fp32", t32), ("fp64", t64), ("hbm", tb)), key=lambda kv: kv[1])
    if kind == "hbm":
        achieved, peak, unit = work["bytes"] / seconds / 1e9, hbm_gbs, "GB/s"
    elif kind == "fp32":
        achieved, peak, unit = work["w32"] / seconds / 1e12, peak32_tflops, "TFLOP/s"
    else:
        achieved, peak, unit = work["w64"] / seconds / 1e12, peak64_tflops, "TFLOP/s"
    return {"bound": kind, "achieved": achieved, "peak": peak, "unit": unit, "frac": t_roof / seconds,
            "t_roof_s": t_roof, "t32_s": t32, "t64_s": t64, "thbm_s": tb}
