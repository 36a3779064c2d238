"""Step files of the 3D solver and their comparison (warp_weno5_3d_rk3/binary_io.py).

Format (the C++ code's, little-endian native packing): a 20-byte header ``uint32 nz, ny, nx; float64 time``
followed by ``float64 primitive[nz][ny][nx][5]`` with components (rho, u, v, w, p) of the interior cells.
``read_step`` raises ValueError on a truncated header or payload and on trailing bytes, as the reference does.
"""
from __future__ import annotations

import hashlib
import json
import struct
from pathlib import Path

import numpy as np
import torch

HEADER = struct.Struct("=IIId")
COMPONENT_NAMES = ("rho", "u", "v", "w", "p")
GHOST = 3


def read_step(path: str | Path) -> tuple[float, np.ndarray]:
    path = Path(path)
    with path.open("rb") as stream:
        head = stream.read(HEADER.size)
        if len(head) != HEADER.size:
            raise ValueError(f"truncated step header: {path}")
        nz, ny, nx, time = HEADER.unpack(head)
        count = int(nz) * int(ny) * int(nx) * 5
        values = np.fromfile(stream, dtype=np.float64, count=count)
        extra = stream.read(1)
    if values.size != count:
        raise ValueError(f"truncated payload: expected {count}, got {values.size}")
    if extra:
        raise ValueError(f"unexpected trailing bytes in {path}")
    return float(time), values.reshape((nz, ny, nx, 5))


def write_step(path: str | Path, time: float, primitive: np.ndarray) -> None:
    primitive = np.ascontiguousarray(primitive, dtype=np.float64)
    if primitive.ndim != 4 or primitive.shape[-1] != 5:
        raise ValueError("primitive must have shape (nz, ny, nx, 5)")
    nz, ny, nx, _ = primitive.shape
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("wb") as stream:
        stream.write(HEADER.pack(nz, ny, nx, float(time)))
        primitive.tofile(stream)


def primitive_interior(q, nx: int, ny: int, nz: int) -> np.ndarray:
    """(rho, u, v, w, p) of the interior of a padded conserved state [nz+6][ny+6][nx+6][5] (a CUDA tensor is
    copied to the host first), with gamma 1.4 in the reference's expression order
    (warp_weno5_3d_rk3/kernels.py:30-42)."""
    if isinstance(q, torch.Tensor):
        q = q.detach().cpu().numpy()
    c = np.asarray(q, dtype=np.float64)[GHOST:GHOST + nz, GHOST:GHOST + ny, GHOST:GHOST + nx]
    out = np.empty_like(c)
    out[..., 0] = c[..., 0]
    for k in (1, 2, 3):
        out[..., k] = c[..., k] / c[..., 0]
    kinetic = out[..., 1] * out[..., 1] + out[..., 2] * out[..., 2] + out[..., 3] * out[..., 3]
    out[..., 4] = (1.4 - 1.0) * (c[..., 4] - 0.5 * c[..., 0] * kinetic)
    return out


def write_state(path: str | Path, time: float, q, nx: int, ny: int, nz: int) -> None:
    """Write the padded conserved 3D state q as a step file."""
    write_step(path, time, primitive_interior(q, nx, ny, nz))


def sha256(path: str | Path) -> str:
    h = hashlib.sha256()
    with Path(path).open("rb") as stream:
        for block in iter(lambda: stream.read(1 << 20), b""):
            h.update(block)
    return h.hexdigest()


def ulp_distance(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Number of doubles between a and b (monotone mapping of the bit patterns onto unsigned integers)."""
    def ordered(x):
        bits = np.asarray(x, dtype=np.float64).view(np.uint64)
        sign = np.uint64(1) << np.uint64(63)
        return np.where((bits & sign) != 0, ~bits, bits | sign)
    oa, ob = ordered(a), ordered(b)
    return np.maximum(oa, ob) - np.minimum(oa, ob)


def compare_steps(candidate: str | Path, reference: str | Path) -> dict:
    """Bitwise / ulp / absolute-error report of two step files (keys as in the reference's report)."""
    tc, uc = read_step(candidate)
    tr, ur = read_step(reference)
    if uc.shape != ur.shape:
        raise ValueError(f"shape mismatch: {uc.shape} != {ur.shape}")
    same = uc.view(np.uint64) == ur.view(np.uint64)
    err = np.abs(uc - ur)
    ulp = ulp_distance(uc, ur)
    denom = float(np.sum(np.abs(ur)))
    rep = {
        "candidate": str(candidate), "reference": str(reference),
        "candidate_sha256": sha256(candidate), "reference_sha256": sha256(reference),
        "file_bitwise_identical": Path(candidate).read_bytes() == Path(reference).read_bytes(),
        "array_bitwise_identical": bool(np.all(same)),
        "header": {"shape_equal": True, "candidate_time": tc, "reference_time": tr,
                   "time_bitwise_equal": struct.pack("=d", tc) == struct.pack("=d", tr)},
        "unequal_count": int(np.count_nonzero(~same)),
        "finite_pair_count": int(np.count_nonzero(np.isfinite(uc) & np.isfinite(ur))),
        "normalized_l1": float(np.sum(err)) / denom if denom else (0.0 if not np.any(err) else float("inf")),
        "mean_absolute_error": float(np.mean(err)), "max_absolute_error": float(np.max(err)),
        "max_ulp": int(np.max(ulp)), "components": {},
    }
    for c, name in enumerate(COMPONENT_NAMES):
        d = float(np.sum(np.abs(ur[..., c])))
        rep["components"][name] = {
            "unequal_count": int(np.count_nonzero(~same[..., c])),
            "mean_absolute_error": float(np.mean(err[..., c])), "max_absolute_error": float(np.max(err[..., c])),
            "normalized_l1": float(np.sum(err[..., c])) / d if d else 0.0, "max_ulp": int(np.max(ulp[..., c])),
        }
    if not np.all(same):
        def detail(flat):
            z, y, x, c = (int(v) for v in np.unravel_index(flat, uc.shape))
            return {"index": {"z": z, "y": y, "x": x, "component": COMPONENT_NAMES[c]},
                    "candidate": float(uc[z, y, x, c]), "reference": float(ur[z, y, x, c]),
                    "absolute_error": float(err[z, y, x, c]), "ulp": int(ulp[z, y, x, c])}
        rep["first_difference"] = detail(int(np.flatnonzero(~same.ravel())[0]))
        rep["largest_absolute_difference"] = detail(int(np.argmax(err.ravel())))
    return rep


def write_comparison(report: dict, path: str | Path) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(report, indent=2, sort_keys=True) + "\n", encoding="ascii")
