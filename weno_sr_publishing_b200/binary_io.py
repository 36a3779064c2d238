"""Step files of the 3D solver and their comparison (warp_weno5_3d_rk3/binary_io.py).

Format (an interface, kept as the reference's C++ code writes it): a packed 20-byte header
``uint32 nz, ny, nx; float64 time`` followed by ``float64 primitive[nz][ny][nx][5]`` with components
(rho, u, v, w, p) of the interior cells, all little-endian. ``read_step`` raises ValueError on a truncated
header or payload and on trailing bytes, the reference's error type for those cases.
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import torch

# The 20-byte header as one packed little-endian record (the C++ writer's native packing on x86).
STEP_HEADER = np.dtype([("nz", "<u4"), ("ny", "<u4"), ("nx", "<u4"), ("time", "<f8")])
COMPONENT_NAMES = ("rho", "u", "v", "w", "p")
GHOST = 3


def _payload_shape(head) -> tuple[int, int, int, int]:
    return int(head["nz"]), int(head["ny"]), int(head["nx"]), len(COMPONENT_NAMES)


def read_step(path: str | Path) -> tuple[float, np.ndarray]:
    """(time, primitive[nz][ny][nx][5]) of a step file. The file size is checked against the size the header
    implies before any payload is read: a short header, a short payload or trailing bytes raise ValueError."""
    path = Path(path)
    size = path.stat().st_size
    if size < STEP_HEADER.itemsize:
        raise ValueError(f"{path}: {size} bytes, shorter than the {STEP_HEADER.itemsize}-byte step header")
    head = np.fromfile(path, dtype=STEP_HEADER, count=1)[0]
    shape = _payload_shape(head)
    expected = STEP_HEADER.itemsize + 8 * int(np.prod(shape, dtype=np.int64))
    if size != expected:
        what = "truncated payload" if size < expected else "trailing bytes after the payload"
        raise ValueError(f"{path}: {what}: header {shape[:3]} implies {expected} bytes, file has {size}")
    values = np.fromfile(path, dtype="<f8", offset=STEP_HEADER.itemsize).reshape(shape)
    return float(head["time"]), values


def write_step(path: str | Path, time: float, primitive: np.ndarray) -> None:
    """Write one step file: the header record, then the primitive array as little-endian float64."""
    prim = np.asarray(primitive)
    if prim.ndim != 4 or prim.shape[-1] != len(COMPONENT_NAMES):
        raise ValueError(f"primitive must have shape (nz, ny, nx, 5), got {prim.shape}")
    head = np.zeros((), dtype=STEP_HEADER)
    head["nz"], head["ny"], head["nx"] = prim.shape[:3]
    head["time"] = time
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    body = np.ascontiguousarray(prim, dtype="<f8")
    with path.open("wb") as out:
        out.write(head.tobytes())
        out.write(memoryview(body).cast("B"))


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
                   "time_bitwise_equal": np.float64(tc).tobytes() == np.float64(tr).tobytes()},
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
