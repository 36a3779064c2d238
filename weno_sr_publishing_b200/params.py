"""Grid/run parameters, mirroring warp_weno5_helpers.Params (warp_weno5_helpers.py:66-87)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Params:
    nx: int = 450
    ny: int = 178
    ghost: int = 3
    gamma: float = 1.4
    x_length: float = 0.225
    y_length: float = 0.089
    cfl: float = 0.228
    t_end: float = 0.0002

    @property
    def dx(self) -> float:
        return self.x_length / float(self.nx)

    @property
    def dy(self) -> float:
        return self.y_length / float(self.ny)

    @property
    def padded_shape(self) -> tuple[int, int, int]:
        return (self.ny + 2 * self.ghost, self.nx + 2 * self.ghost, 4)


def primitive_from_conserved(u: np.ndarray, gamma: float) -> np.ndarray:
    """Primitive (rho, u, v, p) of conserved (rho, rho u, rho v, E) cells, the density floored at 1e-15 before it
    divides (the host-side decoding of warp_weno5_helpers.py:167-172, same operations in the same order)."""
    cons = np.asarray(u, dtype=np.float64)
    prim = np.empty(cons.shape[:-1] + (4,), dtype=np.float64)
    rho = np.maximum(cons[..., 0], 1.0e-15, out=prim[..., 0])
    vx = np.divide(cons[..., 1], rho, out=prim[..., 1])
    vy = np.divide(cons[..., 2], rho, out=prim[..., 2])
    prim[..., 3] = (gamma - 1.0) * (cons[..., 3] - 0.5 * rho * (vx * vx + vy * vy))
    return prim


def interior_stats(u_host: np.ndarray, params: Params) -> dict[str, float]:
    """Health summary of the interior cells that the adapters report (warp_weno5_helpers.py:210-224): mass (the
    raw density summed, times dx dy), the ranges of the floored density and of the pressure, the NaN count of the
    conserved values, and the counts of non-positive (floored) densities and pressures."""
    g = params.ghost
    cells = u_host[g: g + params.ny, g: g + params.nx, :]
    prim = primitive_from_conserved(cells, params.gamma)
    rho, pres = prim[..., 0], prim[..., 3]
    stats = {"mass": float(np.sum(cells[..., 0]) * params.dx * params.dy)}
    stats.update(rho_min=float(rho.min()), rho_max=float(rho.max()), p_min=float(pres.min()), p_max=float(pres.max()))
    stats["nan_count"] = float(np.count_nonzero(np.isnan(cells)))
    stats["rho_neg"] = float(np.count_nonzero(rho <= 0.0))
    stats["p_neg"] = float(np.count_nonzero(pres <= 0.0))
    return stats
