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
    """warp_weno5_helpers.py:167-172 (rho floored at 1e-15)."""
    rho = np.maximum(u[..., 0], 1.0e-15)
    vel_x = u[..., 1] / rho
    vel_y = u[..., 2] / rho
    p = (gamma - 1.0) * (u[..., 3] - 0.5 * rho * (vel_x * vel_x + vel_y * vel_y))
    return np.stack([rho, vel_x, vel_y, p], axis=-1)


def interior_stats(u_host: np.ndarray, params: Params) -> dict[str, float]:
    """warp_weno5_helpers.py:210-224."""
    gc = params.ghost
    interior = u_host[gc: gc + params.ny, gc: gc + params.nx, :]
    pri = primitive_from_conserved(interior, params.gamma)
    return {
        "mass": float(np.sum(interior[..., 0]) * params.dx * params.dy),
        "rho_min": float(np.min(pri[..., 0])),
        "rho_max": float(np.max(pri[..., 0])),
        "p_min": float(np.min(pri[..., 3])),
        "p_max": float(np.max(pri[..., 3])),
        "nan_count": float(np.isnan(interior).sum()),
        "rho_neg": float(np.sum(pri[..., 0] <= 0.0)),
        "p_neg": float(np.sum(pri[..., 3] <= 0.0)),
    }
