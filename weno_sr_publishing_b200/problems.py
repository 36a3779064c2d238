"""Seeded initial conditions for the 2D Euler workloads.

The four-quadrant Riemann problem follows for_paper_results/run_quadrant.py:62-103 of the reference:
quadrant 1 = upper right, 2 = upper left, 3 = lower left, 4 = lower right, split at (0.5, 0.5) of
the unit square, cell averages by tensor Gauss-Legendre quadrature (15 points per direction in the
reference's timing run, run_weno5_timing.py:86-91). Instead of the fixed C.3-C.6 tables, the states are
drawn from a seeded generator: rho in [0.5, 2], u, v in [-1, 1], p in [0.1, 1.5] per quadrant.
"""
from __future__ import annotations

import numpy as np

GHOST = 3


def conserved_from_primitive(rho, u, v, p, gamma: float = 1.4):
    e = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return np.stack([rho, rho * u, rho * v, e], axis=-1)


def seeded_quadrant_states(seed: int) -> tuple[tuple[float, float, float, float], ...]:
    """Four primitive (rho, u, v, p) states, in quadrant order 1..4."""
    rng = np.random.default_rng(seed)
    states = []
    for _ in range(4):
        rho = float(rng.uniform(0.5, 2.0))
        u = float(rng.uniform(-1.0, 1.0))
        v = float(rng.uniform(-1.0, 1.0))
        p = float(rng.uniform(0.1, 1.5))
        states.append((rho, u, v, p))
    return tuple(states)


def quadrant_primitive(x, y, states):
    rho = np.empty_like(x)
    vx = np.empty_like(x)
    vy = np.empty_like(x)
    pr = np.empty_like(x)
    regions = ((x >= 0.5) & (y >= 0.5), (x < 0.5) & (y >= 0.5), (x < 0.5) & (y < 0.5), (x >= 0.5) & (y < 0.5))
    for mask, (r, a, b, p) in zip(regions, states):
        rho[mask] = r
        vx[mask] = a
        vy[mask] = b
        pr[mask] = p
    return rho, vx, vy, pr


def make_quadrant_state(nx: int, ny: int, states, quadrature: int = 15, gamma: float = 1.4,
                        x_min: float = 0.0, x_max: float = 1.0, y_min: float = 0.0, y_max: float = 1.0,
                        ghost: int = GHOST) -> np.ndarray:
    """Padded [(ny+2g), (nx+2g), 4] cell averages (run_quadrant.py:88-103)."""
    if quadrature < 1:
        raise ValueError("quadrature order must be at least one")
    xi, wi = np.polynomial.legendre.leggauss(quadrature)
    dx = (x_max - x_min) / nx
    dy = (y_max - y_min) / ny
    jj, ii = np.indices((ny + 2 * ghost, nx + 2 * ghost))
    xc = x_min + (ii - ghost + 0.5) * dx
    yc = y_min + (jj - ghost + 0.5) * dy
    state = np.zeros((ny + 2 * ghost, nx + 2 * ghost, 4))
    for sx, wx in zip(xi, wi):
        x = xc + 0.5 * dx * float(sx)
        for sy, wy in zip(xi, wi):
            y = yc + 0.5 * dy * float(sy)
            rho, vx, vy, pr = quadrant_primitive(x, y, states)
            state += 0.25 * float(wx) * float(wy) * conserved_from_primitive(rho, vx, vy, pr, gamma)
    return state


def isentropic_vortex(nx: int, ny: int, t: float = 0.0, quadrature: int = 5, gamma: float = 1.4,
                      strength: float = 5.0, length: float = 10.0, ghost: int = GHOST) -> np.ndarray:
    """Periodic isentropic vortex on [0, L]^2 advected by (1, 1): exact cell averages at time t.

    The standard Shu vortex (strength 5, mean flow (1, 1)), the exact-solution accuracy test of the
    reference's vortex experiment (weno7_point_rk4_shu/point_rk4.py:81-118)."""
    xi, wi = np.polynomial.legendre.leggauss(quadrature)
    dx = length / nx
    dy = length / ny
    jj, ii = np.indices((ny + 2 * ghost, nx + 2 * ghost))
    xc = (ii - ghost + 0.5) * dx
    yc = (jj - ghost + 0.5) * dy
    state = np.zeros((ny + 2 * ghost, nx + 2 * ghost, 4))
    x0 = 0.5 * length + t
    y0 = 0.5 * length + t
    for sx, wx in zip(xi, wi):
        x = xc + 0.5 * dx * float(sx)
        for sy, wy in zip(xi, wi):
            y = yc + 0.5 * dy * float(sy)
            rx = np.mod(x - x0 + 0.5 * length, length) - 0.5 * length
            ry = np.mod(y - y0 + 0.5 * length, length) - 0.5 * length
            r2 = rx * rx + ry * ry
            du = strength / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2)) * (-ry)
            dv = strength / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2)) * rx
            dtemp = -(gamma - 1.0) * strength ** 2 / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
            temp = 1.0 + dtemp
            rho = temp ** (1.0 / (gamma - 1.0))
            p = rho ** gamma
            state += 0.25 * float(wx) * float(wy) * conserved_from_primitive(rho, 1.0 + du, 1.0 + dv, p, gamma)
    return state
