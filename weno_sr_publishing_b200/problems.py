"""Seeded initial conditions for the 2D Euler workloads.

The four-quadrant Riemann problem follows for_paper_results/run_quadrant.py:62-103 of the reference:
quadrant 1 = upper right, 2 = upper left, 3 = lower left, 4 = lower right, split at (0.5, 0.5) of
the unit square, cell averages by tensor Gauss-Legendre quadrature (15 points per direction in the
reference's timing run, run_weno5_timing.py:86-91). Instead of the fixed C.3-C.6 tables, the states are
drawn from a seeded generator: rho in [0.5, 2], u, v in [-1, 1], p in [0.1, 1.5] per quadrant.
"""
from __future__ import annotations

from dataclasses import dataclass

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


def vortex_point_rk4(nx: int, ny: int, t: float = 0.0, quadrature: int = 15, gamma: float = 1.4,
                     x_min: float = -10.0, x_max: float = 10.0, y_min: float = -10.0, y_max: float = 10.0,
                     ghost: int = 4) -> np.ndarray:
    """Cell averages (quadrature^2 Gauss-Legendre points) of the periodic isentropic vortex of the WENO7
    point-value path (weno7_point_rk4_shu/point_rk4.py:77-117): strength 5, mean flow (1, 1), period 20,
    centre displaced by (t, t) with the nearest periodic image, on the padded [ny+2g][nx+2g] grid."""
    xi, wi = np.polynomial.legendre.leggauss(quadrature)
    dx, dy = (x_max - x_min) / nx, (y_max - y_min) / ny
    jj, ii = np.indices((ny + 2 * ghost, nx + 2 * ghost))
    xc = x_min + (ii - ghost + 0.5) * dx
    yc = y_min + (jj - ghost + 0.5) * dy
    length, beta = 20.0, 5.0
    out = np.zeros((ny + 2 * ghost, nx + 2 * ghost, 4))
    for sx, wx in zip(xi, wi):
        x = xc + 0.5 * dx * float(sx)
        for sy, wy in zip(xi, wi):
            y = yc + 0.5 * dy * float(sy)
            ddx = x - t - length * np.round((x - t) / length)
            ddy = y - t - length * np.round((y - t) / length)
            r2 = ddx * ddx + ddy * ddy
            d_t = -((gamma - 1.0) * beta * beta) / (8.0 * gamma * np.pi * np.pi) * np.exp(1.0 - r2)
            rho = 1.0 + (np.power(1.0 + d_t, 1.0 / (gamma - 1.0)) - 1.0)
            p = 1.0 + (np.power(1.0 + d_t, gamma / (gamma - 1.0)) - 1.0)
            f = beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
            u, v = 1.0 - f * ddy, 1.0 + f * ddx
            out += 0.25 * float(wx) * float(wy) * conserved_from_primitive(rho, u, v, p, gamma)
    return out


def double_mach_primitive(x, y, t: float = 0.0):
    """Double-Mach reflection: a Mach-10 shock through (1/6, 0) at 60 degrees to the wall, moving right;
    post-shock (8, 8.25 cos 30, -8.25 sin 30, 116.5) left of it, (1.4, 0, 0, 1) right of it
    (run_double_mach_compare.py:50-56)."""
    r3 = np.sqrt(3.0)
    left = np.asarray(x) < 1.0 / 6.0 + np.asarray(y) / r3 + 20.0 * t / r3
    return (np.where(left, 8.0, 1.4), np.where(left, 8.25 * r3 * 0.5, 0.0), np.where(left, -8.25 * 0.5, 0.0),
            np.where(left, 116.5, 1.0))


def double_mach_state(nx: int, ny: int, quadrature: int = 15, gamma: float = 1.4, x_length: float = 4.0,
                      y_length: float = 1.0, ghost: int = GHOST) -> np.ndarray:
    """Padded initial state of the double-Mach problem on [0, 4] x [0, 1]: Gauss-Legendre cell averages
    (quadrature^2 points) of every padded cell (run_double_mach_compare.py:69-88)."""
    xi, wi = np.polynomial.legendre.leggauss(quadrature)
    dx, dy = x_length / nx, y_length / ny
    jj, ii = np.indices((ny + 2 * ghost, nx + 2 * ghost))
    xc = (ii - ghost + 0.5) * dx
    yc = (jj - ghost + 0.5) * dy
    state = np.zeros((ny + 2 * ghost, nx + 2 * ghost, 4))
    for sx, wx in zip(xi, wi):
        x = xc + 0.5 * dx * float(sx)
        for sy, wy in zip(xi, wi):
            rho, u, v, p = double_mach_primitive(x, yc + 0.5 * dy * float(sy))
            state += 0.25 * float(wx) * float(wy) * conserved_from_primitive(rho, u, v, p, gamma)
    return state


# ------------------------------------------------------------------------------------------------
# 3D shock-bubble interaction
# ------------------------------------------------------------------------------------------------
_GL3_NODES = (-0.77459666924148340427791481488384306430816650390625, 0.0,
              0.77459666924148340427791481488384306430816650390625)
_GL3_WEIGHTS = (0.55555555555555546920487586248782463371753692626953125,
                0.88888888888888917261255073754000477492809295654296875,
                0.55555555555555546920487586248782463371753692626953125)


def _gauss27(value_fn, nx, ny, nz, x0, y0, z0, dx, dy, dz, ghost=3):
    """0.125 sum_{a,b,c} w_a w_b w_c value(x_a, y_b, z_c) over every padded cell, in the reference's loop
    order (warp_weno5_3d_rk3/kernels.py:747-773); value_fn returns the 5 conserved components."""
    k, j, i = np.meshgrid(np.arange(nz + 2 * ghost), np.arange(ny + 2 * ghost), np.arange(nx + 2 * ghost),
                          indexing="ij")
    xc = x0 + ((i - ghost).astype(np.float64) + 0.5) * dx
    yc = y0 + ((j - ghost).astype(np.float64) + 0.5) * dy
    zc = z0 + ((k - ghost).astype(np.float64) + 0.5) * dz
    total = np.zeros(xc.shape + (5,))
    for a in range(3):
        x = xc + 0.5 * dx * _GL3_NODES[a]
        for b in range(3):
            y = yc + 0.5 * dy * _GL3_NODES[b]
            for c in range(3):
                z = zc + 0.5 * dz * _GL3_NODES[c]
                w = _GL3_WEIGHTS[a] * _GL3_WEIGHTS[b] * _GL3_WEIGHTS[c]
                total = total + w * value_fn(x, y, z)
    return 0.125 * total


def _conserved5(rho, u, v, w, p, gamma=1.4):
    return np.stack([rho, rho * u, rho * v, rho * w, 0.5 * rho * (u * u + v * v + w * w) + p / (gamma - 1.0)],
                    axis=-1)


def shockbubble_reference_state(nx: int = 224, ny: int = 88, nz: int = 88, x_end: float = 0.225,
                                y_end: float = 0.089, z_end: float = 0.089) -> np.ndarray:
    """The reference's Ma = 3 air/helium shock-bubble initial state (kernels.py:686-773, config.py):
    post-shock air for x < 0.005 moving at 736.911, a helium sphere of radius 0.025 at (0.035, 0.0445,
    0.0445) at the ambient pressure, 3 x 3 x 3 Gauss cell averages on every padded cell."""
    gamma, mach, rho_air, p_air, rho_he = 1.4, 3.0, 1.29, 101325.0, 0.214
    rho_post = (((gamma + 1.0) * mach * mach) / ((gamma - 1.0) * mach * mach + 2.0)) * rho_air
    p_post = ((((2.0 * gamma) * mach * mach) - (gamma - 1.0)) / (gamma + 1.0)) * p_air

    def value(x, y, z):
        rho = np.full(x.shape, rho_air)
        u = np.zeros(x.shape)
        p = np.full(x.shape, p_air)
        post = x < 0.005
        rho = np.where(post, rho_post, rho)
        u = np.where(post, 736.911, u)
        p = np.where(post, p_post, p)
        dxb, dyb, dzb = x - 0.035, y - 0.0445, z - 0.0445
        inside = dxb * dxb + dyb * dyb + dzb * dzb <= 0.025 * 0.025
        rho = np.where(inside, rho_he, rho)
        u = np.where(inside, 0.0, u)
        p = np.where(inside, p_air, p)
        z0 = np.zeros(x.shape)
        return _conserved5(rho, u, z0, z0, p, gamma)

    return _gauss27(value, nx, ny, nz, 0.0, 0.0, 0.0, x_end / nx, y_end / ny, z_end / nz)


@dataclass(frozen=True)
class ShockBubble:
    """A planar shock of Mach `mach` moving in +x into quiescent gas (rho 1, p 1) that holds a sphere of
    radius 0.25 and density `density_ratio` at the same pressure, on [0, 2.545] x [0, 1] x [0, 1]."""
    mach: float
    density_ratio: float
    nx: int = 224
    ny: int = 88
    nz: int = 88
    length: tuple = (2.545, 1.0, 1.0)
    shock_x: float = 0.2
    centre: tuple = (0.6, 0.5, 0.5)
    radius: float = 0.25
    gamma: float = 1.4

    @staticmethod
    def seeded(seed: int, nx: int = 224, ny: int = 88, nz: int = 88) -> "ShockBubble":
        rng = np.random.default_rng(seed)
        return ShockBubble(float(rng.uniform(2.0, 3.0)), float(rng.uniform(0.1, 0.3)), nx, ny, nz)

    @property
    def spacing(self) -> tuple:
        return (self.length[0] / self.nx, self.length[1] / self.ny, self.length[2] / self.nz)

    def post_shock(self) -> tuple:
        """Rankine-Hugoniot state behind the shock: (rho, u, p)."""
        g, m = self.gamma, self.mach
        rho2 = (g + 1.0) * m * m / ((g - 1.0) * m * m + 2.0)
        p2 = (2.0 * g * m * m - (g - 1.0)) / (g + 1.0)
        u2 = m * np.sqrt(g) * (1.0 - 1.0 / rho2)
        return rho2, u2, p2

    def inflow(self) -> np.ndarray:
        rho, u, p = self.post_shock()
        return _conserved5(np.array(rho), np.array(u), np.array(0.0), np.array(0.0), np.array(p), self.gamma)

    def state(self) -> np.ndarray:
        rho2, u2, p2 = self.post_shock()
        cx, cy, cz = self.centre

        def value(x, y, z):
            post = x < self.shock_x
            inside = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 <= self.radius ** 2
            rho = np.where(post, rho2, np.where(inside, self.density_ratio, 1.0))
            u = np.where(post, u2, 0.0)
            p = np.where(post, p2, 1.0)
            z0 = np.zeros(x.shape)
            return _conserved5(rho, u, z0, z0, p, self.gamma)

        dx, dy, dz = self.spacing
        return _gauss27(value, self.nx, self.ny, self.nz, 0.0, 0.0, 0.0, dx, dy, dz)
