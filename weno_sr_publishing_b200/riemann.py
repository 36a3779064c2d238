"""Shock-tube validation of the 2D Euler path against exact Riemann solutions.

The reference validates its Euler kernels on one-dimensional problems run through the 2D solver on thin
nx x ny grids (ny = 10, transmissive boundaries), comparing the y-averaged state with exact finite-volume
cell averages of the exact Riemann solution:

* Sod, [0, 1], x0 = 0.5, t = 0.2, N = 100, CFL 0.8 (for_paper_results/run_sod.py:19-57, 66-121; exact cell
  averages by unsplit 15-point Gauss-Legendre, weno_z_borges_p2_results/run_riemann_1d.py:45-63);
* Lax, [-5, 5], x0 = 0, t = 1.3, N = 200, CFL 0.8 (for_paper_results/run_shock_tube_benchmark.py:33-42, 56-77;
  exact cell averages split at every wave boundary, for_paper_results/exact_riemann.py:243-280, and the
  error table of for_paper_results/make_shock_tube_figures.py:54-84, 136-140, 237-256);
* Titarev-Toro shock / entropy-wave interaction, [-5, 5], t = 5, CFL 0.8, N = 1001 and 2000, against a
  WENO5-JS run on N = 10001 interpolated to each mesh (for_paper_results/run_weno5_titarev_toro.py:22-61,
  make_titarev_toro_figures.py:43-50, 120-133).

The exact solver is the standard two-rarefaction / two-shock construction (E. F. Toro, Riemann Solvers and
Numerical Methods for Fluid Dynamics, ch. 4): Newton iteration on the pressure function from the
primitive-variable guess, then sampling of the self-similar solution. It is host-side numpy; the numerical
solutions come from the CUDA kernels.
"""
from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache

import numpy as np
import torch

from . import euler2d as E
from . import euler2d_w7 as E7
from .params import Params

Primitive = tuple[float, float, float]


# ------------------------------------------------------------------------------------------------
# Exact Riemann solver
# ------------------------------------------------------------------------------------------------
def _pressure_branch(p: float, rho: float, pk: float, ak: float, g: float) -> tuple[float, float]:
    """f_K(p) and f_K'(p) of one side: Rankine-Hugoniot branch if p > p_K, isentropic branch otherwise."""
    if p > pk:
        a_coef = 2.0 / ((g + 1.0) * rho)
        b_coef = (g - 1.0) / (g + 1.0) * pk
        s = np.sqrt(a_coef / (p + b_coef))
        return float((p - pk) * s), float(s * (1.0 - 0.5 * (p - pk) / (p + b_coef)))
    ratio = p / pk
    return (float(2.0 * ak / (g - 1.0) * (ratio ** ((g - 1.0) / (2.0 * g)) - 1.0)),
            float(ratio ** (-(g + 1.0) / (2.0 * g)) / (rho * ak)))


@lru_cache(maxsize=64)
def star_state(left: Primitive, right: Primitive, gamma: float = 1.4) -> tuple[float, float]:
    """(p*, u*) of the Riemann problem. Newton on f_L(p) + f_R(p) + u_R - u_L = 0 from the PV guess
    (floored at the smallest normal double), halving on a non-positive iterate, until the relative change
    is at most 1e-13."""
    rl, ul, pl = left
    rr, ur, pr = right
    al, ar = np.sqrt(gamma * pl / rl), np.sqrt(gamma * pr / rr)
    if 2.0 * (al + ar) / (gamma - 1.0) <= ur - ul:
        raise ValueError("the initial data generate a vacuum")
    p = max(0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (al + ar), float(np.finfo(np.float64).tiny))
    for _ in range(100):
        fl, dfl = _pressure_branch(p, rl, pl, al, gamma)
        fr, dfr = _pressure_branch(p, rr, pr, ar, gamma)
        nxt = p - (fl + fr + ur - ul) / (dfl + dfr)
        if not (nxt > 0.0) or not np.isfinite(nxt):
            nxt = 0.5 * p
        done = abs(nxt - p) <= 1.0e-13 * 0.5 * (nxt + p)
        p = nxt
        if done:
            break
    else:
        raise RuntimeError("exact Riemann pressure iteration did not converge")
    fl, _ = _pressure_branch(p, rl, pl, al, gamma)
    fr, _ = _pressure_branch(p, rr, pr, ar, gamma)
    return float(p), float(0.5 * (ul + ur + fr - fl))


def wave_speeds(left: Primitive, right: Primitive, gamma: float = 1.4) -> tuple[float, ...]:
    """Sorted speeds of every wave edge: shock, or rarefaction head and tail, on each side, and the contact."""
    p, u = star_state(left, right, gamma)
    out = [u]
    for (rho, vel, pk), sgn in ((left, -1.0), (right, 1.0)):
        a = np.sqrt(gamma * pk / rho)
        if p > pk:
            out.append(vel + sgn * a * np.sqrt((gamma + 1.0) / (2.0 * gamma) * p / pk + (gamma - 1.0) / (2.0 * gamma)))
        else:
            a_star = a * (p / pk) ** ((gamma - 1.0) / (2.0 * gamma))
            out += [vel + sgn * a, u + sgn * a_star]
    return tuple(sorted(float(s) for s in out))


def sample(xi, left: Primitive, right: Primitive, gamma: float = 1.4):
    """(rho, u, p) of the self-similar solution at xi = (x - x0) / t (arrays)."""
    xi = np.asarray(xi, dtype=np.float64)
    p_star, u_star = star_state(left, right, gamma)
    gm, gp = gamma - 1.0, gamma + 1.0
    rho = np.empty_like(xi)
    vel = np.empty_like(xi)
    prs = np.empty_like(xi)
    # side +1 is the left state seen from the contact, -1 the right one; the formulas below mirror with sgn
    for (rk, uk, pk), sgn, region in ((left, 1.0, xi <= u_star), (right, -1.0, xi > u_star)):
        ak = np.sqrt(gamma * pk / rk)
        x = xi[region]
        r, v, p = np.full_like(x, rk), np.full_like(x, uk), np.full_like(x, pk)
        if p_star > pk:  # shock
            s = uk - sgn * ak * np.sqrt(gp / (2.0 * gamma) * p_star / pk + gm / (2.0 * gamma))
            behind = sgn * (x - s) > 0.0
            q = p_star / pk
            r[behind] = rk * (q + gm / gp) / (gm / gp * q + 1.0)
            v[behind], p[behind] = u_star, p_star
        else:  # rarefaction
            head = uk - sgn * ak
            tail = u_star - sgn * ak * (p_star / pk) ** (gm / (2.0 * gamma))
            star = sgn * (x - tail) >= 0.0
            fan = (sgn * (x - head) > 0.0) & ~star
            r[star] = rk * (p_star / pk) ** (1.0 / gamma)
            v[star], p[star] = u_star, p_star
            xf = x[fan]
            c = 2.0 / gp * (ak + sgn * 0.5 * gm * (uk - xf))
            v[fan] = 2.0 / gp * (sgn * ak + 0.5 * gm * uk + xf)
            r[fan] = rk * (c / ak) ** (2.0 / gm)
            p[fan] = pk * (c / ak) ** (2.0 * gamma / gm)
        rho[region], vel[region], prs[region] = r, v, p
    return rho, vel, prs


def _conserved(rho, vel, prs, gamma):
    out = np.zeros(np.shape(rho) + (4,))
    out[..., 0] = rho
    out[..., 1] = rho * vel
    out[..., 3] = prs / (gamma - 1.0) + 0.5 * rho * vel * vel
    return out


def cell_averages(centers, width: float, t: float, x0: float, left: Primitive, right: Primitive,
                  gamma: float = 1.4, quadrature: int = 15, split: bool = True) -> np.ndarray:
    """Exact finite-volume averages (rho, rho u, 0, E) of the cells [c - w/2, c + w/2] at time t.

    split=True integrates each cell piecewise between the wave edges (exact up to the quadrature of the
    rarefaction fan); split=False applies the Gauss rule to the whole cell, the convention of the reference's
    Sod error table."""
    centers = np.asarray(centers, dtype=np.float64)
    nodes, weights = np.polynomial.legendre.leggauss(quadrature)
    edges_w = np.array([x0 + t * s for s in wave_speeds(left, right, gamma)]) if t > 0.0 else np.array([x0])

    def state_at(x):
        if t <= 0.0:
            m = x < x0
            rho = np.where(m, left[0], right[0])
            vel = np.where(m, left[1], right[1])
            prs = np.where(m, left[2], right[2])
        else:
            rho, vel, prs = sample((x - x0) / t, left, right, gamma)
        return _conserved(rho, vel, prs, gamma)

    if not split:
        acc = np.zeros((centers.size, 4))
        for xk, wk in zip(nodes, weights):
            acc += 0.5 * wk * state_at(centers + 0.5 * width * xk)
        return acc
    out = np.zeros((centers.size, 4))
    for n, c in enumerate(centers):
        lo, hi = c - 0.5 * width, c + 0.5 * width
        cuts = np.concatenate(([lo], edges_w[(edges_w > lo) & (edges_w < hi)], [hi]))
        total = np.zeros(4)
        for a, b in zip(cuts[:-1], cuts[1:]):
            mid, half = 0.5 * (a + b), 0.5 * (b - a)
            total += half * (weights[:, None] * state_at(mid + half * nodes)).sum(axis=0)
        out[n] = total / width
    return out


# ------------------------------------------------------------------------------------------------
# Shock tubes through the 2D solver
# ------------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class ShockTube:
    key: str
    x_min: float
    x_max: float
    x0: float
    t_end: float
    nx: int
    ny: int
    cfl: float
    left: Primitive
    right: Primitive
    split_exact: bool  # how the exact reference cell averages are integrated


SOD = ShockTube("sod", 0.0, 1.0, 0.5, 0.2, 100, 10, 0.8, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), False)
LAX = ShockTube("lax", -5.0, 5.0, 0.0, 1.3, 200, 10, 0.8, (0.445, 0.698, 3.528), (0.5, 0.0, 0.571), True)
TUBES = {"sod": SOD, "lax": LAX}


def tube_params(tube: ShockTube, gamma: float = 1.4) -> Params:
    dx = (tube.x_max - tube.x_min) / tube.nx
    return Params(nx=tube.nx, ny=tube.ny, x_length=tube.x_max - tube.x_min, y_length=tube.ny * dx, cfl=tube.cfl,
                  t_end=tube.t_end, gamma=gamma)


def tube_initial_state(tube: ShockTube, gamma: float = 1.4, ghost: int = 3) -> np.ndarray:
    """Padded [ny+2g][nx+2g][4] state: exact cell averages of the initial step (a cell cut by x0 gets the
    length-weighted mix, run_shock_tube_benchmark.py:56-77), the same on every row."""
    g = ghost
    dx = (tube.x_max - tube.x_min) / tube.nx
    xl = tube.x_min + (np.arange(tube.nx + 2 * g) - g) * dx
    left_len = np.clip(np.minimum(xl + dx, tube.x0) - xl, 0.0, dx)
    cl = _conserved(np.float64(tube.left[0]), tube.left[1], tube.left[2], gamma)
    cr = _conserved(np.float64(tube.right[0]), tube.right[1], tube.right[2], gamma)
    row = (left_len[:, None] * cl[None, :] + (dx - left_len)[:, None] * cr[None, :]) / dx
    return np.ascontiguousarray(np.broadcast_to(row[None], (tube.ny + 2 * g, tube.nx + 2 * g, 4)))


def primitive_1d(conserved: np.ndarray, gamma: float = 1.4) -> dict[str, np.ndarray]:
    rho = conserved[:, 0]
    vel = conserved[:, 1] / rho
    vt = conserved[:, 2] / rho
    return {"rho": rho, "velocity": vel,
            "pressure": (gamma - 1.0) * (conserved[:, 3] - 0.5 * rho * (vel * vel + vt * vt))}


def errors(numerical: np.ndarray, reference: np.ndarray, dx: float) -> dict[str, float]:
    d = numerical - reference
    return {"l1_mean": float(np.mean(np.abs(d))), "l1_integral": float(dx * np.sum(np.abs(d))),
            "l2": float(np.sqrt(np.mean(d * d))), "linf": float(np.max(np.abs(d)))}


def _run_padded(init: np.ndarray, p: Params, t_end: float, method: str, mlp_params, device) -> tuple:
    dev = torch.device(device)
    bufs = [torch.as_tensor(init, device=dev).contiguous()] + \
        [torch.zeros(p.padded_shape, dtype=torch.float64, device=dev) for _ in range(3)]
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = E.run(bufs, p, t_end, method, "transmissive", mlp_params=mlp_params)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    final = bufs[res.final_slot].cpu().numpy()
    return final[3:3 + p.ny, 3:3 + p.nx], res, e0.elapsed_time(e1)


def _run_w7(tube: ShockTube, gamma: float, device, method: str = "js", closure=None) -> tuple:
    """WENO7 (JS, Z or SR-FP64 weights) with Shu RK4 on the tube, ghost width 4 (the WENO7 runs of
    run_sod.py:86-99 and run_shock_tube_benchmark.py:127-177)."""
    dx = (tube.x_max - tube.x_min) / tube.nx
    p = E7.Params(nx=tube.nx, ny=tube.ny, x_min=tube.x_min, x_max=tube.x_max, y_min=0.0, y_max=tube.ny * dx,
                  gamma=gamma, cfl=tube.cfl, t_end=tube.t_end)
    dev = torch.device(device)
    u = torch.as_tensor(tube_initial_state(tube, gamma, ghost=4), device=dev).contiguous()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = E7.run(u, p, "transmissive", method=method, closure=closure)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    return u.cpu().numpy()[4:4 + tube.ny, 4:4 + tube.nx], res, e0.elapsed_time(e1)


def shock_tube_run(tube: ShockTube, method: str, mlp_params=None, device="cuda", gamma: float = 1.4) -> dict:
    """Run the tube on the GPU to t_end and compare the y-averaged solution with the exact cell averages.
    method: a WENO5 method of the 2D path ("js", "z", "sr_f64", ...), "w7_js", "w7_z" or "w7_sr_f64" (WENO7-JS,
    WENO7-Z or WENO7-SR with the WENO7 closure `mlp_params`, Shu RK4)."""
    p = tube_params(tube, gamma)
    if method in ("w7_js", "w7_z", "w7_sr_f64"):
        state, res, ms = _run_w7(tube, gamma, device, method[3:], mlp_params)
    else:
        state, res, ms = _run_padded(tube_initial_state(tube, gamma), p, tube.t_end, method, mlp_params, device)
    conserved = state.mean(axis=0)
    x = tube.x_min + (np.arange(tube.nx) + 0.5) * p.dx
    exact = cell_averages(x, p.dx, tube.t_end, tube.x0, tube.left, tube.right, gamma, 15, tube.split_exact)
    num, ref = primitive_1d(conserved, gamma), primitive_1d(exact, gamma)
    out = {"problem": tube.key, "method": method, "nx": tube.nx, "ny": tube.ny, "steps": res.steps, "t": res.t,
           "device_ms": ms, "x": x, "conserved_1d": conserved, "exact_conserved": exact}
    for field in ("rho", "velocity", "pressure"):
        out.update({f"{field}_{k}": v for k, v in errors(num[field], ref[field], p.dx).items()})
    return out


# ------------------------------------------------------------------------------------------------
# Titarev-Toro shock / entropy-wave interaction
# ------------------------------------------------------------------------------------------------
TT_SHOCK = -4.5
TT_LEFT = (1.515695, 0.523346, 1.805)


def titarev_toro_state(nx: int, ny: int = 10, x_min: float = -5.0, x_max: float = 5.0,
                       gamma: float = 1.4) -> np.ndarray:
    """Exact cell averages: the post-shock state left of x = -4.5, rho = 1 + 0.1 sin(20 pi x), u = 0, p = 1
    right of it (a cell cut by the shock gets both parts; run_weno5_titarev_toro.py:31-61)."""
    g = 3
    dx = (x_max - x_min) / nx
    xl = x_min + (np.arange(nx + 2 * g) - g) * dx
    xr = xl + dx
    left_len = np.clip(np.minimum(xr, TT_SHOCK) - xl, 0.0, dx)
    r0 = np.maximum(xl, TT_SHOCK)
    right_len = np.clip(xr - r0, 0.0, dx)
    k = 20.0 * np.pi
    right_mass = np.where(right_len > 0.0, xr - r0 + 0.1 * (np.cos(k * r0) - np.cos(k * xr)) / k, 0.0)
    cl = _conserved(np.float64(TT_LEFT[0]), TT_LEFT[1], TT_LEFT[2], gamma)
    cr = np.array([0.0, 0.0, 0.0, 1.0 / (gamma - 1.0)])
    row = (left_len[:, None] * cl[None, :] + right_len[:, None] * cr[None, :]) / dx
    row[:, 0] += right_mass / dx
    return np.ascontiguousarray(np.broadcast_to(row[None], (ny + 2 * g, nx + 2 * g, 4)))


def titarev_toro_run(nx: int, method: str, mlp_params=None, device="cuda", ny: int = 10, cfl: float = 0.8,
                     t_end: float = 5.0, x_min: float = -5.0, x_max: float = 5.0) -> dict:
    dx = (x_max - x_min) / nx
    p = Params(nx=nx, ny=ny, x_length=x_max - x_min, y_length=ny * dx, cfl=cfl, t_end=t_end)
    state, res, ms = _run_padded(titarev_toro_state(nx, ny, x_min, x_max), p, t_end, method, mlp_params, device)
    return {"method": method, "nx": nx, "x": x_min + (np.arange(nx) + 0.5) * dx, "rho": state[..., 0].mean(axis=0),
            "steps": res.steps, "t": res.t, "device_ms": ms}


def titarev_toro_errors(run: dict, reference: dict) -> dict[str, float]:
    """Density errors against a fine reference run interpolated to the run's cell centres."""
    ref = np.interp(run["x"], reference["x"], reference["rho"])
    d = run["rho"] - ref
    return {"rho_l1": float(np.mean(np.abs(d))), "rho_l2": float(np.sqrt(np.mean(d * d))),
            "rho_linf": float(np.max(np.abs(d)))}
