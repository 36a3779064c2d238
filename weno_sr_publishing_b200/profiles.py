"""Seeded periodic training profiles on [0, 1) with closed-form finite-volume cell averages.

The families follow the reference's training generator (code/snapshot/
teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/fvm_profiles.py:12-425, ``ProfileBatch`` and
``make_profiles``): a base level plus three sine modes, two Gaussians exp(-(d/sigma)^2/2), two triangles,
one semi-ellipse and three top-hat boxes, where d is the nearest-image periodic distance to the centre.
A family ("smooth", "gaussian", "square", "triangle", "ellipse", "multi", "composite", drawn with the
reference's default probabilities) switches components on, with signed log-uniform amplitudes
10^U[-3,0] * max(|base|, 1) and the reference's width ranges in cells.

A batch is a float64 array [B, DESC_LEN] with the layout

    0            base
    1 + 3m       sine m (m < 3):      amplitude, wavenumber k (integer), phase
    10 + 3m      Gaussian m (m < 2):  amplitude, centre, sigma
    16 + 3m      triangle m (m < 2):  amplitude, centre, half-width
    22           semi-ellipse:        amplitude, centre, half-width
    25 + 3m      box m (m < 3):       amplitude, left edge, width

Cell averages are exact integrals of the advected profile q0(x - s) (the reference integrates the
continuous parts with 15-point Gauss-Legendre and the boxes exactly, fvm_profiles.py:242-286): a sine
mode averages to amp * sinc(pi k dx) * sin(2 pi k x_c + phase), every other component through its
antiderivative on the nearest image. The CUDA training kernels evaluate the same expressions on the
device (csrc/train1d.cuh, ``exact_cell_average``).
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf

DESC_LEN = 34
FAMILIES = ("smooth", "gaussian", "square", "triangle", "ellipse", "multi", "composite")
FAMILY_PROBS = (0.25, 0.15, 0.15, 0.15, 0.10, 0.10, 0.10)
SINE, GAUSS, TRI, ELL, BOX = 1, 10, 16, 22, 25


def _uniform(rng, lo, hi, shape):
    """lo + (hi - lo) U[0, 1), also when hi < lo on coarse grids (fvm_profiles.py:23-33)."""
    return lo + (hi - lo) * rng.random(shape)


def _signed_log_amp(rng, scale, shape):
    mag = 10.0 ** _uniform(rng, -3.0, 0.0, shape) * scale
    return np.where(rng.random(shape) < 0.5, -mag, mag)


def make_profiles(rng: np.random.Generator, batch: int, n: int, family: str | None = None):
    """Draw ``batch`` descriptors for an n-cell grid; returns (desc [B, DESC_LEN], family ids [B])."""
    if family is None:
        fam = rng.choice(len(FAMILIES), size=batch, p=np.asarray(FAMILY_PROBS))
    else:
        fam = np.full(batch, FAMILIES.index(family))
    B = batch
    m = [(fam == k).astype(np.float64)[:, None] for k in range(len(FAMILIES))]
    base = _uniform(rng, -2.0, 4.0, (B, 1))
    scale = np.maximum(np.abs(base), 1.0)
    d = np.zeros((B, DESC_LEN))
    d[:, 0] = base[:, 0]
    sine_amp = _signed_log_amp(rng, scale, (B, 3)) / 3.0 * (m[0] + 0.35 * m[6])
    sine_k = rng.integers(1, max(2, n // 10) + 1, (B, 3)).astype(np.float64)
    sine_ph = _uniform(rng, 0.0, 2.0 * math.pi, (B, 3))
    g_amp = _signed_log_amp(rng, scale, (B, 2)) * (m[1] + 0.5 * m[6])
    g_c = _uniform(rng, 0.0, 1.0, (B, 2))
    g_s = _uniform(rng, 1.5 / n, 8.0 / n, (B, 2))
    t_amp = _signed_log_amp(rng, scale, (B, 2)) * (m[3] + 0.5 * m[6])
    t_c = _uniform(rng, 0.0, 1.0, (B, 2))
    t_h = _uniform(rng, 3.0 / n, min(18.0 / n, 0.24), (B, 2))
    e_amp = _signed_log_amp(rng, scale, (B, 1)) * (m[4] + m[6])
    e_c = _uniform(rng, 0.0, 1.0, (B, 1))
    e_h = _uniform(rng, 4.0 / n, min(20.0 / n, 0.24), (B, 1))
    b_amp = _signed_log_amp(rng, scale, (B, 3))
    b_left = _uniform(rng, 0.0, 1.0, (B, 3))
    b_w = _uniform(rng, 3.0 / n, min(32.0 / n, 0.40), (B, 3))
    active = (rng.random((B, 3)) < np.array([1.0, 0.85, 0.55])).astype(np.float64)
    first = np.array([[1.0, 0.0, 0.0]])
    b_amp = b_amp * (m[2] * first + m[5] * active + m[6] * first)
    for j in range(3):
        d[:, SINE + 3 * j:SINE + 3 * j + 3] = np.stack([sine_amp[:, j], sine_k[:, j], sine_ph[:, j]], 1)
        d[:, BOX + 3 * j:BOX + 3 * j + 3] = np.stack([b_amp[:, j], b_left[:, j], b_w[:, j]], 1)
    for j in range(2):
        d[:, GAUSS + 3 * j:GAUSS + 3 * j + 3] = np.stack([g_amp[:, j], g_c[:, j], g_s[:, j]], 1)
        d[:, TRI + 3 * j:TRI + 3 * j + 3] = np.stack([t_amp[:, j], t_c[:, j], t_h[:, j]], 1)
    d[:, ELL:ELL + 3] = np.concatenate([e_amp, e_c, e_h], 1)
    return d, fam


def _near(y, c):
    """Nearest-image displacement of y from c, in [-1/2, 1/2)."""
    return np.mod(y - c + 0.5, 1.0) - 0.5


def _tri_H(z):
    """Antiderivative from -inf of max(0, 1 - |z|), z in half-widths."""
    s = np.clip(z, -1.0, 1.0)
    return np.where(s < 0.0, 0.5 * (1.0 + s) ** 2, 1.0 - 0.5 * (1.0 - s) ** 2)


def _ell_H(z):
    """Antiderivative from -inf of sqrt(max(0, 1 - z^2))."""
    s = np.clip(z, -1.0, 1.0)
    return 0.5 * (s * np.sqrt(1.0 - s * s) + np.arcsin(s)) + 0.25 * math.pi


def cell_averages(desc: np.ndarray, n: int, shift) -> np.ndarray:
    """Exact averages over the n cells of [0, 1) of each profile translated by ``shift`` (= a t).

    desc: [B, DESC_LEN]; shift: scalar or [B]. Returns [B, n]."""
    desc = np.atleast_2d(np.asarray(desc, dtype=np.float64))
    B = desc.shape[0]
    s = np.broadcast_to(np.asarray(shift, dtype=np.float64), (B,))
    s = (s - np.floor(s))[:, None]
    dx = 1.0 / n
    xl = np.arange(n)[None, :] * dx - s          # left edges of the translated cells
    xc = xl + 0.5 * dx
    out = np.broadcast_to(desc[:, :1], (B, n)).copy()
    for j in range(3):
        amp, k, ph = (desc[:, SINE + 3 * j + q][:, None] for q in range(3))
        arg = math.pi * k * dx
        sinc = np.sin(arg) / np.where(arg == 0.0, 1.0, arg)
        out += amp * sinc * np.sin(2.0 * math.pi * k * xc + ph)
    for j in range(2):
        amp, c, sg = (desc[:, GAUSS + 3 * j + q][:, None] for q in range(3))
        dl = _near(xl, c)
        r = 1.0 / (sg * math.sqrt(2.0))
        hi = np.minimum(dl + dx, 0.5)  # the nearest-image form jumps at distance 1/2
        wrap = np.where(dl + dx > 0.5, erf((dl + dx - 1.0) * r) - erf(-0.5 * r), 0.0)
        out += amp * sg * math.sqrt(0.5 * math.pi) * n * (erf(hi * r) - erf(dl * r) + wrap)
    for j in range(2):
        amp, c, h = (desc[:, TRI + 3 * j + q][:, None] for q in range(3))
        dl = _near(xl, c)
        out += amp * h * n * (_tri_H((dl + dx) / h) - _tri_H(dl / h))
    amp, c, h = (desc[:, ELL + q][:, None] for q in range(3))
    dl = _near(xl, c)
    out += amp * h * n * (_ell_H((dl + dx) / h) - _ell_H(dl / h))
    for j in range(3):
        amp, left, w = (desc[:, BOX + 3 * j + q][:, None] for q in range(3))
        c = left + 0.5 * w
        dl = _near(xl, c)
        lo = np.maximum(dl, -0.5 * w)
        hi = np.minimum(dl + dx, 0.5 * w)
        out += amp * n * np.maximum(hi - lo, 0.0)
    return out


def point_values(desc: np.ndarray, x: np.ndarray, shift=0.0) -> np.ndarray:
    """Point values q0(x - shift) of each profile (fvm_profiles.py:87-190), [B, len(x)]."""
    desc = np.atleast_2d(np.asarray(desc, dtype=np.float64))
    B = desc.shape[0]
    s = np.broadcast_to(np.asarray(shift, dtype=np.float64), (B,))[:, None]
    y = np.asarray(x, dtype=np.float64)[None, :] - s
    out = np.broadcast_to(desc[:, :1], (B, y.shape[1])).copy()
    for j in range(3):
        amp, k, ph = (desc[:, SINE + 3 * j + q][:, None] for q in range(3))
        out += amp * np.sin(2.0 * math.pi * k * y + ph)
    for j in range(2):
        amp, c, sg = (desc[:, GAUSS + 3 * j + q][:, None] for q in range(3))
        out += amp * np.exp(-0.5 * (_near(y, c) / sg) ** 2)
    for j in range(2):
        amp, c, h = (desc[:, TRI + 3 * j + q][:, None] for q in range(3))
        out += amp * np.maximum(1.0 - np.abs(_near(y, c)) / h, 0.0)
    amp, c, h = (desc[:, ELL + q][:, None] for q in range(3))
    out += amp * np.sqrt(np.maximum(1.0 - (_near(y, c) / h) ** 2, 0.0))
    for j in range(3):
        amp, left, w = (desc[:, BOX + 3 * j + q][:, None] for q in range(3))
        out += amp * (np.mod(y - left, 1.0) < w)
    return out
