// 2D Euler WENO7 (JS, Z or SR weights) with Shu's fourth-order TVD Runge-Kutta (L and the downwind operator L~),
// sm_100a.
//
// Reference: weno7_point_rk4_shu/point_rk4.py:150-538 with the classical WENO7 helpers of
// weno7_external_clean/warp_weno7_ader4_helpers_classical_only.py:557-855 (betas, face and two-point Gauss
// candidate stencils, optimal weights, characteristic face reconstruction). Layout: padded row-major
// u[ny+8][nx+8][4] FP64 conserved, ghost width 4; ghost cells are not materialised (stencil loads map a padded
// index to its source cell, as apply_boundary_kernel / apply_periodic_boundary_kernel write them).
//
// One right-hand side L(u) (or L~(u), whose interface fluxes take the two Gauss states in swapped order):
//   k7_normal<DIR=1>, <DIR=2>  one thread per face: Roe average of the two cells next to it, the 8 cells
//                              around it projected once, lr=1 of the left cell and lr=2 of the right cell
//   k7_flux<DIR=1>, <DIR=2>    one thread per face: 8 transverse WENO7 stencils on the face values, both
//                              Gauss points from one set of betas, HLLC at each point, f1 + f2
//   k7_rhs                     -1/2 (f_{i+1} - f_i)/dx - 1/2 (g_{j+1} - g_j)/dy on the interior
// Six right-hand sides and four combinations make one Shu RK4 step (point_rk4.py:514-538).
#pragma once
#include <cuda_runtime.h>

#include "adv1d.cuh"
#include "euler2d.cuh"

namespace wsr {
namespace w7 {

constexpr int kG = 4;  // ghost width
constexpr int kBlock7 = 128;
// Resident blocks per SM the WENO7-SR kernels' register budget targets (the FP64 MLP pair is register heavy).
#ifndef WSR_W7SR_MIN_BLOCKS
#define WSR_W7SR_MIN_BLOCKS 4
#endif

__device__ __forceinline__ int map7(int p, int n, int bc) {
  if (bc == BC_TRANSMISSIVE) return p < kG ? kG : (p >= n + kG ? n + kG - 1 : p);
  return p < kG ? p + n : (p >= n + kG ? p - n : p);
}

// Smoothness indicators of the four 4-point substencils (warp_weno7_ader4_helpers_classical_only.py:558-563),
// each polynomial in the reference's term order and rounded operation by operation (no contraction): the
// unnormalised coefficients (up to 17246) cancel to small betas on smooth data, where a fused multiply-add
// would move the weights of the near-linear stencils.
__device__ __forceinline__ double w7_t(double c, double a, double b) { return __dmul_rn(__dmul_rn(c, a), b); }

__device__ __forceinline__ void w7_beta(const double q[7], double b[4]) {
  const double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6];
  double s;
  s = __dsub_rn(w7_t(2107.0, q3, q3), w7_t(9402.0, q4, q3));
  s = __dadd_rn(s, w7_t(7042.0, q3, q5));
  s = __dsub_rn(s, w7_t(1854.0, q3, q6));
  s = __dsub_rn(s, w7_t(17246.0, q4, q5));
  s = __dsub_rn(s, w7_t(3882.0, q5, q6));
  s = __dadd_rn(s, w7_t(11003.0, q4, q4));
  s = __dadd_rn(s, w7_t(7043.0, q5, q5));
  s = __dadd_rn(s, w7_t(547.0, q6, q6));
  b[3] = __dadd_rn(s, w7_t(4642.0, q4, q6));
  s = __dsub_rn(w7_t(267.0, q5, q5), w7_t(1642.0, q5, q4));
  s = __dadd_rn(s, w7_t(1602.0, q5, q3));
  s = __dsub_rn(s, w7_t(494.0, q5, q2));
  s = __dsub_rn(s, w7_t(2522.0, q3, q2));
  s = __dadd_rn(s, w7_t(3443.0, q3, q3));
  s = __dadd_rn(s, w7_t(547.0, q2, q2));
  s = __dsub_rn(s, w7_t(5966.0, q4, q3));
  s = __dadd_rn(s, w7_t(2843.0, q4, q4));
  b[2] = __dadd_rn(s, w7_t(1922.0, q4, q2));
  s = __dsub_rn(w7_t(267.0, q1, q1), w7_t(494.0, q4, q1));
  s = __dsub_rn(s, w7_t(1642.0, q2, q1));
  s = __dadd_rn(s, w7_t(1602.0, q3, q1));
  s = __dsub_rn(s, w7_t(5966.0, q3, q2));
  s = __dadd_rn(s, w7_t(3443.0, q3, q3));
  s = __dsub_rn(s, w7_t(2522.0, q4, q3));
  s = __dadd_rn(s, w7_t(2843.0, q2, q2));
  s = __dadd_rn(s, w7_t(547.0, q4, q4));
  b[1] = __dadd_rn(s, w7_t(1922.0, q4, q2));
  s = __dadd_rn(w7_t(2107.0, q3, q3), w7_t(7042.0, q3, q1));
  s = __dsub_rn(s, w7_t(1854.0, q3, q0));
  s = __dsub_rn(s, w7_t(9402.0, q3, q2));
  s = __dsub_rn(s, w7_t(17246.0, q2, q1));
  s = __dadd_rn(s, w7_t(4642.0, q2, q0));
  s = __dadd_rn(s, w7_t(547.0, q0, q0));
  s = __dsub_rn(s, w7_t(3882.0, q1, q0));
  s = __dadd_rn(s, w7_t(11003.0, q2, q2));
  b[0] = __dadd_rn(s, w7_t(7043.0, q1, q1));
}

// Face candidates (stencil_weno7, dorder 0): location 1..5, four points each.
__device__ __forceinline__ double w7_face(int loc, double a, double b, double c, double d) {
  switch (loc) {
    case 5:
      return 25.0 / 12.0 * a - 23.0 / 12.0 * b + 13.0 / 12.0 * c - 1.0 / 4.0 * d;
    case 4:
      return 1.0 / 4.0 * a + 13.0 / 12.0 * b - 5.0 / 12.0 * c + 1.0 / 12.0 * d;
    case 3:
      return -1.0 / 12.0 * a + 7.0 / 12.0 * b + 7.0 / 12.0 * c - 1.0 / 12.0 * d;
    case 2:
      return 1.0 / 12.0 * a - 5.0 / 12.0 * b + 13.0 / 12.0 * c + 1.0 / 4.0 * d;
    default:
      return -1.0 / 4.0 * a + 13.0 / 12.0 * b - 23.0 / 12.0 * c + 25.0 / 12.0 * d;
  }
}

// Two-point Gauss candidates (stencil_weno7_2gauss, dorder 0): locations 1..4 for the first Gauss point,
// 5..8 for the second, with s = sqrt(3) correctly rounded.
constexpr double kS3 = 1.7320508075688772;
__device__ __forceinline__ double w7_gauss(int loc, double a, double b, double c, double d) {
  constexpr double s = kS3;
  switch (loc) {
    case 1:
      return (-11.0 * s / 216.0) * a + (17.0 * s / 72.0) * b - (35.0 * s / 72.0) * c + ((65.0 * s + 216.0) / 216.0) * d;
    case 2:
      return (7.0 * s / 216.0) * a - (13.0 * s / 72.0) * b + ((7.0 * s + 72.0) / 72.0) * c + (11.0 * s / 216.0) * d;
    case 3:
      return (-11.0 * s / 216.0) * a + ((72.0 - 7.0 * s) / 72.0) * b + (13.0 * s / 72.0) * c - (7.0 * s / 216.0) * d;
    case 4:
      return ((216.0 - 65.0 * s) / 216.0) * a + (35.0 * s / 72.0) * b - (17.0 * s / 72.0) * c + (11.0 * s / 216.0) * d;
    case 5:
      return (11.0 * s / 216.0) * a - (17.0 * s / 72.0) * b + (35.0 * s / 72.0) * c + ((216.0 - 65.0 * s) / 216.0) * d;
    case 6:
      return (-7.0 * s / 216.0) * a + (13.0 * s / 72.0) * b + ((72.0 - 7.0 * s) / 72.0) * c - (11.0 * s / 216.0) * d;
    case 7:
      return (11.0 * s / 216.0) * a + ((7.0 * s + 72.0) / 72.0) * b - (13.0 * s / 72.0) * c + (7.0 * s / 216.0) * d;
    default:
      return ((65.0 * s + 216.0) / 216.0) * a - (35.0 * s / 72.0) * b + (17.0 * s / 72.0) * c - (11.0 * s / 216.0) * d;
  }
}

// JS combination (weno7_lr_scalar): a_k = d_k / (1e-6 + beta_k)^2, value = sum a_k s_k / sum a_k.
__device__ __forceinline__ double w7_combine(const double r[4], const double d[4], const double s[4]) {
  const double a0 = d[0] * r[0] * r[0], a1 = d[1] * r[1] * r[1], a2 = d[2] * r[2] * r[2], a3 = d[3] * r[3] * r[3];
  return (a0 * s[0] + a1 * s[1] + a2 * s[2] + a3 * s[3]) * rcp64(a0 + a1 + a2 + a3);
}

__device__ __forceinline__ void w7_rcp_betas(const double q[7], double r[4]) {
  double b[4];
  w7_beta(q, b);
#pragma unroll
  for (int k = 0; k < 4; ++k) r[k] = rcp64(1.0e-6 + b[k]);
}

// Face value: lr = 1 (right face of the centre cell q[3]) or lr = 2 (left face).
__device__ __forceinline__ double w7_js_face(const double q[7], int lr) {
  double r[4], s[4];
  w7_rcp_betas(q, r);
  const int o = lr == 1 ? 1 : 2;
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_face(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  const double d1[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};
  const double d2[4] = {4.0 / 35.0, 18.0 / 35.0, 12.0 / 35.0, 1.0 / 35.0};
  return w7_combine(r, lr == 1 ? d1 : d2, s);
}

// Both Gauss-point values of one transverse stencil from one set of betas (weno7_gauss_lr_scalar, lr 1, 2).
__device__ __forceinline__ void w7_js_gauss(const double q[7], double& g1, double& g2) {
  double r[4], s[4];
  w7_rcp_betas(q, r);
  constexpr double s3 = kS3;
  const double e0 = 59.0 / 880.0, e1 = 5.0 * s3 / 16632.0, f0 = 381.0 / 880.0, f1 = 587.0 * s3 / 194040.0;
  const double da[4] = {e0 - e1, f0 - f1, f1 + f0, e1 + e0};
  const double db[4] = {e1 + e0, f1 + f0, f0 - f1, e0 - e1};
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_gauss(1 + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  g1 = w7_combine(r, da, s);
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_gauss(5 + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  g2 = w7_combine(r, db, s);
}

// Betas of the WENO-Z module (weno_z_borges_p2_results/weno7_helpers_z.py:557-588): the same quadratic
// forms as w7_beta written as sums of squares with c = 20/3, 260, 781/3, so they stay non-negative.
__device__ __forceinline__ void w7_beta_sq(const double q[7], double b[4]) {
  const double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6];
  constexpr double c0 = 20.0 / 3.0, c1 = 260.0, c2 = 781.0 / 3.0;
  double a0 = -2.0 * q0 + 9.0 * q1 - 18.0 * q2 + 11.0 * q3, a1 = -q0 + 4.0 * q1 - 5.0 * q2 + 2.0 * q3,
         a2 = -q0 + 3.0 * q1 - 3.0 * q2 + q3;
  b[0] = c0 * a0 * a0 + c1 * a1 * a1 + c2 * a2 * a2;
  a0 = q1 - 6.0 * q2 + 3.0 * q3 + 2.0 * q4, a1 = q2 - 2.0 * q3 + q4, a2 = -q1 + 3.0 * q2 - 3.0 * q3 + q4;
  b[1] = c0 * a0 * a0 + c1 * a1 * a1 + c2 * a2 * a2;
  a0 = -2.0 * q2 - 3.0 * q3 + 6.0 * q4 - q5, a1 = q2 - 2.0 * q3 + q4, a2 = -q2 + 3.0 * q3 - 3.0 * q4 + q5;
  b[2] = c0 * a0 * a0 + c1 * a1 * a1 + c2 * a2 * a2;
  a0 = -11.0 * q3 + 18.0 * q4 - 9.0 * q5 + 2.0 * q6, a1 = 2.0 * q3 - 5.0 * q4 + 4.0 * q5 - q6,
  a2 = -q3 + 3.0 * q4 - 3.0 * q5 + q6;
  b[3] = c0 * a0 * a0 + c1 * a1 * a1 + c2 * a2 * a2;
}

// WENO-Z weights of the WENO7 path (weno_z_borges_p2_results/weno7_helpers_z.py:900-957, weight_kind 1):
// betas scaled by 1/240, tau = |-b0 - 3 b1 + 3 b2 + b3|, alpha_k = d_k (1 + (tau / (b_k + h^3))^3),
// w = alpha / sum, value = sum w_k s_k.
__device__ __forceinline__ double w7_z_value(const double b[4], const double d[4], const double s[4], double eps) {
  constexpr double inv240 = 1.0 / 240.0;
  const double b0 = b[0] * inv240, b1 = b[1] * inv240, b2 = b[2] * inv240, b3 = b[3] * inv240;
  const double tau = fabs(-b0 - 3.0 * b1 + 3.0 * b2 + b3);
  const double r0 = tau * rcp64(b0 + eps), r1 = tau * rcp64(b1 + eps), r2 = tau * rcp64(b2 + eps),
               r3 = tau * rcp64(b3 + eps);
  const double a0 = d[0] * (1.0 + r0 * r0 * r0), a1 = d[1] * (1.0 + r1 * r1 * r1), a2 = d[2] * (1.0 + r2 * r2 * r2),
               a3 = d[3] * (1.0 + r3 * r3 * r3);
  const double inv = rcp64(a0 + a1 + a2 + a3);
  return a0 * inv * s[0] + a1 * inv * s[1] + a2 * inv * s[2] + a3 * inv * s[3];
}

// Face value with WENO-Z weights (weno7_lr_scalar_normalized), eps = h^3 of the reconstruction direction.
__device__ __forceinline__ double w7_z_face(const double q[7], int lr, double eps) {
  double b[4], s[4];
  w7_beta_sq(q, b);
  const int o = lr == 1 ? 1 : 2;
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_face(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  const double d1[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};
  const double d2[4] = {4.0 / 35.0, 18.0 / 35.0, 12.0 / 35.0, 1.0 / 35.0};
  return w7_z_value(b, lr == 1 ? d1 : d2, s, eps);
}

__device__ __forceinline__ void w7_z_gauss(const double q[7], double eps, double& g1, double& g2) {
  double b[4], s[4];
  w7_beta_sq(q, b);
  constexpr double s3 = kS3;
  const double e0 = 59.0 / 880.0, e1 = 5.0 * s3 / 16632.0, f0 = 381.0 / 880.0, f1 = 587.0 * s3 / 194040.0;
  const double da[4] = {e0 - e1, f0 - f1, f0 + f1, e0 + e1};
  const double db[4] = {e0 + e1, f0 + f1, f0 - f1, e0 - e1};
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_gauss(1 + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  g1 = w7_z_value(b, da, s, eps);
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_gauss(5 + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  g2 = w7_z_value(b, db, s, eps);
}

// Normal reconstruction, one thread per face.
// DIR=1: face (r, c), r in [1, ny+7), c in [0, nx]: padded row r, cells c..c+7; face between cells c+3 and
//        c+4. Writes out_r[r][c] (lr=1 of cell c+3) and out_l[r][c+1] (lr=2 of cell c+4); arrays [ny+8][nx+2].
// DIR=2: face (r, c), r in [0, ny], c in [1, nx+7): padded column c, cells r..r+7; writes out_r[r][c] and
//        out_l[r+1][c]; arrays [ny+2][nx+8].
// Z = true: WENO-Z weights with eps = h^3 of this direction (eps_n).
template <int DIR, bool Z>
__global__ void __launch_bounds__(kBlock7, 4) k7_normal(const double* __restrict__ u, double* __restrict__ out_l,
                                                       double* __restrict__ out_r, int nx, int ny, int bc, Gas gas,
                                                       double eps_n, const StepCtl* __restrict__ ctl) {
  __shared__ double s_ch[4][8][kBlock7];
  if (ctl->done) return;
  const int t = threadIdx.x;
  const int c = DIR == 1 ? blockIdx.x * kBlock7 + t : blockIdx.x * 32 + (t & 31);
  const int r = DIR == 1 ? blockIdx.y : blockIdx.y * 4 + (t >> 5);
  const int nxt = nx + 2 * kG;
  const bool active = DIR == 1 ? (r >= 1 && r < ny + 7 && c <= nx) : (r <= ny && c >= 1 && c < nx + 7);
  if (!active) return;  // no block-wide synchronisation below: each thread uses its own shared slots
  auto cell = [&](int k) {
    const int pj = DIR == 1 ? r : r + k;
    const int pi = DIR == 1 ? c + k : c;
    return load_cell(u, nxt, map7(pj, ny, bc), map7(pi, nx, bc));
  };
  const RoeJ J = roe_jacobian(cell(3), cell(4), gas);
  {
    const CharL L = char_left<DIR>(J, gas);
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
      const d4 qk = cell(k);
#pragma unroll
      for (int f = 0; f < 4; ++f) s_ch[f][k][t] = project<DIR>(L, f, qk);
    }
  }
#pragma unroll 1
  for (int side = 0; side < 2; ++side) {
    double cf[4];
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
      double q[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) q[k] = s_ch[f][k + side][t];
      cf[f] = Z ? w7_z_face(q, side == 0 ? 1 : 2, eps_n) : w7_js_face(q, side == 0 ? 1 : 2);
    }
    const d4 face = char_to_con<DIR>(cf, J);
    const size_t idx = DIR == 1 ? (size_t)r * (nx + 2) + c + side : (size_t)(r + side) * (nx + 8) + c;
    store_cell(side == 0 ? out_r : out_l, idx, face);
  }
}

// Transverse reconstruction and flux, one thread per face.
// x faces (j, i), j in [0, ny), i in [0, nx]: u_L from xr[j+1..j+7][i], u_R from xl[j+1..j+7][i+1].
// y faces (j, i), j in [0, ny], i in [0, nx): u_L from yr[j][i+1..i+7], u_R from yl[j+1][i+1..i+7].
// Output f[j][i] = F(g1) + F(g2) (unscaled); with `reverse` the Riemann problem takes (u_R, u_L).
// Z = true: WENO-Z weights with eps = h^3 of the transverse direction (eps_t).
template <int DIR, bool Z>
__global__ void __launch_bounds__(kBlock7, 4) k7_flux(const double* __restrict__ fl, const double* __restrict__ fr,
                                                     double* __restrict__ fout, int nx, int ny, Gas gas, int reverse,
                                                     double eps_t, const StepCtl* __restrict__ ctl) {
  if (ctl->done) return;
  const int t = threadIdx.x;
  const int i = DIR == 1 ? blockIdx.x * 32 + (t & 31) : blockIdx.x * kBlock7 + t;
  const int j = DIR == 1 ? blockIdx.y * 4 + (t >> 5) : blockIdx.y;
  const int nfx = DIR == 1 ? nx + 1 : nx, nfy = DIR == 1 ? ny : ny + 1;
  if (i >= nfx || j >= nfy) return;
  d4 l1, l2, r1, r2;
#pragma unroll 1
  for (int n = 0; n < 8; ++n) {
    const int comp = n >> 1, side = n & 1;  // side 0: u_L from fr, side 1: u_R from fl
    double q[7];
    const double* src = side == 0 ? fr : fl;
    if (DIR == 1) {
      const int ncols = nx + 2, col = side == 0 ? i : i + 1;
#pragma unroll
      for (int k = 0; k < 7; ++k) q[k] = __ldg(src + ((size_t)(j + 1 + k) * ncols + col) * 4 + comp);
    } else {
      const int ncols = nx + 8, row = side == 0 ? j : j + 1;
#pragma unroll
      for (int k = 0; k < 7; ++k) q[k] = __ldg(src + ((size_t)row * ncols + (i + 1 + k)) * 4 + comp);
    }
    double g1, g2;
    if (Z)
      w7_z_gauss(q, eps_t, g1, g2);
    else
      w7_js_gauss(q, g1, g2);
    if (side == 0) {
      l1.v[comp] = g1;
      l2.v[comp] = g2;
    } else {
      r1.v[comp] = g1;
      r2.v[comp] = g2;
    }
  }
  const d4 f1 = reverse ? hllc_flux<DIR>(r1, l1, gas) : hllc_flux<DIR>(l1, r1, gas);
  const d4 f2 = reverse ? hllc_flux<DIR>(r2, l2, gas) : hllc_flux<DIR>(l2, r2, gas);
  d4 o;
#pragma unroll
  for (int k = 0; k < 4; ++k) o.v[k] = f1.v[k] + f2.v[k];
  store_cell(fout, (size_t)j * nfx + i, o);
}

// ---------------------------------------------------------------------------------------------
// WENO7-SR (FP64 closure). Betas come from the reflection-symmetric WENO7 MLP (6 -> 24 -> 16 -> 16 -> 4;
// features, plateau test and model as in the 1D path), beta = 4 ratio, all ones on a plateau
// (teacherfree_lab_weno7_rk4_distance_balanced_fast/warp_sod/beta_provider.py:27-33). The lr = 2 face value
// and the second Gauss point take the betas of the flipped stencil, flipped back (beta_provider.py:164-219).
// Weights alpha_k = d_k / (beta_k + 1e-12)^2, normalised by max(sum, 1e-300) with divisions
// (warp_sod/warp_weno7_external_overwrite_fullall.py:67-143).
//
// Closure work is compacted per block as in the WENO5-SR kernels: phase A forms every stencil's plateau
// test and reconstructs plateau stencils at once; the others are queued in shared memory and phase B runs
// the MLP pair over the queue at full SIMT width. Each block adds its queue length (the closure evaluations
// it ran) to *counters with one atomic.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double w7sr_combine(const double s[4], const double d[4], const double b[4]) {
  double a[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double ib = 1.0 / (b[k] + 1.0e-12);
    a[k] = d[k] * ib * ib;
  }
  const double m = fmax(a[0] + a[1] + a[2] + a[3], 1.0e-300);
  return a[0] / m * s[0] + a[1] / m * s[1] + a[2] / m * s[2] + a[3] / m * s[3];
}

// Face value of the stencil q (cells in order) for head lr with betas b.
__device__ __forceinline__ double w7sr_face(const double q[7], int lr, const double b[4]) {
  double s[4];
  const int o = lr == 1 ? 1 : 2;
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_face(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  const double d1[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};
  const double d2[4] = {4.0 / 35.0, 18.0 / 35.0, 12.0 / 35.0, 1.0 / 35.0};
  return w7sr_combine(s, lr == 1 ? d1 : d2, b);
}

// Gauss-point value (loca 1 or 2) of the stencil q with betas b.
__device__ __forceinline__ double w7sr_gauss(const double q[7], int loca, const double b[4]) {
  double s[4];
  constexpr double s3 = kS3;
  const double e0 = 59.0 / 880.0, e1 = 5.0 * s3 / 16632.0, f0 = 381.0 / 880.0, f1 = 587.0 * s3 / 194040.0;
  const double da[4] = {e0 - e1, f0 - f1, f0 + f1, e0 + e1};
  const double db[4] = {e0 + e1, f0 + f1, f0 - f1, e0 - e1};
  const int o = loca == 1 ? 1 : 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) s[k] = w7_gauss(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
  return w7sr_combine(s, loca == 1 ? da : db, b);
}

// FP64 exponential of the closure's swish and softmax, after Tang's table-driven method (P. T. P. Tang,
// ACM TOMS 15(2), 1989): x = (32 m + j) ln2/32 + r with |r| <= ln2/64, exp(x) = 2^m 2^(j/32) (1 + p(r)), p the
// degree-6 Taylor polynomial of e^r - 1 (truncation below 4e-18 on that interval), ln2/32 split in two parts for
// the reduction. t32[j] = 2^(j/32) rounded to double (kExp2_32, copied to shared memory by each block). Error
// about 1 ulp; arguments are clamped to [-700, 700], which keeps every result normal (the swish of an argument
// beyond that range is z or 0 to within 1e-300).
__constant__ double kExp2_32[32] = {
    1.0, 1.0218971486541166, 1.0442737824274138, 1.0671404006768237,
    1.0905077326652577, 1.1143867425958924, 1.1387886347566916, 1.1637248587775775,
    1.189207115002721, 1.215247359980469, 1.241857812073484, 1.2690509571917332,
    1.2968395546510096, 1.3252366431597413, 1.3542555469368927, 1.383909881963832,
    1.4142135623730951, 1.4451808069770467, 1.4768261459394993, 1.5091644275934228,
    1.5422108254079407, 1.5759808451078865, 1.6104903319492543, 1.645755478153965,
    1.681792830507429, 1.718619298122478, 1.7562521603732995, 1.7947090750031072,
    1.8340080864093424, 1.8741676341103, 1.9152065613971474, 1.9571441241754002};

__device__ __forceinline__ double exp_tab(double x, const double* __restrict__ t32) {
  x = x < -700.0 ? -700.0 : (x > 700.0 ? 700.0 : x);  // NaN passes through (fmin/fmax would drop it)
  constexpr double kShift = 6755399441055744.0;  // 1.5 * 2^52: x 32/ln2 + kShift holds round(x 32/ln2) in its low word
  constexpr double kInvL = 46.16624130844683, kL1 = 0.02166084939249829, kL2 = 7.247021293269686e-19;
  const double kd = fma(x, kInvL, kShift);
  const int n = __double2loint(kd);
  const double nd = kd - kShift;
  double r = fma(nd, -kL1, x);
  r = fma(nd, -kL2, r);
  double p = fma(r, 1.0 / 720.0, 1.0 / 120.0);
  p = fma(p, r, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = p * r;
  const double tj = t32[n & 31];
  const double e = fma(tj, p, tj);
  return __hiloint2double(__double2hiint(e) + ((n >> 5) << 20), __double2loint(e));
}

__device__ __forceinline__ double swish_tab(double z, const double* __restrict__ t32) {
  return z * rcp64(1.0 + exp_tab(-z, t32));
}

// Dense layer of the WENO7 MLP for the direct (xa) and reflected (xb) inputs together; packed [in][out]
// weights followed by the biases (the layout of the 1D path).
// The multiply-adds are unrolled (the weights stay constant-bank operands); the activations run in a rolled loop
// per layer, so the exp/reciprocal sequence is in the code once per layer instead of once per neuron: with 112
// inlined copies per closure, instruction fetch was the kernels' first stall (63.5 against 79.6 ms per 1024^2
// step).
template <int NI, int NO>
__device__ __forceinline__ void w7sr_dense_pair(const double* __restrict__ P, int w, int b, const double* xa,
                                                const double* xb, double* ya, double* yb, bool act,
                                                const double* __restrict__ t32) {
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    double za = P[b + o], zb = P[b + o];
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      za = za + xa[k] * P[w + k * NO + o];
      zb = zb + xb[k] * P[w + k * NO + o];
    }
    ya[o] = za;
    yb[o] = zb;
  }
  if (act) {
#pragma unroll 1
    for (int o = 0; o < NO; ++o) {
      ya[o] = swish_tab(ya[o], t32);
      yb[o] = swish_tab(yb[o], t32);
    }
  }
}

// MLP 6 -> 24 -> 16 -> 16 -> 4 (swish, swish, swish, 6 tanh(raw/6), softmax; weno7_core.py:311-318) on the
// direct and reflected features, ratios out.
__device__ __forceinline__ void w7sr_pair(const double* __restrict__ P, const double* __restrict__ t32,
                                          const double xa[6], const double xb[6], double ra[4], double rb[4]) {
  using D = MlpDims<6, 24, 16, 16, 4>;
  double a1[24], b1[24], a2[16], b2[16], a3[16], b3[16], za[4], zb[4];
  w7sr_dense_pair<6, 24>(P, D::W1, D::B1, xa, xb, a1, b1, true, t32);
  w7sr_dense_pair<24, 16>(P, D::W2, D::B2, a1, b1, a2, b2, true, t32);
  w7sr_dense_pair<16, 16>(P, D::W3, D::B3, a2, b2, a3, b3, true, t32);
  w7sr_dense_pair<16, 4>(P, D::W4, D::B4, a3, b3, za, zb, false, t32);
  double ma = -1e30, mb = -1e30;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    za[o] = 6.0 * tanh(div6(za[o]));
    zb[o] = 6.0 * tanh(div6(zb[o]));
    ma = za[o] > ma ? za[o] : ma;
    mb = zb[o] > mb ? zb[o] : mb;
  }
  double sa = 0.0, sb = 0.0;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    za[o] = exp_tab(za[o] - ma, t32);
    zb[o] = exp_tab(zb[o] - mb, t32);
    sa = sa + za[o];
    sb = sb + zb[o];
  }
  const double ia = rcp64(sa), ib = rcp64(sb);
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    ra[o] = za[o] * ia;
    rb[o] = zb[o] * ib;
  }
}

// Closure betas of the stencil c (already in closure order: flipped for the second side); `flip` maps them
// back to the stencil's own order. beta = 4 (direct + reflect(reflected)) / 2 (weno7_core.py:320-324).
__device__ __forceinline__ void w7sr_betas(const double c[7], bool flip, const Mlp7d& P,
                                           const double* __restrict__ t32, double b[4]) {
  double d[4], dmax, qs, f[6], ra[4], rb[4];
  adv_plateau<7>(c, d, dmax, qs);
  adv_features<7>(c, d, dmax, qs, f);
  const double fr[6] = {f[3], f[2], f[1], f[0], f[4], f[5]};
  w7sr_pair(P.p, t32, f, fr, ra, rb);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int o = flip ? 3 - k : k;
    b[k] = 4.0 * (0.5 * (ra[o] + rb[3 - o]));
  }
}

// exp_tab over an array (the probe that checks it against CUDA's exp).
__global__ void k_probe_exp_tab(const double* __restrict__ x, double* __restrict__ out, int n) {
  __shared__ double t32[32];
  if (threadIdx.x < 32) t32[threadIdx.x] = kExp2_32[threadIdx.x];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = exp_tab(x[i], t32);
}

// Normal reconstruction, one thread per face, same faces and outputs as k7_normal. Stencil n = 2 f + side:
// characteristic field f; side 0 -> cells 0..6, head lr = 1; side 1 -> cells 1..7, head lr = 2, closure on the
// flipped cells 7..1.
template <int DIR>
__global__ void __launch_bounds__(kBlock7, WSR_W7SR_MIN_BLOCKS) k7s_normal(const double* __restrict__ u, double* __restrict__ out_l,
                                                        double* __restrict__ out_r, int nx, int ny, int bc, Gas gas,
                                                        const StepCtl* __restrict__ ctl,
                                                        unsigned long long* __restrict__ counters, int opts,
                                                        unsigned long long* __restrict__ fallbacks,
                                                        const __grid_constant__ Mlp7d P) {
  __shared__ double s_ch[4][8][kBlock7];
  __shared__ double s_val[8][kBlock7];
  __shared__ double s_t32[32];
  __shared__ unsigned short s_q[8 * kBlock7];
  __shared__ int s_count;
  if (ctl->done) return;  // uniform across the launch
  const int t = threadIdx.x;
  if (t < 32) s_t32[t] = kExp2_32[t];
  const int c = DIR == 1 ? blockIdx.x * kBlock7 + t : blockIdx.x * 32 + (t & 31);
  const int r = DIR == 1 ? blockIdx.y : blockIdx.y * 4 + (t >> 5);
  const int nxt = nx + 2 * kG;
  const bool active = DIR == 1 ? (r >= 1 && r < ny + 7 && c <= nx) : (r <= ny && c >= 1 && c < nx + 7);
  if (t == 0) s_count = 0;
  int fb = 0;  // JS fallbacks taken by this thread
  RoeJ J;
  if (active) {
    auto cell = [&](int k) {
      const int pj = DIR == 1 ? r : r + k;
      const int pi = DIR == 1 ? c + k : c;
      return load_cell(u, nxt, map7(pj, ny, bc), map7(pi, nx, bc));
    };
    J = roe_jacobian(cell(3), cell(4), gas);
    const CharL L = char_left<DIR>(J, gas);
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
      const d4 qk = cell(k);
#pragma unroll
      for (int f = 0; f < 4; ++f) s_ch[f][k][t] = project<DIR>(L, f, qk);
    }
  }
  __syncthreads();
  // Phase A
#pragma unroll 1
  for (int n = 0; n < 8; ++n) {
    const int f = n >> 1, side = n & 1;
    bool need = false;
    if (active) {
      double q[7], cq[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) q[k] = s_ch[f][k + side][t];
#pragma unroll
      for (int k = 0; k < 7; ++k) cq[k] = side ? q[6 - k] : q[k];
      need = !adv_plateau_test<7>(cq);
      if (!need) {
        const double one[4] = {1.0, 1.0, 1.0, 1.0};
        s_val[n][t] = w7sr_face(q, side + 1, one);
      }
    }
    queue_push(need, n * kBlock7 + t, s_q, &s_count);
  }
  __syncthreads();
  // Phase B
  const int count = s_count;
#pragma unroll 1
  for (int e = t; e < count; e += kBlock7) {
    const int id = s_q[e];
    const int n = id / kBlock7, o = id % kBlock7, f = n >> 1, side = n & 1;
    double q[7], cq[7], b[4];
#pragma unroll
    for (int k = 0; k < 7; ++k) q[k] = s_ch[f][k + side][o];
#pragma unroll
    for (int k = 0; k < 7; ++k) cq[k] = side ? q[6 - k] : q[k];
    w7sr_betas(cq, side == 1, P, s_t32, b);
    if ((opts & OPT_JS_FALLBACK) && !(isfinite(b[0]) && isfinite(b[1]) && isfinite(b[2]) && isfinite(b[3]))) {
      s_val[n][o] = w7_js_face(q, side + 1);  // the closure's betas are not finite: WENO7-JS weights
      ++fb;
    } else {
      s_val[n][o] = w7sr_face(q, side + 1, b);
    }
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const double cf[4] = {s_val[side][t], s_val[2 + side][t], s_val[4 + side][t], s_val[6 + side][t]};
      d4 face = char_to_con<DIR>(cf, J);
      if ((opts & OPT_JS_FALLBACK) && !admissible(face, gas.g)) {
        // positivity fallback: this face value again, all four fields with WENO7-JS weights
        double jf[4];
#pragma unroll 1
        for (int f = 0; f < 4; ++f) {
          double q[7];
#pragma unroll
          for (int k = 0; k < 7; ++k) q[k] = s_ch[f][k + side][t];
          jf[f] = w7_js_face(q, side + 1);
        }
        face = char_to_con<DIR>(jf, J);
        ++fb;
      }
      const size_t idx = DIR == 1 ? (size_t)r * (nx + 2) + c + side : (size_t)(r + side) * (nx + 8) + c;
      store_cell(side == 0 ? out_r : out_l, idx, face);
    }
  }
  if (t == 0 && count) atomicAdd(counters, (unsigned long long)count);
  if (fb) atomicAdd(fallbacks, (unsigned long long)fb);
}

// Transverse stencil m = 2 comp + side of face (i, j) (side 0: u_L from fr, side 1: u_R from fl), the
// layout of k7_flux.
template <int DIR>
__device__ __forceinline__ void w7_load_transverse(const double* __restrict__ fl, const double* __restrict__ fr,
                                                   int nx, int i, int j, int m, double q[7]) {
  const int comp = m >> 1, side = m & 1;
  const double* src = side == 0 ? fr : fl;
  if (DIR == 1) {
    const int ncols = nx + 2, col = side == 0 ? i : i + 1;
#pragma unroll
    for (int k = 0; k < 7; ++k) q[k] = __ldg(src + ((size_t)(j + 1 + k) * ncols + col) * 4 + comp);
  } else {
    const int ncols = nx + 8, row = side == 0 ? j : j + 1;
#pragma unroll
    for (int k = 0; k < 7; ++k) q[k] = __ldg(src + ((size_t)row * ncols + (i + 1 + k)) * 4 + comp);
  }
}

// Transverse reconstruction and flux, one thread per face, same faces and outputs as k7_flux. Job
// n = 2 m + gp: transverse stencil m, Gauss point gp + 1 (the second from the flipped stencil's closure).
template <int DIR>
__global__ void __launch_bounds__(kBlock7, WSR_W7SR_MIN_BLOCKS) k7s_flux(const double* __restrict__ fl, const double* __restrict__ fr,
                                                      double* __restrict__ fout, int nx, int ny, Gas gas, int reverse,
                                                      const StepCtl* __restrict__ ctl,
                                                      unsigned long long* __restrict__ counters, int opts,
                                                      unsigned long long* __restrict__ fallbacks,
                                                      const __grid_constant__ Mlp7d P) {
  __shared__ double s_g[16][kBlock7];
  __shared__ double s_t32[32];
  __shared__ unsigned short s_q[16 * kBlock7];
  __shared__ int s_count;
  if (ctl->done) return;  // uniform across the launch
  const int t = threadIdx.x;
  if (t < 32) s_t32[t] = kExp2_32[t];
  auto face_i = [&](int th) { return DIR == 1 ? (int)blockIdx.x * 32 + (th & 31) : (int)blockIdx.x * kBlock7 + th; };
  auto face_j = [&](int th) { return DIR == 1 ? (int)blockIdx.y * 4 + (th >> 5) : (int)blockIdx.y; };
  const int i = face_i(t), j = face_j(t);
  const int nfx = DIR == 1 ? nx + 1 : nx, nfy = DIR == 1 ? ny : ny + 1;
  const bool active = i < nfx && j < nfy;
  if (t == 0) s_count = 0;
  int fb = 0;  // JS fallbacks taken by this thread
  __syncthreads();
  // Phase A
#pragma unroll 1
  for (int m = 0; m < 8; ++m) {
    double q[7];
    if (active) w7_load_transverse<DIR>(fl, fr, nx, i, j, m, q);
#pragma unroll 1
    for (int gp = 0; gp < 2; ++gp) {
      bool need = false;
      if (active) {
        double cq[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) cq[k] = gp ? q[6 - k] : q[k];
        need = !adv_plateau_test<7>(cq);
        if (!need) {
          const double one[4] = {1.0, 1.0, 1.0, 1.0};
          s_g[2 * m + gp][t] = w7sr_gauss(q, gp + 1, one);
        }
      }
      queue_push(need, (2 * m + gp) * kBlock7 + t, s_q, &s_count);
    }
  }
  __syncthreads();
  // Phase B
  const int count = s_count;
#pragma unroll 1
  for (int e = t; e < count; e += kBlock7) {
    const int id = s_q[e];
    const int n = id / kBlock7, o = id % kBlock7, m = n >> 1, gp = n & 1;
    double q[7], cq[7], b[4];
    w7_load_transverse<DIR>(fl, fr, nx, face_i(o), face_j(o), m, q);
#pragma unroll
    for (int k = 0; k < 7; ++k) cq[k] = gp ? q[6 - k] : q[k];
    w7sr_betas(cq, gp == 1, P, s_t32, b);
    if ((opts & OPT_JS_FALLBACK) && !(isfinite(b[0]) && isfinite(b[1]) && isfinite(b[2]) && isfinite(b[3]))) {
      double g1, g2;  // the closure's betas are not finite: WENO7-JS weights
      w7_js_gauss(q, g1, g2);
      s_g[n][o] = gp ? g2 : g1;
      ++fb;
    } else {
      s_g[n][o] = w7sr_gauss(q, gp + 1, b);
    }
  }
  __syncthreads();
  if (active) {
    d4 l1, l2, r1, r2;
#pragma unroll
    for (int comp = 0; comp < 4; ++comp) {
      l1.v[comp] = s_g[4 * comp + 0][t];
      l2.v[comp] = s_g[4 * comp + 1][t];
      r1.v[comp] = s_g[4 * comp + 2][t];
      r2.v[comp] = s_g[4 * comp + 3][t];
    }
    const d4 f1 = reverse ? hllc_flux<DIR>(r1, l1, gas) : hllc_flux<DIR>(l1, r1, gas);
    const d4 f2 = reverse ? hllc_flux<DIR>(r2, l2, gas) : hllc_flux<DIR>(l2, r2, gas);
    d4 o;
#pragma unroll
    for (int k = 0; k < 4; ++k) o.v[k] = f1.v[k] + f2.v[k];
    store_cell(fout, (size_t)j * nfx + i, o);
  }
  if (t == 0 && count) atomicAdd(counters, (unsigned long long)count);
  if (fb) atomicAdd(fallbacks, (unsigned long long)fb);
}

// rhs[j][i] = -1/2 (f[j][i+1] - f[j][i]) / dx - 1/2 (g[j+1][i] - g[j][i]) / dy (point_rk4.py:290-312).
__global__ void __launch_bounds__(256) k7_rhs(const double* __restrict__ fx, const double* __restrict__ fy,
                                              double* __restrict__ rhs, int nx, int ny, double inv_dx, double inv_dy,
                                              const StepCtl* __restrict__ ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (ctl->done || i >= nx) return;
  const d4 fxl = load_cell(fx, nx + 1, j, i), fxr = load_cell(fx, nx + 1, j, i + 1);
  const d4 fyb = load_cell(fy, nx, j, i), fyt = load_cell(fy, nx, j + 1, i);
  d4 o;
#pragma unroll
  for (int k = 0; k < 4; ++k) o.v[k] = -0.5 * (fxr.v[k] - fxl.v[k]) * inv_dx - 0.5 * (fyt.v[k] - fyb.v[k]) * inv_dy;
  store_cell(rhs, (size_t)j * nx + i, o);
}

// Shu RK4 combinations on the interior (point_rk4.py:315-403), in the reference's coefficient and operand
// order; rhs arrays are interior-only [ny][nx][4], states padded.
struct ShuArgs {
  const double* u;
  const double* u1;
  const double* u2;
  const double* u3;
  const double* rhs0;
  const double* rhs_t0;
  const double* rhs1;
  const double* rhs_t1;
  const double* rhs2;
  const double* rhs3;
  double* out;
};

template <int S>
__global__ void __launch_bounds__(256) k7_shu(ShuArgs a, int nx, int ny, const StepCtl* __restrict__ ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (ctl->done || i >= nx) return;
  const double dt = ctl->dt;
  const int nxt = nx + 2 * kG;
  const size_t p = (size_t)(j + kG) * nxt + (i + kG);
  const d4 u0 = load_cell(a.u, nxt, j + kG, i + kG);
  d4 o;
  if constexpr (S == 1) {
    const d4 r0 = load_cell(a.rhs0, nx, j, i);
#pragma unroll
    for (int k = 0; k < 4; ++k) o.v[k] = u0.v[k] + 0.5 * dt * r0.v[k];
  } else if constexpr (S == 2) {
    const d4 rt0 = load_cell(a.rhs_t0, nx, j, i), v1 = load_cell(a.u1, nxt, j + kG, i + kG);
    const d4 r1 = load_cell(a.rhs1, nx, j, i);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      o.v[k] = 649.0 / 1600.0 * u0.v[k] - 10890423.0 / 25193600.0 * dt * rt0.v[k] + 951.0 / 1600.0 * v1.v[k] +
               5000.0 / 7873.0 * dt * r1.v[k];
  } else if constexpr (S == 3) {
    const d4 rt0 = load_cell(a.rhs_t0, nx, j, i), v1 = load_cell(a.u1, nxt, j + kG, i + kG);
    const d4 rt1 = load_cell(a.rhs_t1, nx, j, i), v2 = load_cell(a.u2, nxt, j + kG, i + kG);
    const d4 r2 = load_cell(a.rhs2, nx, j, i);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      o.v[k] = 53989.0 / 2500000.0 * u0.v[k] - 102261.0 / 5000000.0 * dt * rt0.v[k] +
               4806213.0 / 20000000.0 * v1.v[k] - 5121.0 / 20000.0 * dt * rt1.v[k] + 23619.0 / 32000.0 * v2.v[k] +
               7873.0 / 10000.0 * dt * r2.v[k];
  } else {
    const d4 r0 = load_cell(a.rhs0, nx, j, i), v1 = load_cell(a.u1, nxt, j + kG, i + kG);
    const d4 r1 = load_cell(a.rhs1, nx, j, i), v2 = load_cell(a.u2, nxt, j + kG, i + kG);
    const d4 v3 = load_cell(a.u3, nxt, j + kG, i + kG), r3 = load_cell(a.rhs3, nx, j, i);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      o.v[k] = 1.0 / 5.0 * u0.v[k] + 1.0 / 10.0 * dt * r0.v[k] + 6127.0 / 30000.0 * v1.v[k] +
               1.0 / 6.0 * dt * r1.v[k] + 7873.0 / 30000.0 * v2.v[k] + 1.0 / 3.0 * v3.v[k] + 1.0 / 6.0 * dt * r3.v[k];
  }
  store_cell(a.out, p, o);
}

// Max wave speed of the interior (compute_max_speed_kernel, classical_only.py:2147-2159).
__global__ void __launch_bounds__(256) k7_max_speed(const double* __restrict__ u, int nx, int ny, double g,
                                                    StepCtl* __restrict__ ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (ctl->done) return;
  unsigned long long sb = 0;
  if (i < nx) sb = speed_bits(load_cell(u, nx + 2 * kG, j + kG, i + kG), g);
  block_max_to(sb, &ctl->max_speed_bits);
}

// dt of the next step (point_rk4.py:136-147, 568-590): cfl min(dx, dy) / max speed (1e10 below 1e-15),
// the loop runs while t < t_end and a step that would pass t_end is shortened to reach it. Resets the
// max-speed slot for the next step. `ring` records each step's dt (slot steps mod ring_len).
__global__ void k7_step_begin(StepCtl* ctl, double* ring, int ring_len) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ctl->done) return;
  if (!(ctl->t < ctl->t_end) || ctl->steps >= ctl->max_steps) {
    ctl->done = 1;
    return;
  }
  const double ms = __longlong_as_double((long long)ctl->max_speed_bits);
  double dt = ms < 1.0e-15 ? 1.0e10 : ctl->cfl * ctl->hmin / ms;
  if (ctl->t + dt > ctl->t_end) dt = ctl->t_end - ctl->t;
  if (!(dt > 0.0)) {
    ctl->done = 1;
    return;
  }
  ctl->dt = dt;
  ctl->max_speed_bits = 0ull;
  ring[ctl->steps % ring_len] = dt;
}

}  // namespace w7
}  // namespace wsr
