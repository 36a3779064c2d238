// Batched 1D periodic linear advection u_t + a u_x = 0 with WENO5 / WENO7 reconstruction (JS, WENO-Z or
// SR closure), SSPRK3 or Shu's fourth-order TVD Runge-Kutta with the downwind operator, sm_100a.
//
// Reference (code/snapshot/): teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/
// rk3_advection.py:82-186 (signed upwind face state, rhs, SSPRK3, CFL schedule), weno5_core.py:158-239;
// teacherfree_lab_weno7_rk4_distance_balanced_fast/weno7_core.py:28-324 (WENO7 candidates, weights,
// delta forms, features, MLP 6->24->16->16->4) and rk4_advection.py:31-220 (face states, L and L~, Shu RK4);
// for_paper_results/run_gste.py:103-118 (uniform GSTE schedule); weno_z_borges_p2_results/torch_weno_z.py:14-79
// (WENO5-Z p = 2, eps = h^2, tau5 = |b0 - b2|; WENO7-Z p = 3, eps = h^3, tau7 = |-b0 - 3 b1 + 3 b2 + b3|).
//
// One CTA per trajectory keeps the whole trajectory in shared memory for all of its steps: trajectories
// are independent, so there is no global synchronisation between steps, and ragged lengths and step
// counts cost nothing extra. Trajectories may be visited in a caller-given order (longest first).
// Closure evaluations of a right-hand side are compacted per CTA exactly as in the 2D kernels: plateau
// stencils take the linear weights in phase A, the others are queued and evaluated densely in phase B.
#pragma once
#include <cuda_runtime.h>

#include "closure.cuh"

namespace wsr {

constexpr int kAdvThreads = 256;
constexpr int kAdvNmax = 2048;

// ---------------------------------------------------------------------------------------------
// Generic MLP I -> H1 -> H2 -> H3 -> O (swish, swish, swish, 6 tanh(raw/6), softmax), packed
// [in][out] row-major weights followed by biases per layer; direct and reflected inputs together.
// ---------------------------------------------------------------------------------------------
template <int I, int H1, int H2, int H3, int O>
struct MlpDims {
  static constexpr int W1 = 0, B1 = W1 + I * H1, W2 = B1 + H1, B2 = W2 + H1 * H2, W3 = B2 + H2, B3 = W3 + H2 * H3,
                       W4 = B3 + H3, B4 = W4 + H3 * O, N = B4 + O;
};

template <typename T, bool BF16, int NI, int NO>
__device__ __forceinline__ void dense_pair(const T* __restrict__ P, int w, int b, const T* xa, const T* xb, T* ya,
                                           T* yb, bool act) {
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    T za = P[b + o], zb = P[b + o];
#pragma unroll
    for (int k = 0; k < NI; ++k) {
      za = za + xa[k] * P[w + k * NO + o];
      zb = zb + xb[k] * P[w + k * NO + o];
    }
    if (act && !kRollActAlways<T>) {
      za = swish<T>(za);
      zb = swish<T>(zb);
      if (BF16) {
        za = bf16r(za);
        zb = bf16r(zb);
      }
    }
    ya[o] = za;
    yb[o] = zb;
  }
  if (act) swish_rolled<T, kRollActAlways<T>>(ya, yb, NO);
}

template <typename T, bool BF16, int I, int H1, int H2, int H3, int O>
__device__ __forceinline__ void mlp_pair_g(const T* __restrict__ P, const T* xa, const T* xb, T* ra, T* rb) {
  using D = MlpDims<I, H1, H2, H3, O>;
  T a1[H1], b1[H1], a2[H2], b2[H2], a3[H3], b3[H3], za[O], zb[O];
  dense_pair<T, BF16, I, H1>(P, D::W1, D::B1, xa, xb, a1, b1, true);
  dense_pair<T, BF16, H1, H2>(P, D::W2, D::B2, a1, b1, a2, b2, true);
  dense_pair<T, BF16, H2, H3>(P, D::W3, D::B3, a2, b2, a3, b3, true);
  dense_pair<T, BF16, H3, O>(P, D::W4, D::B4, a3, b3, za, zb, false);
  T ma = T(-1e30), mb = T(-1e30);
#pragma unroll
  for (int o = 0; o < O; ++o) {
    za[o] = T(6) * tanh_t(div6(za[o]));
    zb[o] = T(6) * tanh_t(div6(zb[o]));
    ma = za[o] > ma ? za[o] : ma;
    mb = zb[o] > mb ? zb[o] : mb;
  }
  T sa = T(0), sb = T(0);
#pragma unroll
  for (int o = 0; o < O; ++o) {
    za[o] = exp_t(za[o] - ma);
    zb[o] = exp_t(zb[o] - mb);
    sa = sa + za[o];
    sb = sb + zb[o];
  }
  const T ia = rcp_t(sa), ib = rcp_t(sb);
#pragma unroll
  for (int o = 0; o < O; ++o) {
    ra[o] = za[o] * ia;
    rb[o] = zb[o] * ib;
  }
}

// Closure parameter blocks for WENO7.
constexpr int kParams7 = MlpDims<6, 24, 16, 16, 4>::N;  // 908
struct Mlp7d {
  double p[kParams7];
};
struct Mlp7f {
  float p[kParams7];
};

template <int SCHEME, int M>
struct AdvParams {
  using type = typename ClosureParams<M>::type;
};
template <>
struct AdvParams<7, M_SR64> {
  using type = Mlp7d;
};
template <>
struct AdvParams<7, M_SR32> {
  using type = Mlp7f;
};
template <>
struct AdvParams<7, M_SRBF16> {
  using type = Mlp7f;
};

// ---------------------------------------------------------------------------------------------
// Scheme descriptions
// ---------------------------------------------------------------------------------------------
template <int SCHEME>
struct Weno;

template <>
struct Weno<5> {
  static constexpr int W = 5, R = 3, NF = 5;
  static constexpr double BSCALE = 3.0, SCALE_OFF = 4.0;
  __device__ static void deltas(const double q[5], double d[3]) {
    const Sens s = sensors5(q);
    d[0] = s.d0;
    d[1] = s.d1;
    d[2] = s.d2;
  }
  __device__ static void lin(int lr, double d[3]) {
    if (lr == 1) {
      d[0] = 0.1; d[1] = 0.6; d[2] = 0.3;
    } else {
      d[0] = 0.3; d[1] = 0.6; d[2] = 0.1;
    }
  }
  __device__ static void cand(const double q[5], int lr, double s[3]) { candidates(q, lr == 1 ? 0 : 1, s); }
  __device__ static void js_beta(const double q[5], double b[3]) {
    const double t2 = q[2] - 2.0 * q[3] + q[4], u2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
    const double t1 = q[1] - 2.0 * q[2] + q[3], u1 = q[1] - q[3];
    const double t0 = q[0] - 2.0 * q[1] + q[2], u0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
    b[0] = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
    b[1] = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
    b[2] = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
  }
  // WENO-Z factors g_k = 1 + (tau5 / (b_k + h^2))^2 (torch_weno_z.py:14-20)
  __device__ static void z_factors(const double q[5], double h, double g[3]) {
    double b[3];
    js_beta(q, b);
    const double tau = fabs(b[0] - b[2]), eps = h * h;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double r = tau / (b[k] + eps);
      g[k] = 1.0 + r * r;
    }
  }
};

template <>
struct Weno<7> {
  static constexpr int W = 7, R = 4, NF = 6;
  static constexpr double BSCALE = 4.0, SCALE_OFF = 16.0;
  __device__ static void forms(const double q[7], double f[4][3]) {
    f[0][0] = -2.0 * q[0] + 9.0 * q[1] - 18.0 * q[2] + 11.0 * q[3];
    f[0][1] = -q[0] + 4.0 * q[1] - 5.0 * q[2] + 2.0 * q[3];
    f[0][2] = -q[0] + 3.0 * q[1] - 3.0 * q[2] + q[3];
    f[1][0] = q[1] - 6.0 * q[2] + 3.0 * q[3] + 2.0 * q[4];
    f[1][1] = q[2] - 2.0 * q[3] + q[4];
    f[1][2] = -q[1] + 3.0 * q[2] - 3.0 * q[3] + q[4];
    f[2][0] = -2.0 * q[2] - 3.0 * q[3] + 6.0 * q[4] - q[5];
    f[2][1] = q[2] - 2.0 * q[3] + q[4];
    f[2][2] = -q[2] + 3.0 * q[3] - 3.0 * q[4] + q[5];
    f[3][0] = -11.0 * q[3] + 18.0 * q[4] - 9.0 * q[5] + 2.0 * q[6];
    f[3][1] = 2.0 * q[3] - 5.0 * q[4] + 4.0 * q[5] - q[6];
    f[3][2] = -q[3] + 3.0 * q[4] - 3.0 * q[5] + q[6];
  }
  __device__ static void deltas(const double q[7], double d[4]) {
    double f[4][3];
    forms(q, f);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      d[k] = fabs(f[k][0]) * (1.0 / 36.0) + fabs(f[k][1]) * (13.0 / 12.0) + fabs(f[k][2]) * (781.0 / 720.0);
  }
  __device__ static void js_beta(const double q[7], double b[4]) {
    double f[4][3];
    forms(q, f);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      b[k] = f[k][0] * f[k][0] * (1.0 / 36.0) + f[k][1] * f[k][1] * (13.0 / 12.0) + f[k][2] * f[k][2] * (781.0 / 720.0);
  }
  // WENO-Z factors g_k = 1 + (tau7 / (b_k + h^3))^3 with Castro-Costa-Don's tau7 (torch_weno_z.py:23-32)
  __device__ static void z_factors(const double q[7], double h, double g[4]) {
    double b[4];
    js_beta(q, b);
    const double tau = fabs(-b[0] - 3.0 * b[1] + 3.0 * b[2] + b[3]), eps = h * h * h;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double r = tau / (b[k] + eps);
      g[k] = 1.0 + r * r * r;
    }
  }
  __device__ static void lin(int lr, double d[4]) {
    if (lr == 1) {
      d[0] = 1.0 / 35.0; d[1] = 12.0 / 35.0; d[2] = 18.0 / 35.0; d[3] = 4.0 / 35.0;
    } else {
      d[0] = 4.0 / 35.0; d[1] = 18.0 / 35.0; d[2] = 12.0 / 35.0; d[3] = 1.0 / 35.0;
    }
  }
  __device__ static void cand(const double q[7], int lr, double s[4]) {
    if (lr == 1) {
      s[0] = (-1.0 / 4.0) * q[0] + (13.0 / 12.0) * q[1] + (-23.0 / 12.0) * q[2] + (25.0 / 12.0) * q[3];
      s[1] = (1.0 / 12.0) * q[1] + (-5.0 / 12.0) * q[2] + (13.0 / 12.0) * q[3] + (1.0 / 4.0) * q[4];
      s[2] = (-1.0 / 12.0) * q[2] + (7.0 / 12.0) * q[3] + (7.0 / 12.0) * q[4] + (-1.0 / 12.0) * q[5];
      s[3] = (1.0 / 4.0) * q[3] + (13.0 / 12.0) * q[4] + (-5.0 / 12.0) * q[5] + (1.0 / 12.0) * q[6];
    } else {
      s[0] = (1.0 / 12.0) * q[0] + (-5.0 / 12.0) * q[1] + (13.0 / 12.0) * q[2] + (1.0 / 4.0) * q[3];
      s[1] = (-1.0 / 12.0) * q[1] + (7.0 / 12.0) * q[2] + (7.0 / 12.0) * q[3] + (-1.0 / 12.0) * q[4];
      s[2] = (1.0 / 4.0) * q[2] + (13.0 / 12.0) * q[3] + (-5.0 / 12.0) * q[4] + (1.0 / 12.0) * q[5];
      s[3] = (25.0 / 12.0) * q[3] + (-23.0 / 12.0) * q[4] + (13.0 / 12.0) * q[5] + (-1.0 / 4.0) * q[6];
    }
  }
};

// Plateau test and MLP inputs of a stencil (weno5_core.py:158-180, weno7_core.py:182-212).
template <int SCHEME>
__device__ __forceinline__ bool adv_plateau(const double q[Weno<SCHEME>::W], double d[Weno<SCHEME>::R], double& dmax,
                                            double& qs) {
  using S = Weno<SCHEME>;
  S::deltas(q, d);
  dmax = d[0];
#pragma unroll
  for (int k = 1; k < S::R; ++k) dmax = fmax(dmax, d[k]);
  qs = fabs(q[0]);
#pragma unroll
  for (int k = 1; k < S::W; ++k) qs = fmax(qs, fabs(q[k]));
  qs = fmax(qs, 1.0);
  return dmax <= 1.0e-13 * qs;
}

// adv_plateau's decision alone: the scale max(max|q|, 1) is formed only when dmax > 1e-13 (below that, every scale
// >= 1 gives a plateau, the product 1e-13 * scale being rounded monotonically). Same decision for every input.
template <int SCHEME>
__device__ __forceinline__ bool adv_plateau_test(const double q[Weno<SCHEME>::W]) {
  using S = Weno<SCHEME>;
  double d[S::R];
  S::deltas(q, d);
  double dmax = d[0];
#pragma unroll
  for (int k = 1; k < S::R; ++k) dmax = fmax(dmax, d[k]);
  if (dmax <= 1.0e-13) return true;
  double qs = fabs(q[0]);
#pragma unroll
  for (int k = 1; k < S::W; ++k) qs = fmax(qs, fabs(q[k]));
  return dmax <= 1.0e-13 * fmax(qs, 1.0);
}

template <int SCHEME>
__device__ __forceinline__ void adv_features(const double q[Weno<SCHEME>::W], const double d[Weno<SCHEME>::R], double dmax,
                                             double qs, double f[Weno<SCHEME>::NF]) {
  using S = Weno<SCHEME>;
  const double inv = rcp64(fmax(dmax, 1.0e-15));
#pragma unroll
  for (int k = 0; k < S::R; ++k) f[k] = d[k] * inv;
  double g = 0.0;
#pragma unroll
  for (int k = 0; k + 2 < S::W; ++k) {
    const double d2 = q[k] - 2.0 * q[k + 1] + q[k + 2];
    g = fmax(g, fabs(d2) * rcp64(fabs(q[k + 1] - q[k]) + fabs(q[k + 2] - q[k + 1]) + 1.0e-15));
  }
  f[S::R] = fmin(1.0, fmax(0.0, g));
  const double rel = fmax(dmax * rcp64(qs), 1.0e-30);
  const double off = S::SCALE_OFF;
  f[S::R + 1] = fmin(1.0, fmax(0.0, (log(rel) / 2.302585092994046 + off) / off));
}

template <int SCHEME, int M>
__device__ __forceinline__ void adv_ratios(const double f[Weno<SCHEME>::NF], const typename AdvParams<SCHEME, M>::type& P,
                                           double r[Weno<SCHEME>::R]) {
  using S = Weno<SCHEME>;
  constexpr int NF = S::NF, R = S::R;
  if constexpr (M == M_SR64) {
    double xa[NF], xb[NF], ra[R], rb[R];
#pragma unroll
    for (int k = 0; k < NF; ++k) xa[k] = f[k];
#pragma unroll
    for (int k = 0; k < R; ++k) xb[k] = f[R - 1 - k];
#pragma unroll
    for (int k = R; k < NF; ++k) xb[k] = f[k];
    if constexpr (SCHEME == 5)
      mlp_pair_g<double, false, 5, 10, 6, 6, 3>(reinterpret_cast<const double*>(&P), xa, xb, ra, rb);
    else
      mlp_pair_g<double, false, 6, 24, 16, 16, 4>(reinterpret_cast<const double*>(&P), xa, xb, ra, rb);
#pragma unroll
    for (int k = 0; k < R; ++k) r[k] = 0.5 * (ra[k] + rb[R - 1 - k]);
  } else {
    constexpr bool B = M == M_SRBF16;
    float xa[NF], xb[NF], ra[R], rb[R];
#pragma unroll
    for (int k = 0; k < NF; ++k) xa[k] = B ? bf16r((float)f[k]) : (float)f[k];
#pragma unroll
    for (int k = 0; k < R; ++k) xb[k] = xa[R - 1 - k];
#pragma unroll
    for (int k = R; k < NF; ++k) xb[k] = xa[k];
    if constexpr (SCHEME == 5)
      mlp_pair_g<float, B, 5, 10, 6, 6, 3>(reinterpret_cast<const float*>(&P), xa, xb, ra, rb);
    else
      mlp_pair_g<float, B, 6, 24, 16, 16, 4>(reinterpret_cast<const float*>(&P), xa, xb, ra, rb);
#pragma unroll
    for (int k = 0; k < R; ++k) r[k] = 0.5 * ((double)ra[k] + (double)rb[R - 1 - k]);
  }
}

// Weighted value with WENO-Z weights: w = alpha / sum, alpha_k = d_k * g_k.
template <int SCHEME>
__device__ __forceinline__ double weighted_z(const double q[Weno<SCHEME>::W], int lr, const double* g) {
  using S = Weno<SCHEME>;
  double d[S::R], s[S::R], a[S::R], sum = 0.0;
  S::lin(lr, d);
  S::cand(q, lr, s);
#pragma unroll
  for (int k = 0; k < S::R; ++k) {
    a[k] = d[k] * g[k];
    sum += a[k];
  }
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < S::R; ++k) v += (a[k] / sum) * s[k];
  return v;
}

// Weighted value: w = alpha / sum, alpha_k = d_k * rk^2, with rk the reciprocal of (beta_k + eps).
template <int SCHEME>
__device__ __forceinline__ double weighted(const double q[Weno<SCHEME>::W], int lr, const double* rk, bool linear) {
  using S = Weno<SCHEME>;
  double d[S::R], s[S::R];
  S::lin(lr, d);
  S::cand(q, lr, s);
  if (linear) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < S::R; ++k) v += d[k] * s[k];
    return v;
  }
  double a[S::R], sum = 0.0;
#pragma unroll
  for (int k = 0; k < S::R; ++k) {
    a[k] = d[k] * (rk[k] * rk[k]);
    sum += a[k];
  }
  const double inv = rcp64(sum);
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < S::R; ++k) v += (a[k] * inv) * s[k];
  return v;
}

struct AdvTraj {
  int n;
  double a, dx;
};

// One right-hand-side reconstruction of the CTA's trajectory: face values fl[i] (lr=1 of cell i, the left
// state at face i+1/2) and, when BOTH, fr[i] (lr=2 of cell i, the right state at face i-1/2). With
// BOTH = false only the upwind head of the velocity sign is formed (into fl).
template <int SCHEME, int M, bool BOTH>
__device__ __forceinline__ void adv_faces(const double* __restrict__ v, const AdvTraj& T, double* fl, double* fr,
                                          unsigned short* q, int* qcount,
                                          const typename AdvParams<SCHEME, M>::type& P, int opts, Tally& tally) {
  using S = Weno<SCHEME>;
  constexpr int W = S::W, H = W / 2, R = S::R;
  constexpr bool kClosure = M != M_JS && M != M_Z;
  const int lr_up = T.a > 0.0 ? 1 : 2;
  auto stencil = [&](int i, double s[W]) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      int j = i + k - H;
      j = j < 0 ? j + T.n : (j >= T.n ? j - T.n : j);
      s[k] = v[j];
    }
  };
  if (threadIdx.x == 0) *qcount = 0;
  __syncthreads();
  // phase A
  for (int base = 0; base < T.n; base += kAdvThreads) {
    const int i = base + threadIdx.x;
    const bool active = i < T.n;
    bool need = false;
    if (active) {
      double s[W];
      stencil(i, s);
      if constexpr (M == M_JS) {
        double b[R], rk[R];
        S::js_beta(s, b);
#pragma unroll
        for (int k = 0; k < R; ++k) rk[k] = rcp64(b[k] + 1.0e-6);
        if (BOTH) {
          fl[i] = weighted<SCHEME>(s, 1, rk, false);
          fr[i] = weighted<SCHEME>(s, 2, rk, false);
        } else {
          fl[i] = weighted<SCHEME>(s, lr_up, rk, false);
        }
      } else if constexpr (M == M_Z) {
        double g[R];
        S::z_factors(s, T.dx, g);
        if (BOTH) {
          fl[i] = weighted_z<SCHEME>(s, 1, g);
          fr[i] = weighted_z<SCHEME>(s, 2, g);
        } else {
          fl[i] = weighted_z<SCHEME>(s, lr_up, g);
        }
      } else {
        need = !adv_plateau_test<SCHEME>(s);
        if (!need) {
          if (BOTH) {
            fl[i] = weighted<SCHEME>(s, 1, nullptr, true);
            fr[i] = weighted<SCHEME>(s, 2, nullptr, true);
          } else {
            fl[i] = weighted<SCHEME>(s, lr_up, nullptr, true);
          }
        }
        ++(need ? tally.mlp : tally.plateau);
      }
    }
    if constexpr (kClosure) {
      const unsigned m = __ballot_sync(0xffffffffu, need);
      if (m) {
        const int lane = threadIdx.x & 31;
        int b0 = 0;
        if (lane == __ffs(m) - 1) b0 = atomicAdd(qcount, __popc(m));
        b0 = __shfl_sync(0xffffffffu, b0, __ffs(m) - 1);
        if (need) q[b0 + __popc(m & ((1u << lane) - 1u))] = (unsigned short)i;
      }
    }
  }
  if constexpr (kClosure) {
    __syncthreads();
    const int count = *qcount;
    for (int e = threadIdx.x; e < count; e += kAdvThreads) {
      const int i = q[e];
      double s[W], d[R], dmax, qs, f[S::NF], r[R], rk[R];
      stencil(i, s);
      adv_plateau<SCHEME>(s, d, dmax, qs);
      adv_features<SCHEME>(s, d, dmax, qs, f);
      adv_ratios<SCHEME, M>(f, P, r);
      bool ok = true;
#pragma unroll
      for (int k = 0; k < R; ++k) {
        rk[k] = rcp64(S::BSCALE * r[k] + 1.0e-12);
        ok = ok && isfinite(rk[k]);
      }
      if (!ok && (opts & OPT_JS_FALLBACK)) {
        double b[R];
        S::js_beta(s, b);
#pragma unroll
        for (int k = 0; k < R; ++k) rk[k] = rcp64(b[k] + 1.0e-6);
        ++tally.fallbacks;
      }
      if (BOTH) {
        fl[i] = weighted<SCHEME>(s, 1, rk, false);
        fr[i] = weighted<SCHEME>(s, 2, rk, false);
      } else {
        fl[i] = weighted<SCHEME>(s, lr_up, rk, false);
      }
    }
  }
  __syncthreads();
}

// rhs_i = -(F_{i+1/2} - F_{i-1/2}) / dx with F = a * (upwind state, or the downwind one for L~).
// Face i+1/2: left state fl[i], right state fr[i+1]. With BOTH = false, fl holds the upwind head of
// cell i: for a > 0 it is the left state of face i+1/2, for a < 0 the right state of face i-1/2.
template <bool BOTH>
__device__ __forceinline__ double adv_rhs(const double* fl, const double* fr, const AdvTraj& T, int i, bool reverse) {
  const int ip = i + 1 == T.n ? 0 : i + 1, im = i == 0 ? T.n - 1 : i - 1;
  double face_p, face_m;
  if (BOTH) {
    const bool left = (T.a > 0.0) != reverse;
    face_p = left ? fl[i] : fr[ip];
    face_m = left ? fl[im] : fr[i];
  } else {
    face_p = T.a > 0.0 ? fl[i] : fl[ip];
    face_m = T.a > 0.0 ? fl[im] : fl[i];
  }
  const double fp = T.a * face_p, fm = T.a * face_m;
  return -(fp - fm) * (1.0 / T.dx);
}

template <int SCHEME, int M, int INTEG>
__global__ void __launch_bounds__(kAdvThreads) k_adv1d(double* __restrict__ u, const long long* __restrict__ offsets,
                                                        const int* __restrict__ order, const double* __restrict__ vel,
                                                        const double* __restrict__ dxs, const int* __restrict__ nfull,
                                                        const double* __restrict__ dtf, const double* __restrict__ dtl,
                                                        int B, int nmax, int opts, int* __restrict__ fallbacks,
                                                        int* __restrict__ errors, unsigned long long* __restrict__ counters,
                                                        const __grid_constant__ typename AdvParams<SCHEME, M>::type P) {
  extern __shared__ double smem[];
  __shared__ int qcount;
  const int b = order ? order[blockIdx.x] : (int)blockIdx.x;
  if (b < 0 || b >= B) return;
  const long long off = offsets[b];
  AdvTraj T;
  T.n = (int)(offsets[b + 1] - off);
  T.a = vel[b];
  T.dx = dxs[b];
  if (T.n < Weno<SCHEME>::W || T.n > nmax) {
    if (threadIdx.x == 0) atomicAdd(errors, 1);
    return;
  }
  constexpr int NA = INTEG == 0 ? 3 : 11;  // shared arrays of nmax doubles
  double* U = smem;                          // step start
  double* arr[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) arr[k] = smem + (size_t)k * nmax;
  unsigned short* q = reinterpret_cast<unsigned short*>(smem + (size_t)NA * nmax);
  double* g = u + off;
  for (int i = threadIdx.x; i < T.n; i += kAdvThreads) U[i] = g[i];
  __syncthreads();
  Tally tally;
  const int total = nfull[b] + (dtl[b] > 0.0 ? 1 : 0);
  for (int step = 0; step < total; ++step) {
    const double dt = step < nfull[b] ? dtf[b] : dtl[b];
    if constexpr (INTEG == 0) {
      // SSPRK3 (rk3_advection.py:118-131); S holds the stage state, F the upwind face values
      double* S = arr[1];
      double* F = arr[2];
#pragma unroll 1
      for (int stage = 0; stage < 3; ++stage) {
        const double* in = stage == 0 ? U : S;
        adv_faces<SCHEME, M, false>(in, T, F, nullptr, q, &qcount, P, opts, tally);
        for (int i = threadIdx.x; i < T.n; i += kAdvThreads) {
          const double l = adv_rhs<false>(F, nullptr, T, i, false);
          const double x = in[i] + dt * l;
          S[i] = stage == 0 ? x : (stage == 1 ? 0.75 * U[i] + 0.25 * x : U[i] / 3.0 + (2.0 / 3.0) * x);
        }
        __syncthreads();
      }
      for (int i = threadIdx.x; i < T.n; i += kAdvThreads) U[i] = S[i];
      __syncthreads();
    } else {
      // Shu RK4 with L and L~ (rk4_advection.py:137-195)
      double *u1 = arr[1], *u2 = arr[2], *u3 = arr[3], *l0 = arr[4], *lt0 = arr[5], *l1 = arr[6], *lt1 = arr[7],
             *l2 = arr[8], *FL = arr[9], *FR = arr[10];
      adv_faces<SCHEME, M, true>(U, T, FL, FR, q, &qcount, P, opts, tally);
      for (int i = threadIdx.x; i < T.n; i += kAdvThreads) {
        l0[i] = adv_rhs<true>(FL, FR, T, i, false);
        lt0[i] = adv_rhs<true>(FL, FR, T, i, true);
        u1[i] = U[i] + 0.5 * dt * l0[i];
      }
      __syncthreads();
      adv_faces<SCHEME, M, true>(u1, T, FL, FR, q, &qcount, P, opts, tally);
      for (int i = threadIdx.x; i < T.n; i += kAdvThreads) {
        l1[i] = adv_rhs<true>(FL, FR, T, i, false);
        lt1[i] = adv_rhs<true>(FL, FR, T, i, true);
        u2[i] = (649.0 / 1600.0) * U[i] - (10890423.0 / 25193600.0) * dt * lt0[i] + (951.0 / 1600.0) * u1[i] +
                (5000.0 / 7873.0) * dt * l1[i];
      }
      __syncthreads();
      adv_faces<SCHEME, M, true>(u2, T, FL, FR, q, &qcount, P, opts, tally);
      for (int i = threadIdx.x; i < T.n; i += kAdvThreads) {
        l2[i] = adv_rhs<true>(FL, FR, T, i, false);
        u3[i] = (53989.0 / 2500000.0) * U[i] - (102261.0 / 5000000.0) * dt * lt0[i] +
                (4806213.0 / 20000000.0) * u1[i] - (5121.0 / 20000.0) * dt * lt1[i] + (23619.0 / 32000.0) * u2[i] +
                (7873.0 / 10000.0) * dt * l2[i];
      }
      __syncthreads();
      adv_faces<SCHEME, M, true>(u3, T, FL, FR, q, &qcount, P, opts, tally);
      for (int i = threadIdx.x; i < T.n; i += kAdvThreads) {
        const double l3 = adv_rhs<true>(FL, FR, T, i, false);
        U[i] = (1.0 / 5.0) * U[i] + (1.0 / 10.0) * dt * l0[i] + (6127.0 / 30000.0) * u1[i] + (1.0 / 6.0) * dt * l1[i] +
               (7873.0 / 30000.0) * u2[i] + (1.0 / 3.0) * u3[i] + (1.0 / 6.0) * dt * l3;
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < T.n; i += kAdvThreads) g[i] = U[i];
  if (tally.fallbacks) atomicAdd(fallbacks, tally.fallbacks);
  if ((opts & OPT_COUNT) && counters) {
    if (tally.mlp) atomicAdd(&counters[0], (unsigned long long)tally.mlp);
    if (tally.plateau) atomicAdd(&counters[1], (unsigned long long)tally.plateau);
  }
}

template <int INTEG>
constexpr size_t adv_smem_bytes(int nmax) {
  return (size_t)(INTEG == 0 ? 3 : 11) * nmax * sizeof(double) + (size_t)nmax * sizeof(unsigned short) + 16;
}

}  // namespace wsr
