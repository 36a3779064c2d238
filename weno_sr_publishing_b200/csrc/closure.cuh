// WENO5 weights: Jiang-Shu and the reflection-averaged MLP smoothness-ratio closure (WENO5-SR).
//
// Reference (code/snapshot/):
//   warp_weno5_helpers.py (wh) 240-242 safe_rcp, 438-446 stencil_2d, 512-570 weno5_lr_value,
//       798-873 stencil_gauss / weno5_gauss_lr_value (JS, eps 1e-6, p 2);
//   teacherfree_lab_weno5_v20_distance_balanced/weno5_rk3_diff_v20_deploy.py (DEPLOY)
//       76-120 sensors and features, 123-131 plateau test, 134-151 linear weights,
//       154-205 MLP 5->10->6->6->3 with swish, 6 tanh(raw/6) and softmax, 208-279 mlp_weights;
//   teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/warp_mlp_f32/weno5_rk3_diff_mlp_f32.py
//       (F32CORE) 94-283: FP32 inputs/parameters/activations, ratios cast back to FP64.
//
// Differences in structure (not in results beyond rounding):
//   * the reflected stencil's features are formed as the permutation (d2, d1, d0, gamma, scale) of
//     the direct ones instead of being recomputed from the reversed stencil;
//   * ratios are computed once per stencil and shared by every head that uses the stencil (the two
//     Gauss points of a transverse reconstruction);
//   * the two MLP passes (direct and reflected) are evaluated together for instruction-level
//     parallelism.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "euler_math.cuh"

namespace wsr {

// M_SRBF16_TC: the BF16 closure with its MLP on the tensor cores (closure_mma.cuh; the 2D reconstruction kernels only)
enum Method { M_JS = 0, M_SR64 = 1, M_SR32 = 2, M_SRBF16 = 3, M_Z = 4, M_SRBF16_TC = 5 };

// Methods whose weights come from the MLP closure (and so run the compacted plateau/queue split).
template <int M>
__host__ __device__ constexpr bool has_mlp() { return M == M_SR64 || M == M_SR32 || M == M_SRBF16 || M == M_SRBF16_TC; }

// Packed parameters, layout w1[5][10] b1[10] w2[10][6] b2[6] w3[6][6] b3[6] w4[6][3] b4[3].
constexpr int kW1 = 0, kB1 = 50, kW2 = 60, kB2 = 120, kW3 = 126, kB3 = 162, kW4 = 168, kB4 = 186;
constexpr int kParams5 = 189;

struct Mlp5d {
  double p[kParams5];
};
struct Mlp5f {
  float p[kParams5];
  float2 d[kParams5];  // each parameter twice: the packed (direct, reflected) operand of mlp_pair_x2
  __host__ __device__ void duplicate() {
    for (int k = 0; k < kParams5; ++k) d[k] = make_float2(p[k], p[k]);
  }
};
struct NoParams {};
// WENO-Z smoothness epsilon h^2 per grid direction (x: dx^2, y: dy^2).
struct ZEps {
  double ex, ey;
};

template <int M>
struct ClosureParams {
  using type = NoParams;
};
template <>
struct ClosureParams<M_SR64> {
  using type = Mlp5d;
};
template <>
struct ClosureParams<M_SR32> {
  using type = Mlp5f;
};
template <>
struct ClosureParams<M_SRBF16> {
  using type = Mlp5f;  // pre-rounded to bfloat16 on upload
};
template <>
struct ClosureParams<M_SRBF16_TC> {
  using type = Mlp5f;  // pre-rounded to bfloat16 on upload
};
template <>
struct ClosureParams<M_Z> {
  using type = ZEps;
};

// Options bitmask. OPT_COUNT makes the reconstruction kernels count closure evaluations (SR stencils
// that ran the MLP pair, and plateau stencils that took the linear weights) for the roofline tally.
enum : int { OPT_ENO_CUTOFF = 1, OPT_JS_FALLBACK = 2, OPT_COUNT = 4 };

// Per-thread tallies, flushed with one atomic each when OPT_COUNT is set.
struct Tally {
  int fallbacks = 0;
  int mlp = 0;
  int plateau = 0;
};

__device__ __forceinline__ void flush_tally(const Tally& t, int opts, int* fallbacks,
                                            unsigned long long* counters) {
  if (t.fallbacks) atomicAdd(fallbacks, t.fallbacks);
  if ((opts & OPT_COUNT) && counters) {
    if (t.mlp) atomicAdd(&counters[0], (unsigned long long)t.mlp);
    if (t.plateau) atomicAdd(&counters[1], (unsigned long long)t.plateau);
  }
}

// Heads: 0 face lr=1 (x_{i+1/2}^-), 1 face lr=2 (x_{i-1/2}^+), 2 Gauss loca=1, 3 Gauss loca=2.
struct Lin3 {
  double d0, d1, d2;
};

__device__ __forceinline__ Lin3 linear_weights(int head) {
  // (210 +- sqrt 3)/1080 evaluated in FP64 exactly as the reference does at run time.
  const double r3 = 1.7320508075688772;  // sqrt(3.0) correctly rounded
  if (head == 0) return {0.1, 0.6, 0.3};
  if (head == 1) return {0.3, 0.6, 0.1};
  if (head == 2) return {(210.0 + r3) / 1080.0, 11.0 / 18.0, (210.0 - r3) / 1080.0};
  return {(210.0 - r3) / 1080.0, 11.0 / 18.0, (210.0 + r3) / 1080.0};
}

// Candidate values of the three sub-stencils for a head (wh stencil_2d / stencil_gauss literals).
__device__ __forceinline__ void candidates(const double q[5], int head, double s[3]) {
  if (head == 0) {
    s[0] = (1.0 / 3.0) * q[0] - (7.0 / 6.0) * q[1] + (11.0 / 6.0) * q[2];
    s[1] = (-1.0 / 6.0) * q[1] + (5.0 / 6.0) * q[2] + (1.0 / 3.0) * q[3];
    s[2] = (1.0 / 3.0) * q[2] + (5.0 / 6.0) * q[3] - (1.0 / 6.0) * q[4];
  } else if (head == 1) {
    s[0] = (-1.0 / 6.0) * q[0] + (5.0 / 6.0) * q[1] + (1.0 / 3.0) * q[2];
    s[1] = (1.0 / 3.0) * q[1] + (5.0 / 6.0) * q[2] - (1.0 / 6.0) * q[3];
    s[2] = (11.0 / 6.0) * q[2] - (7.0 / 6.0) * q[3] + (1.0 / 3.0) * q[4];
  } else if (head == 2) {
    s[0] = -0.144337567297407 * q[0] + 0.577350269189626 * q[1] + 0.566987298107780 * q[2];
    s[1] = 0.144337567297406 * q[1] + q[2] - 0.144337567297407 * q[3];
    s[2] = 1.433012701892220 * q[2] - 0.577350269189626 * q[3] + 0.144337567297406 * q[4];
  } else {
    s[0] = 0.144337567297406 * q[0] - 0.577350269189626 * q[1] + 1.433012701892220 * q[2];
    s[1] = -0.144337567297407 * q[1] + q[2] + 0.144337567297406 * q[3];
    s[2] = 0.566987298107781 * q[2] + 0.577350269189625 * q[3] - 0.144337567297406 * q[4];
  }
}

// Per-stencil state shared by all heads: JS reciprocal betas, or SR averaged ratios.
struct StencilW {
  double a0, a1, a2;  // JS: 1/(1e-6+beta_k); SR: 1/(3 r_k + 1e-12)
  bool linear;        // SR plateau: use the linear weights
};

__device__ __forceinline__ StencilW js_stencil(const double q[5]) {
  double t2 = q[2] - 2.0 * q[3] + q[4], u2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
  double t1 = q[1] - 2.0 * q[2] + q[3], u1 = q[1] - q[3];
  double t0 = q[0] - 2.0 * q[1] + q[2], u0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
  double b2 = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
  double b1 = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
  double b0 = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
  StencilW s;
  s.a0 = rcp64(1.0e-6 + b0);
  s.a1 = rcp64(1.0e-6 + b1);
  s.a2 = rcp64(1.0e-6 + b2);
  s.linear = false;
  return s;
}

// JS: w_k = d_k rcp_k^2 / sum   (wh:557-568); one reciprocal of the sum instead of three divisions.
__device__ __forceinline__ void js_head_weights(const StencilW& s, const Lin3& d, double w[3]) {
  double a0 = d.d0 * s.a0 * s.a0, a1 = d.d1 * s.a1 * s.a1, a2 = d.d2 * s.a2 * s.a2;
  double inv = rcp64(a0 + a1 + a2);
  w[0] = a0 * inv;
  w[1] = a1 * inv;
  w[2] = a2 * inv;
}

// SR: alpha_k = d_k / (3 r_k + 1e-12)^2; w = alpha / max(sum, 1e-300); optional ENO cutoff
// (DEPLOY:240-277).
__device__ __forceinline__ void sr_head_weights(const StencilW& s, const Lin3& d, bool eno_cutoff, double w[3]) {
  if (s.linear) {
    w[0] = d.d0;
    w[1] = d.d1;
    w[2] = d.d2;
    return;
  }
  double a0 = d.d0 * (s.a0 * s.a0), a1 = d.d1 * (s.a1 * s.a1), a2 = d.d2 * (s.a2 * s.a2);
  // The reference divides by max(sum, 1e-300). Here a_k = 1/(3 r_k + 1e-12) >= 1/(3 + 1e-12) for ratios in
  // [0, 1], so the sum lies in [1e-2, 1e24] and the guard never binds: one Newton-refined reciprocal.
  double inv = rcp64(a0 + a1 + a2);
  w[0] = a0 * inv;
  w[1] = a1 * inv;
  w[2] = a2 * inv;
  if (eno_cutoff) {
    const double cut = 4.0e-7;
    double p0 = w[0] <= cut ? 0.0 : 1.0, p1 = w[1] <= cut ? 0.0 : 1.0, p2 = w[2] <= cut ? 0.0 : 1.0;
    double ci = 1.0 / fmax(p0 * w[0] + p1 * w[1] + p2 * w[2], 1.0e-300);
    w[0] = p0 * w[0] * ci;
    w[1] = p1 * w[1] * ci;
    w[2] = p2 * w[2] * ci;
  }
}

// ---------------------------------------------------------------------------------------------
// MLP 5->10->6->6->3, two inputs at once (direct and reflected). Parameters are read from kernel
// parameter space (constant bank), every lane the same address, so they are broadcast operands.
// ---------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T swish(T z);
template <>
__device__ __forceinline__ double swish<double>(double z) {
  return z * rcp64(1.0 + exp(-z));
}
// FP32-closure transcendentals: 1 = hardware approximations (ex2.approx via __expf, rcp.approx via
// __fdividef), 0 = the accurate expf/tanhf and IEEE division, 2 = exp on the FMA pipe (exp_fma) with a
// Newton-refined reciprocal. Mode 1 keeps the end-of-run density L1 of the 2D quadrant problem within
// 2.2e-9 of the FP64 closure (the FP32 closure's precision bound is 1e-8), so it is the default.
#ifndef WSR_SWISH_MODE
#define WSR_SWISH_MODE 1
#endif

// e^x for |x| <= 87 on the FMA pipe: Cody-Waite reduction x = k ln2 + r (two-part ln2), e^r by its
// degree-6 Taylor polynomial (|r| <= ln2/2, truncation < 1.2e-7 relative), 2^k added to the exponent.
__device__ __forceinline__ float exp_fma(float x) {
  x = fminf(fmaxf(x, -87.0f), 88.0f);
  const float k = rintf(x * 1.44269504f);
  float r = fmaf(k, -0.693145752f, x);
  r = fmaf(k, -1.42860677e-06f, r);
  float p = 1.38888889e-3f;
  p = fmaf(p, r, 8.33333333e-3f);
  p = fmaf(p, r, 4.16666667e-2f);
  p = fmaf(p, r, 1.66666667e-1f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  return __int_as_float(__float_as_int(p) + (static_cast<int>(k) << 23));
}

// 1/d from the hardware approximation refined by one Newton step.
__device__ __forceinline__ float rcp_nr(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  const float e = fmaf(-d, r, 1.0f);
  return fmaf(r, e, r);
}

template <>
__device__ __forceinline__ float swish<float>(float z) {
#if WSR_SWISH_MODE == 1
  return __fdividef(z, 1.0f + __expf(-z));
#elif WSR_SWISH_MODE == 2
  return z * rcp_nr(1.0f + exp_fma(-z));
#else
  return z / (1.0f + expf(-z));
#endif
}

__device__ __forceinline__ double tanh_t(double x) { return tanh(x); }
__device__ __forceinline__ double exp_t(double x) { return exp(x); }
__device__ __forceinline__ double rcp_t(double x) { return rcp64(x); }
__device__ __forceinline__ double div6(double x) { return x / 6.0; }
#if WSR_SWISH_MODE == 1
__device__ __forceinline__ float tanh_t(float x) { return tanhf(x); }
__device__ __forceinline__ float exp_t(float x) { return __expf(x); }
__device__ __forceinline__ float rcp_t(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ float div6(float x) { return x * (1.0f / 6.0f); }
#else
__device__ __forceinline__ float tanh_t(float x) { return tanhf(x); }
__device__ __forceinline__ float exp_t(float x) { return expf(x); }
__device__ __forceinline__ float rcp_t(float x) { return 1.0f / x; }
__device__ __forceinline__ float div6(float x) { return x / 6.0f; }
#endif

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Multiply-add with one rounding: what the compiler's contraction gives, written out so that a
// translation unit built without contraction keeps it in the MLP.
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }

// FP64 activations in a rolled loop per layer after the layer's unrolled multiply-adds: inlined once per neuron,
// the FP64 exp/reciprocal sequences can make a closure kernel's code large enough that instruction fetch stalls
// it. Measured per kernel family: the 3D kernels run 37% faster rolled (64.5 -> 41.0 ms per shock-bubble SR-FP64
// step) and the 1D batch 10% (dense_pair, adv1d.cuh); the 2D WENO5 kernels, with their smaller MLP, 3% slower,
// so the choice is made per translation unit (WSR_ROLL_FP64_ACT, off by default). Single precision stays fully
// unrolled (its exp and reciprocal are single hardware instructions).
#ifndef WSR_ROLL_FP64_ACT
#define WSR_ROLL_FP64_ACT 0
#endif
template <typename T>
constexpr bool kRollAct = WSR_ROLL_FP64_ACT && sizeof(T) == 8;
template <typename T>
constexpr bool kRollActAlways = sizeof(T) == 8;

template <typename T, bool ROLL = kRollAct<T>>
__device__ __forceinline__ void swish_rolled(T* a, T* b, int n) {
  if constexpr (ROLL) {
#pragma unroll 1
    for (int o = 0; o < n; ++o) {
      a[o] = swish<T>(a[o]);
      b[o] = swish<T>(b[o]);
    }
  }
}

template <typename T, bool BF16, bool ROLL = kRollAct<T>>
__device__ __forceinline__ void mlp_pair(const T* __restrict__ P, const T xa[5], const T xb[5], T ra[3], T rb[3]) {
  T ha[10], hb[10];
#pragma unroll
  for (int o = 0; o < 10; ++o) {
    T za = P[kB1 + o], zb = P[kB1 + o];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      za = fma_t(xa[k], P[kW1 + k * 10 + o], za);
      zb = fma_t(xb[k], P[kW1 + k * 10 + o], zb);
    }
    ha[o] = ROLL ? za : swish<T>(za);
    hb[o] = ROLL ? zb : swish<T>(zb);
    if (BF16) {
      ha[o] = bf16r(ha[o]);
      hb[o] = bf16r(hb[o]);
    }
  }
  swish_rolled<T, ROLL>(ha, hb, 10);
  T ga[6], gb[6];
#pragma unroll
  for (int o = 0; o < 6; ++o) {
    T za = P[kB2 + o], zb = P[kB2 + o];
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      za = fma_t(ha[k], P[kW2 + k * 6 + o], za);
      zb = fma_t(hb[k], P[kW2 + k * 6 + o], zb);
    }
    ga[o] = ROLL ? za : swish<T>(za);
    gb[o] = ROLL ? zb : swish<T>(zb);
    if (BF16) {
      ga[o] = bf16r(ga[o]);
      gb[o] = bf16r(gb[o]);
    }
  }
  swish_rolled<T, ROLL>(ga, gb, 6);
  T ka[6], kb[6];
#pragma unroll
  for (int o = 0; o < 6; ++o) {
    T za = P[kB3 + o], zb = P[kB3 + o];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      za = fma_t(ga[k], P[kW3 + k * 6 + o], za);
      zb = fma_t(gb[k], P[kW3 + k * 6 + o], zb);
    }
    ka[o] = ROLL ? za : swish<T>(za);
    kb[o] = ROLL ? zb : swish<T>(zb);
    if (BF16) {
      ka[o] = bf16r(ka[o]);
      kb[o] = bf16r(kb[o]);
    }
  }
  swish_rolled<T, ROLL>(ka, kb, 6);
  T ba[3], bb[3];
#pragma unroll
  for (int o = 0; o < 3; ++o) {
    T za = P[kB4 + o], zb = P[kB4 + o];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      za = fma_t(ka[k], P[kW4 + k * 3 + o], za);
      zb = fma_t(kb[k], P[kW4 + k * 3 + o], zb);
    }
    ba[o] = T(6) * tanh_t(div6(za));
    bb[o] = T(6) * tanh_t(div6(zb));
  }
  T ma = ba[0] > ba[1] ? ba[0] : ba[1];
  ma = ma > ba[2] ? ma : ba[2];
  T mb = bb[0] > bb[1] ? bb[0] : bb[1];
  mb = mb > bb[2] ? mb : bb[2];
  T ea0 = exp_t(ba[0] - ma), ea1 = exp_t(ba[1] - ma), ea2 = exp_t(ba[2] - ma);
  T eb0 = exp_t(bb[0] - mb), eb1 = exp_t(bb[1] - mb), eb2 = exp_t(bb[2] - mb);
  T ia = rcp_t(ea0 + ea1 + ea2), ib = rcp_t(eb0 + eb1 + eb2);
  ra[0] = ea0 * ia;
  ra[1] = ea1 * ia;
  ra[2] = ea2 * ia;
  rb[0] = eb0 * ib;
  rb[1] = eb1 * ib;
  rb[2] = eb2 * ib;
}

__device__ __forceinline__ double combine(const double w[3], const double s[3]) {
  return w[0] * s[0] + w[1] * s[1] + w[2] * s[2];
}

// ---------------------------------------------------------------------------------------------
// Split closure for the compacted kernels: phase A decides plateau vs MLP from the cheap sensors,
// phase B evaluates the MLP pair of the queued stencils densely, phase C forms the weights.
// ---------------------------------------------------------------------------------------------

// delta_k, delta_max and q_scale (DEPLOY:76-93, 123-131) without the gamma ratios, which only the
// MLP needs.
struct Sens {
  double d0, d1, d2, dmax, qscale;
};

__device__ __forceinline__ Sens sensors5(const double q[5]) {
  double d20 = q[0] - 2.0 * q[1] + q[2], d21 = q[1] - 2.0 * q[2] + q[3], d22 = q[2] - 2.0 * q[3] + q[4];
  Sens s;
  s.d0 = (13.0 / 12.0) * fabs(d20) + 0.25 * fabs(q[0] - 4.0 * q[1] + 3.0 * q[2]);
  s.d1 = (13.0 / 12.0) * fabs(d21) + 0.25 * fabs(q[1] - q[3]);
  s.d2 = (13.0 / 12.0) * fabs(d22) + 0.25 * fabs(3.0 * q[2] - 4.0 * q[3] + q[4]);
  s.dmax = fmax(fmax(s.d0, s.d1), s.d2);
  double qs = fmax(fmax(fmax(fabs(q[0]), fabs(q[1])), fmax(fabs(q[2]), fabs(q[3]))), fabs(q[4]));
  s.qscale = fmax(qs, 1.0);
  return s;
}

__device__ __forceinline__ bool is_plateau(const Sens& s) { return s.dmax <= 1.0e-13 * s.qscale; }

// is_plateau(sensors5(q)) with the scale max(max|q|, 1) formed only when it can change the answer: the threshold
// 1e-13 * scale is at least 1e-13 (scale >= 1, and the product is rounded monotonically), so dmax <= 1e-13 is a
// plateau whatever q is. Same decision for every input, NaN included.
__device__ __forceinline__ bool plateau5(const double q[5]) {
  const double d20 = q[0] - 2.0 * q[1] + q[2], d21 = q[1] - 2.0 * q[2] + q[3], d22 = q[2] - 2.0 * q[3] + q[4];
  const double d0 = (13.0 / 12.0) * fabs(d20) + 0.25 * fabs(q[0] - 4.0 * q[1] + 3.0 * q[2]);
  const double d1 = (13.0 / 12.0) * fabs(d21) + 0.25 * fabs(q[1] - q[3]);
  const double d2 = (13.0 / 12.0) * fabs(d22) + 0.25 * fabs(3.0 * q[2] - 4.0 * q[3] + q[4]);
  const double dmax = fmax(fmax(d0, d1), d2);
  if (dmax <= 1.0e-13) return true;
  const double qs = fmax(fmax(fmax(fabs(q[0]), fabs(q[1])), fmax(fabs(q[2]), fabs(q[3]))), fabs(q[4]));
  return dmax <= 1.0e-13 * fmax(qs, 1.0);
}

__device__ __forceinline__ double gamma_s(const double q[5]) {
  const double eps = 1.0e-15;
  double d20 = q[0] - 2.0 * q[1] + q[2], d21 = q[1] - 2.0 * q[2] + q[3], d22 = q[2] - 2.0 * q[3] + q[4];
  double g0 = fabs(d20) * rcp64(fabs(q[1] - q[0]) + fabs(q[2] - q[1]) + eps);
  double g1 = fabs(d21) * rcp64(fabs(q[2] - q[1]) + fabs(q[3] - q[2]) + eps);
  double g2 = fabs(d22) * rcp64(fabs(q[3] - q[2]) + fabs(q[4] - q[3]) + eps);
  return fmin(1.0, fmax(fmax(g0, g1), g2));
}

#ifndef WSR_FEATURES_F32
#define WSR_FEATURES_F32 1
#endif

// FP32 MLP of the direct and reflected inputs together with Blackwell's packed FP32 arithmetic
// (fma/mul/add .f32x2: two independent single-precision operations per instruction, each rounded as its
// scalar form). The two orientations share every weight, so each weight is read once as a duplicated pair
// from the parameter block; the transcendental units stay scalar. Same values as mlp_pair<float, false>.
__device__ __forceinline__ unsigned long long pk2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(unsigned long long v, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ unsigned long long wpair(const float2& w) {
  return *reinterpret_cast<const unsigned long long*>(&w);
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// swish of two lanes: z / (1 + e^-z) with e^-z = 2^(-z log2 e) and the reciprocal from the transcendental
// unit (scalar), the scaling, the 1 + e and the final product as packed pairs.
__device__ __forceinline__ unsigned long long swish2(unsigned long long z) {
#if WSR_SWISH_MODE == 1
  const float nl2e = -1.44269502f;  // -log2(e) rounded to float
  float ta, tb;
  upk2(mul2(z, pk2(nl2e, nl2e)), ta, tb);
  float sa, sb;
  upk2(add2(pk2(ex2_approx(ta), ex2_approx(tb)), pk2(1.0f, 1.0f)), sa, sb);
  return mul2(z, pk2(rcp_approx(sa), rcp_approx(sb)));
#else
  float a, b;
  upk2(z, a, b);
  return pk2(swish<float>(a), swish<float>(b));
#endif
}

template <int NI, int NO>
__device__ __forceinline__ void dense_x2(const float2* __restrict__ D, int w, int bias, const unsigned long long* x,
                                         unsigned long long* y, bool act) {
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    unsigned long long z = wpair(D[bias + o]);
#pragma unroll
    for (int k = 0; k < NI; ++k) z = fma2(x[k], wpair(D[w + k * NO + o]), z);
    y[o] = act ? swish2(z) : z;
  }
}

__device__ __forceinline__ void mlp_pair_x2(const float2* __restrict__ D, const float xa[5], const float xb[5],
                                            float ra[3], float rb[3]) {
  unsigned long long x[5], h1[10], h2[6], h3[6], z4[3];
#pragma unroll
  for (int k = 0; k < 5; ++k) x[k] = pk2(xa[k], xb[k]);
  dense_x2<5, 10>(D, kW1, kB1, x, h1, true);
  dense_x2<10, 6>(D, kW2, kB2, h1, h2, true);
  dense_x2<6, 6>(D, kW3, kB3, h2, h3, true);
  dense_x2<6, 3>(D, kW4, kB4, h3, z4, false);
  float ba[3], bb[3];
#pragma unroll
  for (int o = 0; o < 3; ++o) {
    float za, zb;
    upk2(z4[o], za, zb);
    ba[o] = 6.0f * tanh_t(div6(za));
    bb[o] = 6.0f * tanh_t(div6(zb));
  }
  float ma = ba[0] > ba[1] ? ba[0] : ba[1];
  ma = ma > ba[2] ? ma : ba[2];
  float mb = bb[0] > bb[1] ? bb[0] : bb[1];
  mb = mb > bb[2] ? mb : bb[2];
  const float ea0 = exp_t(ba[0] - ma), ea1 = exp_t(ba[1] - ma), ea2 = exp_t(ba[2] - ma);
  const float eb0 = exp_t(bb[0] - mb), eb1 = exp_t(bb[1] - mb), eb2 = exp_t(bb[2] - mb);
  const float ia = rcp_t(ea0 + ea1 + ea2), ib = rcp_t(eb0 + eb1 + eb2);
  ra[0] = ea0 * ia;
  ra[1] = ea1 * ia;
  ra[2] = ea2 * ia;
  rb[0] = eb0 * ib;
  rb[1] = eb1 * ib;
  rb[2] = eb2 * ib;
}

// Queue element types: MLP inputs in the closure precision.
template <int M>
struct QIn {
  using T = float;
};
template <>
struct QIn<M_SR64> {
  using T = double;
};

// Phase B: reflection-averaged ratios of one queued stencil -> reciprocal scaled betas.
template <int M>
__device__ __forceinline__ void closure_from_features(const typename QIn<M>::T* x, const typename ClosureParams<M>::type& P,
                                                      double& a0, double& a1, double& a2) {
  double r0, r1, r2;
  if constexpr (M == M_SR64) {
    double xa[5] = {x[0], x[1], x[2], x[3], x[4]};
    double xb[5] = {x[2], x[1], x[0], x[3], x[4]};
    double ra[3], rb[3];
    mlp_pair<double, false>(reinterpret_cast<const double*>(&P), xa, xb, ra, rb);
    r0 = 0.5 * (ra[0] + rb[2]);
    r1 = 0.5 * (ra[1] + rb[1]);
    r2 = 0.5 * (ra[2] + rb[0]);
  } else {
    constexpr bool B = M == M_SRBF16 || M == M_SRBF16_TC;
    float xa[5] = {x[0], x[1], x[2], x[3], x[4]};
    float xb[5] = {x[2], x[1], x[0], x[3], x[4]};
    float ra[3], rb[3];
    if constexpr (B)
      mlp_pair<float, true>(reinterpret_cast<const float*>(&P), xa, xb, ra, rb);
    else
      mlp_pair_x2(P.d, xa, xb, ra, rb);
    r0 = 0.5 * ((double)ra[0] + (double)rb[2]);
    r1 = 0.5 * ((double)ra[1] + (double)rb[1]);
    r2 = 0.5 * ((double)ra[2] + (double)rb[0]);
  }
  a0 = rcp64(3.0 * r0 + 1.0e-12);
  a1 = rcp64(3.0 * r1 + 1.0e-12);
  a2 = rcp64(3.0 * r2 + 1.0e-12);
}

// Cast FP64 features to the queue type (BF16 inputs are rounded to bfloat16, as the oracle does).
template <int M>
__device__ __forceinline__ typename QIn<M>::T to_queue(double f) {
  if constexpr (M == M_SR64)
    return f;
  else if constexpr (M == M_SRBF16 || M == M_SRBF16_TC)
    return bf16r((float)f);
  else
    return (float)f;
}


// MLP inputs of the reduced-precision closures (FP32; BF16 rounds them to bfloat16): the differences are FP64
// (they cancel), the normalisation, gamma and the scale feature are formed in FP32 (the MLP consumes FP32 inputs;
// dmax >= 1e-13 here, so every value is a normal float).
template <int M>
__device__ __forceinline__ void sr_features32(const double s[5], const Sens& se, float x[5]) {
  const double d20 = s[0] - 2.0 * s[1] + s[2], d21 = s[1] - 2.0 * s[2] + s[3], d22 = s[2] - 2.0 * s[3] + s[4];
  const float inv = rcp_nr((float)se.dmax);
  const float e = 1.0e-15f;
  x[0] = (float)se.d0 * inv;
  x[1] = (float)se.d1 * inv;
  x[2] = (float)se.d2 * inv;
  const float g0 = __fdividef(fabsf((float)d20), (float)(fabs(s[1] - s[0]) + fabs(s[2] - s[1])) + e);
  const float g1 = __fdividef(fabsf((float)d21), (float)(fabs(s[2] - s[1]) + fabs(s[3] - s[2])) + e);
  const float g2 = __fdividef(fabsf((float)d22), (float)(fabs(s[3] - s[2]) + fabs(s[4] - s[3])) + e);
  x[3] = fminf(1.0f, fmaxf(fmaxf(g0, g1), g2));
  const float rel = (float)se.dmax * rcp_nr((float)se.qscale);
  x[4] = rel >= 1.0f ? 1.0f : (rel <= 1.0e-4f ? 0.0f : fminf(1.0f, fmaxf(0.0f, (__log10f(rel) + 4.0f) * 0.25f)));
  if constexpr (M == M_SRBF16 || M == M_SRBF16_TC) {
#pragma unroll
    for (int k = 0; k < 5; ++k) x[k] = bf16r(x[k]);
  }
}

// SR closure of one non-plateau stencil -> reciprocal scaled betas (features FP64 as in DEPLOY:96-120,
// the MLP in the closure precision, ratios averaged and inverted in FP64 as in DEPLOY:234-247).
template <int M>
__device__ __forceinline__ void sr_betas(const double s[5], const typename ClosureParams<M>::type& P,
                                         double& a0, double& a1, double& a2) {
  const Sens se = sensors5(s);
#if WSR_FEATURES_F32
  if constexpr (M != M_SR64) {
    float x[5];
    sr_features32<M>(s, se, x);
    closure_from_features<M>(x, P, a0, a1, a2);
    return;
  }
#endif
  double f[5];
  const double inv = rcp64(fmax(se.dmax, 1.0e-15));
  f[0] = se.d0 * inv;
  f[1] = se.d1 * inv;
  f[2] = se.d2 * inv;
  f[3] = gamma_s(s);
  // clip((log10(rel) + 4)/4, 0, 1): the logarithm is needed only when rel is strictly inside (1e-4, 1)
  const double rel = fmax(se.dmax * rcp64(se.qscale), 1.0e-30);
  f[4] = rel >= 1.0 ? 1.0 : (rel <= 1.0e-4 ? 0.0 : fmin(1.0, fmax(0.0, (log(rel) / 2.302585092994046 + 4.0) / 4.0)));
  typename QIn<M>::T x[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) x[k] = to_queue<M>(f[k]);
  closure_from_features<M>(x, P, a0, a1, a2);
}

template <int M>
__device__ __forceinline__ double sr_value(const double s[5], int head, double a0, double a1, double a2, int opts,
                                           Tally& tally) {
  double w[3], c[3];
  const Lin3 d = linear_weights(head);
  if ((opts & OPT_JS_FALLBACK) && !(isfinite(a0) && isfinite(a1) && isfinite(a2))) {
    js_head_weights(js_stencil(s), d, w);
    ++tally.fallbacks;
  } else {
    StencilW sw;
    sw.a0 = a0;
    sw.a1 = a1;
    sw.a2 = a2;
    sw.linear = false;
    sr_head_weights(sw, d, (opts & OPT_ENO_CUTOFF) != 0, w);
  }
  candidates(s, head, c);
  return combine(w, c);
}

// The linear-weight value of a head as one five-term combination of the stencil, its coefficients
// sum_k d_k C_k,i formed at compile time from the same candidate literals and linear weights (a plateau
// stencil's value then costs five multiply-adds; it differs from the candidate-by-candidate evaluation
// by rounding only).
struct Lin5 {
  double c[5];
};
__host__ __device__ constexpr Lin5 lin5(int head) {
  constexpr double r3 = 1.7320508075688772;
  if (head == 0) return {{0.1 * (1.0 / 3.0), 0.1 * (-7.0 / 6.0) + 0.6 * (-1.0 / 6.0),
                          0.1 * (11.0 / 6.0) + 0.6 * (5.0 / 6.0) + 0.3 * (1.0 / 3.0),
                          0.6 * (1.0 / 3.0) + 0.3 * (5.0 / 6.0), 0.3 * (-1.0 / 6.0)}};
  if (head == 1) return {{0.3 * (-1.0 / 6.0), 0.3 * (5.0 / 6.0) + 0.6 * (1.0 / 3.0),
                          0.3 * (1.0 / 3.0) + 0.6 * (5.0 / 6.0) + 0.1 * (11.0 / 6.0),
                          0.6 * (-1.0 / 6.0) + 0.1 * (-7.0 / 6.0), 0.1 * (1.0 / 3.0)}};
  const double da = (210.0 + r3) / 1080.0, db = 11.0 / 18.0, dc = (210.0 - r3) / 1080.0;
  if (head == 2) return {{da * -0.144337567297407, da * 0.577350269189626 + db * 0.144337567297406,
                          da * 0.566987298107780 + db + dc * 1.433012701892220,
                          db * -0.144337567297407 + dc * -0.577350269189626, dc * 0.144337567297406}};
  return {{dc * 0.144337567297406, dc * -0.577350269189626 + db * -0.144337567297407,
           dc * 1.433012701892220 + db + da * 0.566987298107781,
           db * 0.144337567297406 + da * 0.577350269189625, da * -0.144337567297406}};
}

__device__ __forceinline__ double linear_value(const double s[5], int head) {
  constexpr Lin5 k0 = lin5(0), k1 = lin5(1), k2 = lin5(2), k3 = lin5(3);
  const Lin5& k = head == 0 ? k0 : (head == 1 ? k1 : (head == 2 ? k2 : k3));
  return fma(k.c[4], s[4], fma(k.c[3], s[3], fma(k.c[2], s[2], fma(k.c[1], s[1], k.c[0] * s[0]))));
}

__device__ __forceinline__ double js_value(const double s[5], int head) {
  double w[3], c[3];
  js_head_weights(js_stencil(s), linear_weights(head), w);
  candidates(s, head, c);
  return combine(w, c);
}

// WENO-Z (Borges, Carmona, Costa & Don 2008, p = 2) with eps = h^2 along the reconstruction direction
// (weno_z_borges_p2_results/weno5_helpers_z.py:545-574, 853-879): tau5 = |beta0 - beta2|,
// alpha_k = d_k (1 + (tau5 / (beta_k + eps))^2), w = alpha / sum. The head-independent factors
// g_k = 1 + ratio_k^2 are formed once per stencil and serve both Gauss heads.
__device__ __forceinline__ StencilW z_stencil(const double q[5], double eps) {
  double t2 = q[2] - 2.0 * q[3] + q[4], u2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
  double t1 = q[1] - 2.0 * q[2] + q[3], u1 = q[1] - q[3];
  double t0 = q[0] - 2.0 * q[1] + q[2], u0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
  double b2 = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
  double b1 = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
  double b0 = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
  const double tau = fabs(b0 - b2);
  const double r0 = tau * rcp64(b0 + eps), r1 = tau * rcp64(b1 + eps), r2 = tau * rcp64(b2 + eps);
  StencilW s;
  s.a0 = 1.0 + r0 * r0;
  s.a1 = 1.0 + r1 * r1;
  s.a2 = 1.0 + r2 * r2;
  s.linear = false;
  return s;
}

__device__ __forceinline__ void z_head_weights(const StencilW& s, const Lin3& d, double w[3]) {
  double a0 = d.d0 * s.a0, a1 = d.d1 * s.a1, a2 = d.d2 * s.a2;
  double inv = rcp64(a0 + a1 + a2);
  w[0] = a0 * inv;
  w[1] = a1 * inv;
  w[2] = a2 * inv;
}

__device__ __forceinline__ double z_value_w(const StencilW& z, const double s[5], int head) {
  double w[3], c[3];
  z_head_weights(z, linear_weights(head), w);
  candidates(s, head, c);
  return combine(w, c);
}

__device__ __forceinline__ double z_value(const double s[5], int head, double eps) {
  return z_value_w(z_stencil(s, eps), s, head);
}

}  // namespace wsr
