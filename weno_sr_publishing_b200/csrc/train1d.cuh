// Closure training through 1D periodic advection trajectories on sm_100a: WENO5-SR + SSPRK3 rollouts
// with checkpoints, and a hand-written adjoint (reverse mode) of the whole rollout with respect to the
// 189 MLP parameters (and the initial state).
//
// Reference (code/snapshot/teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/): the objective
// follows fast_losses.py:412-648 (autoregressive rollout whose state stays in the graph, exact cell-average
// targets at every completed SSPRK3 step, autograd through activation checkpoints) with the plain L1
// state loss; the differentiated operator is rk3_advection.py:71-131 (signed upwind face state, plateau
// mask, omega_from_ratio) over weno5_core.py:135-239 (deltas, gamma, scale feature, candidates) and
// model.py:16-80 (scale remap, MLP 5->10->6->6->3, reflection average 0.5 [M(x) + P M(Px)]).
//
// Loss: L = sum over trajectories b, completed steps k = 1..S and cells i of |u_bki - e_bki| / (B S n),
// e the exact cell averages of the advected profile.
//
// k_train_fwd: one CTA per trajectory runs the SSPRK3 steps of the 1D path (adv_faces), stores the state
// every C steps (checkpoints), evaluates the exact averages of every completed step on the fly, sums
// |u - e| and keeps sign(u - e) as two ballot words (positive, negative) per 32 cells and step.
//
// k_train_bwd: one CTA per trajectory walks the checkpoint segments from the last to the first. A segment
// is recomputed from its checkpoint, the three stage states of each of its steps going to a global scratch
// area; then its steps are reversed: the loss sign of the step's result adds to the adjoint, which goes
// back through the three SSPRK3 stages with one vector-Jacobian product (VJP) of the right-hand side each.
//
// VJP of a right-hand side: mu_c, the adjoint of the upwind face value g_c of cell c, comes from the flux
// difference. A plateau stencil contributes mu_c times the linear weights' candidate coefficients. The
// other stencils are queued and taken by thread pairs, one thread per MLP orientation: each recomputes its
// MLP evaluation with the activations, the pair exchanges outputs and input adjoints with one shuffle each,
// and the adjoint runs back through the weights, the reflection average, the MLP and the features to the
// five stencil values. Each thread writes its activations and pre-activation adjoints as one row in shared
// memory; after each chunk, the threads add the outer-product terms of the rows into registers that live
// for the whole trajectory (accumulate_rows). k_train_reduce sums the per-trajectory partial losses and
// gradients in a fixed order, so the result is deterministic.
//
// Non-smooth points follow torch autograd's conventions, so that the gradient is the one autograd gives
// for the same loss: |x|' = sign(x) with sign(0) = 0; a tie in torch.maximum splits the gradient evenly;
// a max over a dimension sends it to the first maximal element; clamp passes it when min <= x <= max.
#pragma once
#include <cuda_runtime.h>

#include "adv1d.cuh"

namespace wsr {

constexpr int kTrainThreads = 256;
constexpr int kTrainNmax = 1024;
constexpr int kDescLen = 34;
constexpr int kP5 = MlpDims<5, 10, 6, 6, 3>::N;  // 189
constexpr int kRowA = 27;                          // x(5) h1(10) h2(6) h3(6)
constexpr int kRowD = 25;                          // z1bar(10) z2bar(6) z3bar(6) z4bar(3)
constexpr int kRow = kRowA + kRowD;

template <int M>
struct TrainReal {
  using T = double;
};
template <>
struct TrainReal<M_SR32> {
  using T = float;
};

// ---------------------------------------------------------------------------------------------
// Exact cell averages of the profile descriptor (weno_sr_publishing_b200/profiles.py layout):
// [base, 3 x (amp, k, phase), 2 x (amp, centre, sigma), 2 x (amp, centre, half-width),
//  (amp, centre, half-width), 3 x (amp, left, width)].
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double near_image(double y, double c) {
  const double z = y - c + 0.5;
  return (z - floor(z)) - 0.5;
}

__device__ __forceinline__ double tri_H(double z) {
  const double s = fmin(fmax(z, -1.0), 1.0);
  return s < 0.0 ? 0.5 * ((1.0 + s) * (1.0 + s)) : 1.0 - 0.5 * ((1.0 - s) * (1.0 - s));
}

__device__ __forceinline__ double ell_H(double z) {
  const double s = fmin(fmax(z, -1.0), 1.0);
  return 0.5 * (s * sqrt(1.0 - s * s) + asin(s)) + 0.7853981633974483;
}

// d: descriptor in shared memory followed by the three sine cell-average factors sinc(pi k dx).
__device__ __forceinline__ double exact_average(const double* d, int n, int i, double shift, double dx) {
  const double nn = (double)n;
  const double xl = (double)i * dx - shift;
  const double xc = xl + 0.5 * dx;
  double out = d[0];
#pragma unroll 1
  for (int j = 0; j < 3; ++j) {
    const double amp = d[1 + 3 * j];
    if (amp != 0.0) out += amp * d[kDescLen + j] * sin(6.283185307179586 * d[2 + 3 * j] * xc + d[3 + 3 * j]);
  }
#pragma unroll 1
  for (int j = 0; j < 2; ++j) {
    const double amp = d[10 + 3 * j];
    if (amp != 0.0) {
      const double c = d[11 + 3 * j], sg = d[12 + 3 * j];
      const double dl = near_image(xl, c);
      const double r = 1.0 / (sg * 1.4142135623730951);
      const double hi = fmin(dl + dx, 0.5);  // the nearest-image form jumps at distance 1/2
      const double wrap = dl + dx > 0.5 ? erf((dl + dx - 1.0) * r) - erf(-0.5 * r) : 0.0;
      out += amp * sg * 1.2533141373155003 * nn * ((erf(hi * r) - erf(dl * r)) + wrap);
    }
  }
#pragma unroll 1
  for (int j = 0; j < 2; ++j) {
    const double amp = d[16 + 3 * j];
    if (amp != 0.0) {
      const double h = d[18 + 3 * j];
      const double dl = near_image(xl, d[17 + 3 * j]);
      out += amp * h * nn * (tri_H((dl + dx) / h) - tri_H(dl / h));
    }
  }
  if (d[22] != 0.0) {
    const double h = d[24];
    const double dl = near_image(xl, d[23]);
    out += d[22] * h * nn * (ell_H((dl + dx) / h) - ell_H(dl / h));
  }
#pragma unroll 1
  for (int j = 0; j < 3; ++j) {
    const double amp = d[25 + 3 * j];
    if (amp != 0.0) {
      const double w = d[27 + 3 * j];
      const double dl = near_image(xl, d[26 + 3 * j] + 0.5 * w);
      const double lo = fmax(dl, -0.5 * w), hi = fmin(dl + dx, 0.5 * w);
      out += amp * nn * fmax(hi - lo, 0.0);
    }
  }
  return out;
}

// ---------------------------------------------------------------------------------------------
// One SSPRK3 step of the CTA's trajectory (rk3_advection.py:118-131), the arithmetic of k_adv1d. When
// st is given, the three stage states (u^n, u^(1), u^(2)) go to st[0..n), st[n..2n), st[2n..3n).
// Ends with the new state in U and a barrier.
// ---------------------------------------------------------------------------------------------
template <int M>
__device__ __forceinline__ void ssprk3_step_cta(double* U, double* S, double* F, const AdvTraj& T, double dt,
                                                unsigned short* q, int* qcount,
                                                const typename ClosureParams<M>::type& P, Tally& tally,
                                                double* __restrict__ st) {
#pragma unroll 1
  for (int stage = 0; stage < 3; ++stage) {
    const double* in = stage == 0 ? U : S;
    if (st && stage == 0)
      for (int i = threadIdx.x; i < T.n; i += kTrainThreads) st[i] = U[i];
    adv_faces<5, M, false>(in, T, F, nullptr, q, qcount, P, 0, tally);
    for (int i = threadIdx.x; i < T.n; i += kTrainThreads) {
      const double l = adv_rhs<false>(F, nullptr, T, i, false);
      const double x = in[i] + dt * l;
      const double v = stage == 0 ? x : (stage == 1 ? 0.75 * U[i] + 0.25 * x : U[i] / 3.0 + (2.0 / 3.0) * x);
      S[i] = v;
      if (st && stage < 2) st[(stage + 1) * T.n + i] = v;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < T.n; i += kTrainThreads) U[i] = S[i];
  __syncthreads();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int M>
__global__ void __launch_bounds__(kTrainThreads) k_train_fwd(const double* __restrict__ u0, const double* __restrict__ desc,
                                                             const double* __restrict__ vel, int n, double dx, double dt,
                                                             int steps, int every, double* __restrict__ ck,
                                                             unsigned* __restrict__ signs, double* __restrict__ loss_part,
                                                             double* __restrict__ u_final,
                                                             const __grid_constant__ typename ClosureParams<M>::type P) {
  extern __shared__ double smem[];
  __shared__ int qcount;
  __shared__ double sd[kDescLen + 3];
  __shared__ double red[kTrainThreads / 32];
  const int b = blockIdx.x;
  double* U = smem;
  double* S = smem + n;
  double* F = smem + 2 * n;
  unsigned short* q = reinterpret_cast<unsigned short*>(smem + 3 * n);
  AdvTraj T;
  T.n = n;
  T.a = vel[b];
  T.dx = dx;
  if (threadIdx.x < kDescLen) sd[threadIdx.x] = desc[(size_t)b * kDescLen + threadIdx.x];
  __syncthreads();
  if (threadIdx.x < 3) {
    const double arg = 3.141592653589793 * sd[2 + 3 * threadIdx.x] * dx;
    sd[kDescLen + threadIdx.x] = arg != 0.0 ? sin(arg) / arg : 1.0;
  }
  __syncthreads();
  // the initial state: given, or the exact cell averages of the profile at t = 0
  for (int i = threadIdx.x; i < n; i += kTrainThreads) U[i] = u0 ? u0[(size_t)b * n + i] : exact_average(sd, n, i, 0.0, dx);
  __syncthreads();
  const int words = (n + 31) >> 5;
  const int K = (steps + every - 1) / every;
  double lsum = 0.0;
  Tally tally;
#pragma unroll 1
  for (int step = 0; step < steps; ++step) {
    if (step % every == 0) {
      double* c = ck + ((size_t)b * K + step / every) * n;
      for (int i = threadIdx.x; i < n; i += kTrainThreads) c[i] = U[i];
    }
    ssprk3_step_cta<M>(U, S, F, T, dt, q, &qcount, P, tally, nullptr);
    double shift = T.a * ((double)(step + 1) * dt);
    shift -= floor(shift);
    for (int base = 0; base < n; base += kTrainThreads) {
      const int i = base + threadIdx.x;
      double diff = 0.0;
      if (i < n) {
        diff = U[i] - exact_average(sd, n, i, shift, dx);
        lsum += fabs(diff);
      }
      const unsigned pos = __ballot_sync(0xffffffffu, diff > 0.0), neg = __ballot_sync(0xffffffffu, diff < 0.0);
      if ((threadIdx.x & 31) == 0 && i < n) {
        unsigned* w = signs + (((size_t)b * steps + step) * words + (i >> 5)) * 2;
        w[0] = pos;
        w[1] = neg;
      }
    }
  }
  lsum = warp_sum(lsum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTrainThreads / 32; ++w) t += red[w];
    loss_part[b] = t;
  }
  if (u_final)
    for (int i = threadIdx.x; i < n; i += kTrainThreads) u_final[(size_t)b * n + i] = U[i];
}

// ---------------------------------------------------------------------------------------------
// Adjoint pieces
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

// q_bar += d(sum_k s_bar_k cand_k(q))/dq for head lr (1: left state of face i+1/2, 2: right state of i-1/2).
__device__ __forceinline__ void cand_grad(int lr, const double sb[3], double qb[5]) {
  if (lr == 1) {
    qb[0] += (1.0 / 3.0) * sb[0];
    qb[1] += -(7.0 / 6.0) * sb[0] - (1.0 / 6.0) * sb[1];
    qb[2] += (11.0 / 6.0) * sb[0] + (5.0 / 6.0) * sb[1] + (1.0 / 3.0) * sb[2];
    qb[3] += (1.0 / 3.0) * sb[1] + (5.0 / 6.0) * sb[2];
    qb[4] += -(1.0 / 6.0) * sb[2];
  } else {
    qb[0] += -(1.0 / 6.0) * sb[0];
    qb[1] += (5.0 / 6.0) * sb[0] + (1.0 / 3.0) * sb[1];
    qb[2] += (1.0 / 3.0) * sb[0] + (5.0 / 6.0) * sb[1] + (11.0 / 6.0) * sb[2];
    qb[3] += -(1.0 / 6.0) * sb[1] - (7.0 / 6.0) * sb[2];
    qb[4] += (1.0 / 3.0) * sb[2];
  }
}

// Gradient of torch.maximum(torch.maximum(a0, a1), a2) = m, given m_bar: ties split evenly.
__device__ __forceinline__ void max3_grad(double a0, double a1, double a2, double mb, double out[3]) {
  const double m01 = fmax(a0, a1);
  const double b01 = m01 > a2 ? mb : (m01 < a2 ? 0.0 : 0.5 * mb);
  out[2] = m01 > a2 ? 0.0 : (m01 < a2 ? mb : 0.5 * mb);
  out[0] = a0 > a1 ? b01 : (a0 < a1 ? 0.0 : 0.5 * b01);
  out[1] = a0 > a1 ? 0.0 : (a0 < a1 ? b01 : 0.5 * b01);
}

// Back-propagates the feature adjoint fb (the sum over both MLP orientations) to the stencil values
// (weno5_core.py:135-180 with model.py:16-26): normalised deltas, gamma, scale feature.
__device__ __forceinline__ void feature_grad(const double q[5], const double d[3], double dmax, double qs,
                                             const double fb[5], double qb[5]) {
  double db[3] = {0.0, 0.0, 0.0};
  double dmaxb = 0.0, qsb = 0.0;
  // scale feature: clamp((16 clamp((log10 rel + 16)/16, 0, 1) - 16 + 4) / 4, 0, 1), rel = clamp(dmax/qs, 1e-30)
  const double iqs = rcp64(qs);
  const double relr = dmax * iqs;
  if (relr >= 1.0e-30) {
    const double L = log(relr) / 2.302585092994046;
    if (L >= -4.0 && L <= 0.0) {
      const double relb = 0.25 * fb[4] * rcp64(relr * 2.302585092994046);
      dmaxb += relb * iqs;
      qsb -= relb * relr * iqs;
    }
  }
  // normalised deltas d_k / max(dmax, 1e-15)
  const double inv = rcp64(fmax(dmax, 1.0e-15));
  double invb = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    db[k] += fb[k] * inv;
    invb += fb[k] * d[k];
  }
  if (dmax >= 1.0e-15) dmaxb -= invb * inv * inv;
  double mg[3];
  max3_grad(d[0], d[1], d[2], dmaxb, mg);
#pragma unroll
  for (int k = 0; k < 3; ++k) db[k] += mg[k];
  // gamma = clamp(max_j |d2_j| / (|q_{j+1}-q_j| + |q_{j+2}-q_{j+1}| + 1e-15), 0, 1)
  {
    double d2[3], den[3], g[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      d2[j] = q[j] - 2.0 * q[j + 1] + q[j + 2];
      den[j] = fabs(q[j + 1] - q[j]) + fabs(q[j + 2] - q[j + 1]) + 1.0e-15;
      g[j] = fabs(d2[j]) * rcp64(den[j]);
    }
    const double m = fmax(fmax(g[0], g[1]), g[2]);
    if (m <= 1.0 && fb[3] != 0.0) {
      double gb[3];
      max3_grad(g[0], g[1], g[2], fb[3], gb);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (gb[j] == 0.0) continue;
        const double iden = rcp64(den[j]);
        const double t = gb[j] * iden * sgn(d2[j]);
        qb[j] += t;
        qb[j + 1] -= 2.0 * t;
        qb[j + 2] += t;
        const double denb = -gb[j] * g[j] * iden;
        const double u1 = denb * sgn(q[j + 1] - q[j]), u2 = denb * sgn(q[j + 2] - q[j + 1]);
        qb[j + 1] += u1 - u2;
        qb[j] -= u1;
        qb[j + 2] += u2;
      }
    }
  }
  // q scale = clamp(max_k |q_k|, min = 1): the first maximal element
  if (qsb != 0.0) {
    int km = 0;
    double am = fabs(q[0]);
#pragma unroll
    for (int k = 1; k < 5; ++k)
      if (fabs(q[k]) > am) {
        am = fabs(q[k]);
        km = k;
      }
    if (am >= 1.0) qb[km] += qsb * sgn(q[km]);
  }
  // deltas: 13/12 |A_k| + 1/4 |B_k|
  {
    const double A0 = q[0] - 2.0 * q[1] + q[2], B0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
    const double A1 = q[1] - 2.0 * q[2] + q[3], B1 = q[1] - q[3];
    const double A2 = q[2] - 2.0 * q[3] + q[4], B2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
    const double a0 = db[0] * (13.0 / 12.0) * sgn(A0), b0 = db[0] * 0.25 * sgn(B0);
    const double a1 = db[1] * (13.0 / 12.0) * sgn(A1), b1 = db[1] * 0.25 * sgn(B1);
    const double a2 = db[2] * (13.0 / 12.0) * sgn(A2), b2 = db[2] * 0.25 * sgn(B2);
    qb[0] += a0 + b0;
    qb[1] += -2.0 * a0 - 4.0 * b0 + a1 + b1;
    qb[2] += a0 + 3.0 * b0 - 2.0 * a1 + a2 + 3.0 * b2;
    qb[3] += a1 - b1 - 2.0 * a2 - 4.0 * b2;
    qb[4] += a2 + b2;
  }
}

template <typename T>
__device__ __forceinline__ T sigmoid_t(T z);
template <>
__device__ __forceinline__ double sigmoid_t<double>(double z) {
  const double e = exp(-z);
  return e > 1.0e300 ? 0.0 : rcp64(1.0 + e);
}
template <>
__device__ __forceinline__ float sigmoid_t<float>(float z) {
  return __frcp_rn(1.0f + __expf(-z));
}

// One thread of a pair: MLP evaluation of one orientation with its activations (row[0..27)), the
// reflection average and weights (shared with the partner through shuffles), and the adjoint back to the
// stencil values (qb, complete on the p == 0 thread) and to the pre-activations (row[27..52)).
template <int M>
__device__ __forceinline__ void pair_vjp(const double q[5], const double d[3], double dmax, double qs, double mu,
                                         int lr, int p, typename TrainReal<M>::T* __restrict__ row,
                                         const typename ClosureParams<M>::type& P, double qb[5]) {
  using T = typename TrainReal<M>::T;
  using D = MlpDims<5, 10, 6, 6, 3>;
  const T* W = reinterpret_cast<const T*>(&P);
  double f[5];
  adv_features<5>(q, d, dmax, qs, f);
  T x[5];
  if (p == 0) {
#pragma unroll
    for (int k = 0; k < 5; ++k) x[k] = (T)f[k];
  } else {
    x[0] = (T)f[2];
    x[1] = (T)f[1];
    x[2] = (T)f[0];
    x[3] = (T)f[3];
    x[4] = (T)f[4];
  }
  T* A = row;
  T* Db = row + kRowA;
#pragma unroll
  for (int k = 0; k < 5; ++k) A[k] = x[k];
  T s1[10], s2[6], s3[6];
  {
    T h[10];
#pragma unroll
    for (int o = 0; o < 10; ++o) {
      T z = W[D::B1 + o];
#pragma unroll
      for (int k = 0; k < 5; ++k) z = z + x[k] * W[D::W1 + k * 10 + o];
      s1[o] = sigmoid_t<T>(z);
      h[o] = z * s1[o];
      A[5 + o] = h[o];
    }
    T h2[6];
#pragma unroll
    for (int o = 0; o < 6; ++o) {
      T z = W[D::B2 + o];
#pragma unroll
      for (int k = 0; k < 10; ++k) z = z + h[k] * W[D::W2 + k * 6 + o];
      s2[o] = sigmoid_t<T>(z);
      h2[o] = z * s2[o];
      A[15 + o] = h2[o];
    }
#pragma unroll
    for (int o = 0; o < 6; ++o) {
      T z = W[D::B3 + o];
#pragma unroll
      for (int k = 0; k < 6; ++k) z = z + h2[k] * W[D::W3 + k * 6 + o];
      s3[o] = sigmoid_t<T>(z);
      A[21 + o] = z * s3[o];
    }
  }
  T th[3], o3[3];
  {
    T bad[3];
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      T z = W[D::B4 + o];
#pragma unroll
      for (int k = 0; k < 6; ++k) z = z + A[21 + k] * W[D::W4 + k * 3 + o];
      th[o] = tanh_t(div6(z));
      bad[o] = T(6) * th[o];
    }
    T m = bad[0] > bad[1] ? bad[0] : bad[1];
    m = m > bad[2] ? m : bad[2];
    T e[3], s = T(0);
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      e[o] = exp_t(bad[o] - m);
      s = s + e[o];
    }
    const T is = rcp_t(s);
#pragma unroll
    for (int o = 0; o < 3; ++o) o3[o] = e[o] * is;
  }
  // reflection average and weights (identical on both threads of the pair)
  double oa[3], ob[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double mine = (double)o3[k];
    const double other = (double)__shfl_xor_sync(0xffffffffu, o3[k], 1);
    oa[k] = p == 0 ? mine : other;
    ob[k] = p == 0 ? other : mine;
  }
  double dl[3], c[3];
  Weno<5>::lin(lr, dl);
  Weno<5>::cand(q, lr, c);
  double r[3], rk[3], al[3], sum = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r[k] = 0.5 * (oa[k] + ob[2 - k]);
    rk[k] = rcp64(3.0 * r[k] + 1.0e-12);
    al[k] = dl[k] * (rk[k] * rk[k]);
    sum += al[k];
  }
  const double inv = rcp64(sum);
  double om[3], omb[3], dot = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    om[k] = al[k] * inv;
    omb[k] = mu * c[k];
    dot += omb[k] * om[k];
  }
  double rb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) rb[k] = -6.0 * ((omb[k] - dot) * inv) * al[k] * rk[k];
  // MLP backward of this orientation
  T obar[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) obar[k] = (T)(0.5 * (p == 0 ? rb[k] : rb[2 - k]));
  T z4b[3];
  {
    T dp = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) dp = dp + obar[k] * o3[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      z4b[k] = o3[k] * (obar[k] - dp) * (T(1) - th[k] * th[k]);
      Db[22 + k] = z4b[k];
    }
  }
  T z3b[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    T hb = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) hb = hb + W[D::W4 + i * 3 + k] * z4b[k];
    const T h = A[21 + i], s = s3[i];
    z3b[i] = hb * (s + h * (T(1) - s));
    Db[16 + i] = z3b[i];
  }
  T z2b[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    T hb = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) hb = hb + W[D::W3 + i * 6 + k] * z3b[k];
    const T h = A[15 + i], s = s2[i];
    z2b[i] = hb * (s + h * (T(1) - s));
    Db[10 + i] = z2b[i];
  }
  T z1b[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    T hb = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) hb = hb + W[D::W2 + i * 6 + k] * z2b[k];
    const T h = A[5 + i], s = s1[i];
    z1b[i] = hb * (s + h * (T(1) - s));
    Db[i] = z1b[i];
  }
  double xa[5], xr[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    T xb = T(0);
#pragma unroll
    for (int k = 0; k < 10; ++k) xb = xb + W[D::W1 + i * 10 + k] * z1b[k];
    const double mine = (double)xb, other = (double)__shfl_xor_sync(0xffffffffu, xb, 1);
    xa[i] = p == 0 ? mine : other;
    xr[i] = p == 0 ? other : mine;
  }
  if (p != 0) return;
  const double fb[5] = {xa[0] + xr[2], xa[1] + xr[1], xa[2] + xr[0], xa[3] + xr[3], xa[4] + xr[4]};
#pragma unroll
  for (int k = 0; k < 5; ++k) qb[k] = 0.0;
  double sb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) sb[k] = mu * om[k];
  cand_grad(lr, sb, qb);
  feature_grad(q, d, dmax, qs, fb, qb);
}

// Parameter reduction. The gradient of the weights and bias of layer l is the sum over samples of the
// outer product (activation row) x (pre-activation adjoint row). The 189 parameters form 31 "rows": one
// per input of a layer plus one for its bias (L1: 5 + 1 rows of 10 outputs, L2: 10 + 1 of 6, L3: 6 + 1
// of 6, L4: 6 + 1 of 3). Thread t takes row t / kGroups for the samples s = t % kGroups (mod kGroups):
// one activation load, then J loads and J FMAs per sample, partial sums of a chunk in the closure
// precision and the running sums in FP64 registers for the whole trajectory.
constexpr int kGroups = 8;
constexpr int kRowTasks = 31;

struct RowTask {
  int ai;  // activation index in the row (-1: bias, activation 1)
  int d0;  // first pre-activation adjoint index
  int J;   // outputs
  int p0;  // first packed parameter index
};

__device__ __forceinline__ RowTask row_task(int r) {
  if (r < 5) return {r, 0, 10, r * 10};
  if (r == 5) return {-1, 0, 10, 50};
  if (r < 16) return {5 + (r - 6), 10, 6, 60 + (r - 6) * 6};
  if (r == 16) return {-1, 10, 6, 120};
  if (r < 23) return {15 + (r - 17), 16, 6, 126 + (r - 17) * 6};
  if (r == 23) return {-1, 16, 6, 162};
  if (r < 30) return {21 + (r - 24), 22, 3, 168 + (r - 24) * 3};
  return {-1, 22, 3, 186};
}

// Running sums in shared memory, acc[j * kTrainThreads + thread] (keeps them out of the registers that the
// closure adjoint needs).
struct GradAcc {
  double* v;
};

// Adds the rows of one chunk (ns samples) into this thread's running sums.
template <typename Tr>
__device__ __forceinline__ void accumulate_rows(const Tr* __restrict__ rows, int ns, GradAcc& acc) {
  const int r = threadIdx.x / kGroups, g = threadIdx.x % kGroups;
  if (r >= kRowTasks) return;
  const RowTask t = row_task(r);
  Tr part[10];
#pragma unroll
  for (int j = 0; j < 10; ++j) part[j] = Tr(0);
  for (int s = g; s < ns; s += kGroups) {
    const Tr* row = rows + (size_t)s * kRow;
    const Tr a = t.ai < 0 ? Tr(1) : row[t.ai];
    const Tr* d = row + kRowA + t.d0;
#pragma unroll
    for (int j = 0; j < 10; ++j)
      if (j < t.J) part[j] = fma_t(a, d[j], part[j]);
  }
#pragma unroll
  for (int j = 0; j < 10; ++j)
    if (j < t.J) acc.v[j * kTrainThreads + threadIdx.x] += (double)part[j];
}

// Sums the kGroups partial rows of every parameter in a fixed order into out[189].
template <typename Tr>
__device__ __forceinline__ void finish_rows(const GradAcc& acc, double* scratch, double* __restrict__ out) {
  const int r = threadIdx.x / kGroups, g = threadIdx.x % kGroups;
  __syncthreads();
  if (r < kRowTasks) {
    const RowTask t = row_task(r);
#pragma unroll
    for (int j = 0; j < 10; ++j)
      if (j < t.J) scratch[g * kP5 + t.p0 + j] = acc.v[j * kTrainThreads + threadIdx.x];
  }
  __syncthreads();
  if (threadIdx.x < kP5) {
    double s = 0.0;
    for (int q = 0; q < kGroups; ++q) s += scratch[q * kP5 + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

// out = J_rhs(w)^T v for the CTA's trajectory, with the parameter term v . d rhs / d theta added to acc
// (accumulate_rows). G: 5 n doubles of scratch; rows: kTrainThreads rows of kRow.
template <int M>
__device__ __forceinline__ void vjp_rhs(const double* __restrict__ w, const double* __restrict__ v,
                                        double* __restrict__ out, double* __restrict__ G, unsigned short* qu,
                                        const AdvTraj& T, typename TrainReal<M>::T* __restrict__ rows,
                                        const typename ClosureParams<M>::type& P, GradAcc& acc) {
  using Tr = typename TrainReal<M>::T;
  const int n = T.n;
  const int lr = T.a > 0.0 ? 1 : 2;
  const double cmu = -(T.a * (1.0 / T.dx));
  auto stencil = [&](int i, double s[5]) {
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      int j = i + k - 2;
      j = j < 0 ? j + n : (j >= n ? j - n : j);
      s[k] = w[j];
    }
  };
  auto mu_of = [&](int i) {
    const int ip = i + 1 == n ? 0 : i + 1, im = i == 0 ? n - 1 : i - 1;
    return T.a > 0.0 ? cmu * (v[i] - v[ip]) : cmu * (v[im] - v[i]);
  };
  __shared__ int wcount[kTrainThreads / 32];
  int queued = 0;  // stencils queued so far, the same on every thread
  // phase A: plateau stencils (linear weights) and zero adjoints; queue the rest in cell order, so that
  // the parameter sums below add in the same order on every run
  for (int base = 0; base < n; base += kTrainThreads) {
    const int i = base + threadIdx.x;
    bool need = false;
    if (i < n) {
      const double mu = mu_of(i);
      double s[5];
      stencil(i, s);
      const bool plat = adv_plateau_test<5>(s);
      need = !plat && mu != 0.0;
      if (!need) {
        double qb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (plat) {
          double dl[3], sb[3];
          Weno<5>::lin(lr, dl);
#pragma unroll
          for (int k = 0; k < 3; ++k) sb[k] = mu * dl[k];
          cand_grad(lr, sb, qb);
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) G[k * n + i] = qb[k];
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, need);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wcount[warp] = __popc(m);
    __syncthreads();
    int off = queued, tot = 0;
#pragma unroll
    for (int w = 0; w < kTrainThreads / 32; ++w) {
      off += w < warp ? wcount[w] : 0;
      tot += wcount[w];
    }
    if (need) qu[off + __popc(m & ((1u << lane) - 1u))] = (unsigned short)i;
    queued += tot;
    __syncthreads();
  }
  const int count = queued;
  // phase B: MLP stencils, two threads per stencil, kTrainThreads / 2 stencils per chunk
  for (int base = 0; base < count; base += kTrainThreads / 2) {
    const int e = base + (threadIdx.x >> 1);
    const bool valid = e < count;
    const int p = threadIdx.x & 1;
    const int i = qu[valid ? e : count - 1];
    double s[5], d[3], dmax, qs, qb[5];
    stencil(i, s);
    adv_plateau<5>(s, d, dmax, qs);
    pair_vjp<M>(s, d, dmax, qs, mu_of(i), lr, p, rows + (size_t)threadIdx.x * kRow, P, qb);
    if (valid && p == 0) {
#pragma unroll
      for (int k = 0; k < 5; ++k) G[k * n + i] = qb[k];
    }
    __syncthreads();
    accumulate_rows<Tr>(rows, 2 * min(kTrainThreads / 2, count - base), acc);
    __syncthreads();
  }
  // gather: out_j = sum_k G[k][j + 2 - k]
  for (int j = threadIdx.x; j < n; j += kTrainThreads) {
    double sacc = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      int c = j + 2 - k;
      c = c < 0 ? c + n : (c >= n ? c - n : c);
      sacc += G[k * n + c];
    }
    out[j] = sacc;
  }
  __syncthreads();
}

template <int M>
constexpr size_t train_bwd_smem(int n) {
  return (size_t)12 * n * sizeof(double) + ((size_t)2 * n + 15) / 16 * 16 +
         (size_t)kTrainThreads * kRow * sizeof(typename TrainReal<M>::T) + (size_t)10 * kTrainThreads * sizeof(double);
}

constexpr size_t train_fwd_smem(int n) { return (size_t)3 * n * sizeof(double) + ((size_t)2 * n + 15) / 16 * 16; }

template <int M>
__global__ void __launch_bounds__(kTrainThreads, M == M_SR32 ? 2 : 1)
    k_train_bwd(const double* __restrict__ ck, const unsigned* __restrict__ signs, const double* __restrict__ vel, int n,
                double dx, double dt, int steps, int every, double gscale, double* __restrict__ seg,
                double* __restrict__ grad_part, double* __restrict__ grad_u0,
                const __grid_constant__ typename ClosureParams<M>::type P) {
  using Tr = typename TrainReal<M>::T;
  extern __shared__ double smem[];
  __shared__ int qcount;
  const int b = blockIdx.x;
  double* U = smem;
  double* S = U + n;
  double* Lam = S + n;
  double* LU = Lam + n;
  double* L2 = LU + n;
  double* V = L2 + n;
  double* R = V + n;
  double* G = R + n;
  unsigned short* qu = reinterpret_cast<unsigned short*>(G + 5 * n);
  Tr* rows = reinterpret_cast<Tr*>(reinterpret_cast<char*>(qu) + ((size_t)2 * n + 15) / 16 * 16);
  AdvTraj T;
  T.n = n;
  T.a = vel[b];
  T.dx = dx;
  GradAcc acc{reinterpret_cast<double*>(reinterpret_cast<char*>(rows) + (size_t)kTrainThreads * kRow * sizeof(Tr))};
#pragma unroll
  for (int j = 0; j < 10; ++j) acc.v[j * kTrainThreads + threadIdx.x] = 0.0;
  for (int i = threadIdx.x; i < n; i += kTrainThreads) Lam[i] = 0.0;
  const int K = (steps + every - 1) / every;
  const int words = (n + 31) >> 5;
  const int segl = every < steps ? every : steps;  // steps per segment (the scratch holds one segment)
  double* sg = seg + (size_t)b * segl * 3 * n;
  Tally tally;
#pragma unroll 1
  for (int c = K - 1; c >= 0; --c) {
    const int k0 = c * every, k1 = min(k0 + every, steps);
    const double* cp = ck + ((size_t)b * K + c) * n;
    for (int i = threadIdx.x; i < n; i += kTrainThreads) U[i] = cp[i];
    __syncthreads();
#pragma unroll 1
    for (int k = k0; k < k1; ++k) ssprk3_step_cta<M>(U, S, G, T, dt, qu, &qcount, P, tally, sg + (size_t)(k - k0) * 3 * n);
#pragma unroll 1
    for (int k = k1 - 1; k >= k0; --k) {
      const double* st = sg + (size_t)(k - k0) * 3 * n;
      const unsigned* sw = signs + ((size_t)b * steps + k) * words * 2;
      // The three stages in reverse, each with one VJP (a single call site keeps the kernel's code small):
      //   r = 2: u3 = u/3 + 2/3 (u2 + dt L(u2));  r = 1: u2 = 3/4 u + 1/4 (u1 + dt L(u1));  r = 0: u1 = u + dt L(u)
#pragma unroll 1
      for (int r = 2; r >= 0; --r) {
        for (int i = threadIdx.x; i < n; i += kTrainThreads) {
          if (r == 2) {
            const unsigned pos = sw[(i >> 5) * 2], neg = sw[(i >> 5) * 2 + 1], bit = 1u << (i & 31);
            const double code = (pos & bit) ? 1.0 : ((neg & bit) ? -1.0 : 0.0);
            const double lam = Lam[i] + gscale * code;
            Lam[i] = lam;
            V[i] = (2.0 / 3.0) * dt * lam;
          } else if (r == 1) {
            const double l2 = (2.0 / 3.0) * Lam[i] + R[i];
            L2[i] = l2;
            LU[i] = Lam[i] / 3.0;
            V[i] = 0.25 * dt * l2;
          } else {
            const double l1 = 0.25 * L2[i] + R[i];
            LU[i] += 0.75 * L2[i];
            L2[i] = l1;
            V[i] = dt * l1;
          }
          S[i] = st[r * n + i];
        }
        __syncthreads();
        vjp_rhs<M>(S, V, R, G, qu, T, rows, P, acc);
      }
      for (int i = threadIdx.x; i < n; i += kTrainThreads) Lam[i] = LU[i] + L2[i] + R[i];
      __syncthreads();
    }
  }
  if (grad_u0)
    for (int i = threadIdx.x; i < n; i += kTrainThreads) grad_u0[(size_t)b * n + i] = Lam[i];
  finish_rows<Tr>(acc, reinterpret_cast<double*>(rows), grad_part + (size_t)b * kP5);
}

// Fixed-order sums over trajectories: grad_out[p] = sum_b grad_part[b][p]; loss_out = lscale * sum_b loss_part[b].
__global__ void __launch_bounds__(256) k_train_reduce(const double* __restrict__ loss_part, const double* __restrict__ grad_part,
                                                      int B, double lscale, double* __restrict__ loss_out,
                                                      double* __restrict__ grad_out) {
  if (grad_out && threadIdx.x < kP5) {
    double s = 0.0;
    for (int b = 0; b < B; ++b) s += grad_part[(size_t)b * kP5 + threadIdx.x];
    grad_out[threadIdx.x] = s;
  }
  if (loss_out && threadIdx.x == 255) {
    double s = 0.0;
    for (int b = 0; b < B; ++b) s += loss_part[b];
    *loss_out = s * lscale;
  }
}

}  // namespace wsr
