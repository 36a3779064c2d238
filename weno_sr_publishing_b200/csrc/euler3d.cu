// 3D Euler WENO5 (JS / SR) finite-volume step on sm_100a: characteristic normal reconstruction with the
// reference's lr = 1 round trip, 2 x 2 Gauss-point transverse reconstruction, EVILIN or HLLC face fluxes,
// and the reference's in-place three-stage Runge-Kutta update.
//
// Reference (code/snapshot/warp_weno5_3d_rk3/): kernels.py (Euler algebra, EVILIN 121-223, Roe 226-268,
// eigenvectors 272-500, JS face and Gauss reconstruction 503-672, boundary 776-829, max speed 832-845,
// normal/transverse/flux kernels 869-1076, RK stages 1079-1163); mlp_normal_scalar.py and mlp_kernels.py
// (the characteristic SR reconstruction and the closure); solver.py:165-329 (sweep order, Gauss flags,
// dt rule, stages). The HLLC flux and the x-low inflow state have no counterpart there: the 3D workload
// asks for them (the 2D HLLC of for_paper_results/solvers/weno5_hllc.py:22-113 in three dimensions).
//
// The file is compiled twice. The main object, with the extern "C" entry points and the WENO5-JS stages, is
// built without floating-point contraction (-fmad=false), like the reference's Warp module (fuse_fp False), so
// that the WENO5-JS path reproduces the reference bit for bit. The SR stages (FP64/FP32/BF16 closure), which
// agree with the reference only to rounding anyway, come from a second object built with contraction
// (-DWSR_EULER3D_SR_UNIT): euler3d_sr_stage below, called by the main object with plain arguments. The MLP
// keeps explicit fused multiply-adds in both (closure.cuh fma_t).
//
// Work decomposition, per direction d of a stage:
//   k3_normal  one thread per cell of the normal-extended block: the characteristic reconstruction of the
//              cell's low-face (lr 2) and high-face (lr 1) states, 10 scalar closures;
//   k3_trans   one thread per cell: the first transverse Gauss pass for both Gauss points of both normal
//              arrays (the reference recomputes the first pass for each of the four flags; two of them are
//              the same, so four arrays hold all that the flags need): 10 stencils, each read once and
//              reconstructed at both Gauss points (one SR closure evaluation serves both), 20 values;
//   k3_flux    one thread per face: the second transverse pass of the four Gauss points of both adjacent
//              cells (20 stencils, each giving two of the 40 values) and the four face fluxes, summed in the
//              reference's flag order and scaled by dt/h.
// k3_update applies the four-point flux difference of all three directions and, at the third stage, takes
// the maximum wave speed for the next step's dt, which k3_step_begin turns into dt on the device.
#include <cuda_runtime.h>

#include <cstring>

// the 3D closure kernels apply the FP64 activations in rolled loops (closure.cuh)
#define WSR_ROLL_FP64_ACT 1
#include "closure.cuh"
#include "wsr_ctx.cuh"

using namespace wsr;
using namespace wsr_detail;

namespace {

constexpr int kT3 = 128;
constexpr double kGam = 1.4;

struct V5 {
  double v[5];
};

struct Inflow {
  double v[5];
  int on;
};

struct Dims3 {
  int nx, ny, nz, px, py, pz;
  __host__ __device__ size_t cell(int k, int j, int i) const { return ((size_t)k * py + j) * px + i; }
};

__device__ __forceinline__ V5 ld5(const double* __restrict__ a, size_t c) {
  V5 x;
#pragma unroll
  for (int q = 0; q < 5; ++q) x.v[q] = a[c * 5 + q];
  return x;
}

__device__ __forceinline__ void st5(double* __restrict__ a, size_t c, const V5& x) {
#pragma unroll
  for (int q = 0; q < 5; ++q) a[c * 5 + q] = x.v[q];
}

// --- Euler algebra (kernels.py:29-119) ---------------------------------------------------------------
__device__ __forceinline__ V5 con_to_pri(const V5& c) {
  V5 p;
  p.v[0] = c.v[0];
  p.v[1] = c.v[1] / c.v[0];
  p.v[2] = c.v[2] / c.v[0];
  p.v[3] = c.v[3] / c.v[0];
  p.v[4] = (kGam - 1.0) * (c.v[4] - 0.5 * c.v[0] * (p.v[1] * p.v[1] + p.v[2] * p.v[2] + p.v[3] * p.v[3]));
  return p;
}

__device__ __forceinline__ V5 pri_to_con(const V5& p) {
  V5 c;
  c.v[0] = p.v[0];
  c.v[1] = p.v[0] * p.v[1];
  c.v[2] = p.v[0] * p.v[2];
  c.v[3] = p.v[0] * p.v[3];
  c.v[4] = p.v[4] / (kGam - 1.0) + 0.5 * p.v[0] * (p.v[1] * p.v[1] + p.v[2] * p.v[2] + p.v[3] * p.v[3]);
  return c;
}

template <int DIR>
__device__ __forceinline__ V5 flux_pri(const V5& p) {
  const double rho = p.v[0], u = p.v[1], v = p.v[2], w = p.v[3], pr = p.v[4];
  const double e = 0.5 * rho * (u * u + v * v + w * w) + pr / (kGam - 1.0);
  V5 f;
  if constexpr (DIR == 1) {
    f.v[0] = rho * u; f.v[1] = rho * u * u + pr; f.v[2] = rho * u * v; f.v[3] = rho * u * w; f.v[4] = u * (pr + e);
  } else if constexpr (DIR == 2) {
    f.v[0] = rho * v; f.v[1] = rho * u * v; f.v[2] = rho * v * v + pr; f.v[3] = rho * v * w; f.v[4] = v * (pr + e);
  } else {
    f.v[0] = rho * w; f.v[1] = rho * u * w; f.v[2] = rho * v * w; f.v[3] = rho * w * w + pr; f.v[4] = w * (pr + e);
  }
  return f;
}

template <int DIR>
__device__ __forceinline__ V5 clamped_flux(V5 p) {
  p.v[0] = fmax(p.v[0], 1.0e-15);
  p.v[4] = fmax(p.v[4], 1.0e-15);
  return flux_pri<DIR>(p);
}

// EVILIN interface state (kernels.py:121-223)
template <int DIR>
__device__ V5 evilin(const V5& ul0, const V5& ur0, double dt_dx) {
  const double eps = 1.0e-15;
  V5 wl0 = con_to_pri(ul0), wr0 = con_to_pri(ur0);
  wl0.v[0] = fmax(wl0.v[0], eps); wl0.v[4] = fmax(wl0.v[4], eps);
  wr0.v[0] = fmax(wr0.v[0], eps); wr0.v[4] = fmax(wr0.v[4], eps);
  const double unl0 = wl0.v[DIR], unr0 = wr0.v[DIR];
  const double al0 = sqrt(kGam * wl0.v[4] / wl0.v[0]), ar0 = sqrt(kGam * wr0.v[4] / wr0.v[0]);
  double smax = fmax(fabs(unl0) + al0, fabs(unr0) + ar0);
  smax = fmax(smax, eps);
  const double dx_dt = 1.0 / dt_dx, courant = smax * dt_dx;
  const V5 fl = clamped_flux<DIR>(wl0), fr = clamped_flux<DIR>(wr0);
  V5 ulw, ffo, fgf, ulh, urh;
#pragma unroll
  for (int c = 0; c < 5; ++c) ulw.v[c] = 0.5 * (ul0.v[c] + ur0.v[c]) - 0.5 * dt_dx * (fr.v[c] - fl.v[c]);
  V5 wlw = con_to_pri(ulw);
  wlw.v[0] = fmax(wlw.v[0], eps); wlw.v[4] = fmax(wlw.v[4], eps);
  const V5 flw = clamped_flux<DIR>(wlw);
#pragma unroll
  for (int c = 0; c < 5; ++c) ffo.v[c] = 0.25 * (fl.v[c] + 2.0 * flw.v[c] + fr.v[c] - dx_dt * (ur0.v[c] - ul0.v[c]));
  const double theta = (1.0 - courant) / (1.0 + courant);
#pragma unroll
  for (int c = 0; c < 5; ++c) fgf.v[c] = theta * flw.v[c] + (1.0 - theta) * ffo.v[c];
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    ulh.v[c] = ul0.v[c] - dt_dx * (fgf.v[c] - fl.v[c]);
    urh.v[c] = ur0.v[c] - dt_dx * (fr.v[c] - fgf.v[c]);
  }
  V5 wl = con_to_pri(ulh), wr = con_to_pri(urh);
  wl.v[0] = fmax(wl.v[0], eps); wl.v[4] = fmax(wl.v[4], eps);
  wr.v[0] = fmax(wr.v[0], eps); wr.v[4] = fmax(wr.v[4], eps);
  const double rho_bar = fmax(0.5 * (wl.v[0] + wr.v[0]), eps), p_bar = fmax(0.5 * (wl.v[4] + wr.v[4]), eps);
  const double a_bar = fmax(sqrt(kGam * p_bar / rho_bar), eps);
  const double c1 = rho_bar * a_bar, c2 = rho_bar / a_bar;
  const double unle = wl.v[DIR], unre = wr.v[DIR];
  const double u_star = 0.5 * (unle + unre) - 0.5 * (wr.v[4] - wl.v[4]) / c1;
  double p_star = 0.5 * (wl.v[4] + wr.v[4]) - 0.5 * (unre - unle) * c1;
  const double rho_sl = fmax(wl.v[0] + (unle - u_star) * c2, eps), rho_sr = fmax(wr.v[0] + (u_star - unre) * c2, eps);
  p_star = fmax(p_star, eps);
  const double u_bar = 0.5 * (unle + unre);
  V5 wf = wr;
  if (u_bar - a_bar >= 0.0) {
    wf = wl;
  } else if (u_bar >= 0.0) {
    wf = wl; wf.v[0] = rho_sl; wf.v[DIR] = u_star; wf.v[4] = p_star;
  } else if (u_bar + a_bar >= 0.0) {
    wf = wr; wf.v[0] = rho_sr; wf.v[DIR] = u_star; wf.v[4] = p_star;
  }
  wf.v[0] = fmax(wf.v[0], eps);
  wf.v[4] = fmax(wf.v[4], eps);
  return pri_to_con(wf);
}

__device__ __forceinline__ double sfloor(double d, double tiny) {
  return fabs(d) < tiny ? (d < 0.0 ? -tiny : tiny) : d;
}

// HLLC in 3D: Davis speeds, 1e-16 floors, both tangential velocities carried by the star state.
template <int DIR>
__device__ V5 hllc(const V5& ul0, const V5& ur0) {
  const double tiny = 1.0e-16;
  const V5 wl = con_to_pri(ul0), wr = con_to_pri(ur0);
  const double rho_l = fmax(wl.v[0], tiny), rho_r = fmax(wr.v[0], tiny);
  const double p_l = fmax(wl.v[4], tiny), p_r = fmax(wr.v[4], tiny);
  const double a_l = sqrt(kGam * p_l / rho_l), a_r = sqrt(kGam * p_r / rho_r);
  const double un_l = wl.v[DIR], un_r = wr.v[DIR];
  const double s_l = fmin(un_l - a_l, un_r - a_r), s_r = fmax(un_l + a_l, un_r + a_r);
  const V5 f_l = flux_pri<DIR>(wl), f_r = flux_pri<DIR>(wr);
  if (0.0 <= s_l) return f_l;
  if (0.0 >= s_r) return f_r;
  const double denom = sfloor(rho_l * (s_l - un_l) - rho_r * (s_r - un_r), tiny);
  const double s_star = (p_r - p_l + rho_l * un_l * (s_l - un_l) - rho_r * un_r * (s_r - un_r)) / denom;
  const bool right = s_star < 0.0;
  const V5& u_side = right ? ur0 : ul0;
  const V5& w_side = right ? wr : wl;
  const V5& f_side = right ? f_r : f_l;
  const double s_side = right ? s_r : s_l;
  const double rho = fmax(w_side.v[0], tiny), p = fmax(w_side.v[4], tiny), un = w_side.v[DIR];
  const double factor = rho * (s_side - un) / sfloor(s_side - s_star, tiny);
  V5 us;
  us.v[0] = factor;
#pragma unroll
  for (int c = 1; c <= 3; ++c) us.v[c] = factor * (c == DIR ? s_star : w_side.v[c]);
  us.v[4] = factor * ((u_side.v[4] / rho) + (s_star - un) * (s_star + p / (rho * sfloor(s_side - un, tiny))));
  V5 out;
#pragma unroll
  for (int c = 0; c < 5; ++c) out.v[c] = f_side.v[c] + s_side * (us.v[c] - u_side.v[c]);
  return out;
}

// --- Roe average and eigenvectors (kernels.py:226-500) ----------------------------------------------
__device__ __forceinline__ V5 roe(const V5& l, const V5& r) {
  const double g = kGam;
  const double rl = l.v[0], ul = l.v[1] / rl, vl = l.v[2] / rl, wl = l.v[3] / rl, el = l.v[4];
  const double pl = (g - 1.0) * (el - 0.5 * rl * (ul * ul + vl * vl + wl * wl));
  const double hl = (el + pl) / rl;
  const double rr = r.v[0], ur = r.v[1] / rr, vr = r.v[2] / rr, wr = r.v[3] / rr, er = r.v[4];
  const double pr = (g - 1.0) * (er - 0.5 * rr * (ur * ur + vr * vr + wr * wr));
  const double hr = (er + pr) / rr;
  const double sl = sqrt(rl), sr = sqrt(rr), inv = 1.0 / (sl + sr);
  const double u = (sl * ul + sr * ur) * inv, v = (sl * vl + sr * vr) * inv, w = (sl * wl + sr * wr) * inv;
  const double h = (sl * hl + sr * hr) * inv, rho = sl * sr;
  const double q2 = u * u + v * v + w * w;
  V5 o;
  o.v[0] = rho; o.v[1] = rho * u; o.v[2] = rho * v; o.v[3] = rho * w;
  o.v[4] = (rho * h + 0.5 * (g - 1.0) * rho * q2) / g;
  return o;
}

// Eigen-system of direction DIR at a conserved state: normal velocity component DIR, tangential
// components T1 < T2.
template <int DIR>
struct Eig {
  static constexpr int T1 = DIR == 1 ? 2 : 1, T2 = DIR == 3 ? 2 : 3;
  double un, a1, a2, c, h, vt, gm1, c2;
  __device__ explicit Eig(const V5& s) {
    gm1 = kGam - 1.0;
    const double rho = s.v[0], u = s.v[1] / rho, v = s.v[2] / rho, w = s.v[3] / rho, e = s.v[4];
    vt = u * u + v * v + w * w;
    const double p = gm1 * (e - 0.5 * rho * vt);
    c = sqrt(kGam * p / rho);
    c2 = c * c;
    h = 0.5 * vt + c2 / gm1;
    const double vel[4] = {0.0, u, v, w};
    un = vel[DIR];
    a1 = vel[T1];
    a2 = vel[T2];
  }
  // L (rows scaled by gm1 / (2 c^2)) applied to x
  __device__ V5 left(const V5& x) const {
    double L[5][5];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int k = 0; k < 5; ++k) L[r][k] = 0.0;
    L[0][0] = h + c * (un - c) / gm1;
    L[0][DIR] = -(un + c / gm1); L[0][T1] = -a1; L[0][T2] = -a2; L[0][4] = 1.0;
    L[1][0] = -2.0 * h + 4.0 * c2 / gm1;
    L[1][DIR] = 2.0 * un; L[1][T1] = 2.0 * a1; L[1][T2] = 2.0 * a2; L[1][4] = -2.0;
    L[2][0] = -2.0 * a1 * c2 / gm1; L[2][T1] = 2.0 * c2 / gm1;
    L[3][0] = -2.0 * a2 * c2 / gm1; L[3][T2] = 2.0 * c2 / gm1;
    L[4][0] = h - c * (un + c) / gm1;
    L[4][DIR] = -(un - c / gm1); L[4][T1] = -a1; L[4][T2] = -a2; L[4][4] = 1.0;
    const double scale = gm1 / (2.0 * c2);
    V5 y;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double t = 0.0;
#pragma unroll
      for (int k = 0; k < 5; ++k) t = t + (L[r][k] * scale) * x.v[k];
      y.v[r] = t;
    }
    return y;
  }
  __device__ V5 right(const V5& x) const {
    double R[5][5];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int k = 0; k < 5; ++k) R[r][k] = 0.0;
    R[0][0] = 1.0; R[0][1] = 1.0; R[0][4] = 1.0;
    R[DIR][0] = un - c; R[DIR][1] = un; R[DIR][4] = un + c;
    R[T1][0] = a1; R[T1][1] = a1; R[T1][2] = 1.0; R[T1][4] = a1;
    R[T2][0] = a2; R[T2][1] = a2; R[T2][3] = 1.0; R[T2][4] = a2;
    R[4][0] = h - un * c; R[4][1] = 0.5 * vt; R[4][2] = a1; R[4][3] = a2; R[4][4] = h + un * c;
    V5 y;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double t = 0.0;
#pragma unroll
      for (int k = 0; k < 5; ++k) t = t + R[r][k] * x.v[k];
      y.v[r] = t;
    }
    return y;
  }
};

// --- scalar reconstruction: JS with IEEE divisions (kernels.py:503-672), or the SR closure -----------
__device__ __forceinline__ double js3(const double q[5], int head) {
  const Lin3 d = linear_weights(head);
  const double t0 = q[0] - 2.0 * q[1] + q[2], u0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
  const double t1 = q[1] - 2.0 * q[2] + q[3], u1 = q[1] - q[3];
  const double t2 = q[2] - 2.0 * q[3] + q[4], u2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
  const double b0 = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
  const double b1 = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
  const double b2 = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
  const double i0 = 1.0 / (1.0e-6 + b0), i1 = 1.0 / (1.0e-6 + b1), i2 = 1.0 / (1.0e-6 + b2);
  const double a0 = d.d0 * i0 * i0, a1 = d.d1 * i1 * i1, a2 = d.d2 * i2 * i2;
  const double s = a0 + a1 + a2;
  double c[3];
  candidates(q, head, c);
  return (a0 / s) * c[0] + (a1 / s) * c[1] + (a2 / s) * c[2];
}

// WENO-Z (Borges et al. 2008, p = 2) with eps = h^2 of the reconstruction direction and IEEE divisions
// (weno_z_borges_p2_results/weno5_3d_kernels_z.py:527-562, 673-706): tau5 = |beta0 - beta2|,
// alpha_k = d_k (1 + (tau5 / (beta_k + eps))^2), w_k = alpha_k / sum. Same betas, linear weights and
// candidates as js3, so the two differ only in the alphas.
// z3 in two parts: the head-independent ratios tau5 / (beta_k + eps) and one head's weights and candidates
struct Z3Ratio {
  double r0, r1, r2;
};

__device__ __forceinline__ Z3Ratio z3_ratio(const double q[5], double eps) {
  const double t0 = q[0] - 2.0 * q[1] + q[2], u0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
  const double t1 = q[1] - 2.0 * q[2] + q[3], u1 = q[1] - q[3];
  const double t2 = q[2] - 2.0 * q[3] + q[4], u2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
  const double b0 = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
  const double b1 = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
  const double b2 = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
  const double tau = fabs(b0 - b2);
  return Z3Ratio{tau / (b0 + eps), tau / (b1 + eps), tau / (b2 + eps)};
}

__device__ __forceinline__ double z3_head(const double q[5], const Z3Ratio& r, int head) {
  const Lin3 d = linear_weights(head);
  const double a0 = d.d0 * (1.0 + r.r0 * r.r0), a1 = d.d1 * (1.0 + r.r1 * r.r1), a2 = d.d2 * (1.0 + r.r2 * r.r2);
  const double s = a0 + a1 + a2;
  double c[3];
  candidates(q, head, c);
  return (a0 / s) * c[0] + (a1 / s) * c[1] + (a2 / s) * c[2];
}

__device__ __forceinline__ double z3(const double q[5], int head, double eps) {
  return z3_head(q, z3_ratio(q, eps), head);
}

// rho > 0 and p > 0 of a conserved 3D state
__device__ __forceinline__ bool admissible5(const V5& q) {
  const double rho = q.v[0];
  if (!(rho > 0.0)) return false;
  const double p = (kGam - 1.0) * (q.v[4] - 0.5 * (q.v[1] * q.v[1] + q.v[2] * q.v[2] + q.v[3] * q.v[3]) / rho);
  return p > 0.0;
}

template <int M>
__device__ __forceinline__ double recon(const double q[5], int head, const typename ClosureParams<M>::type& P,
                                        int opts, Tally& tally) {
  if constexpr (M == M_JS) {
    return js3(q, head);
  } else if constexpr (M == M_Z) {
    return z3(q, head, P.ex);  // P.ex = h^2 of this kernel's reconstruction direction
  } else {
    if (plateau5(q)) {
      ++tally.plateau;
      return linear_value(q, head);
    }
    ++tally.mlp;
    double a0, a1, a2;
    sr_betas<M>(q, P, a0, a1, a2);
    return sr_value<M>(q, head, a0, a1, a2, opts, tally);
  }
}

// Both Gauss-point values (heads 2 and 3) of one transverse stencil. The SR closure's weights are a function of the
// five stencil values alone, so one closure evaluation serves both heads (the reference evaluates it once per head,
// with the same result); WENO-Z shares its smoothness ratios between the heads the same way.
template <int M>
__device__ __forceinline__ void recon_pair(const double q[5], const typename ClosureParams<M>::type& P, int opts,
                                           Tally& tally, double& v2, double& v3) {
  if constexpr (M == M_JS) {
    v2 = js3(q, 2);  // two calls: measured faster here than sharing the smoothness factors (fewer live registers)
    v3 = js3(q, 3);
  } else if constexpr (M == M_Z) {
    const Z3Ratio r = z3_ratio(q, P.ex);
    v2 = z3_head(q, r, 2);
    v3 = z3_head(q, r, 3);
  } else {
    if (plateau5(q)) {
      ++tally.plateau;
      v2 = linear_value(q, 2);
      v3 = linear_value(q, 3);
      return;
    }
    ++tally.mlp;
    double a0, a1, a2;
    sr_betas<M>(q, P, a0, a1, a2);
    v2 = sr_value<M>(q, 2, a0, a1, a2, opts, tally);
    v3 = sr_value<M>(q, 3, a0, a1, a2, opts, tally);
  }
}

// --- control block -------------------------------------------------------------------------------
struct Ctl3 {
  double t, t_end, dt, cfl, hmin;
  unsigned long long speed_bits;
  int steps, done, max_steps, pad;
};

__device__ __forceinline__ unsigned long long speed_of(const V5& q) {
  const V5 p = con_to_pri(q);
  const double a = sqrt(kGam * p.v[4] / p.v[0]);
  const double s = fmax(fabs(p.v[1]) + a, fmax(fabs(p.v[2]) + a, fabs(p.v[3]) + a));
  return (unsigned long long)__double_as_longlong(s);
}

__device__ __forceinline__ void block_max(unsigned long long v, unsigned long long* dst) {
  __shared__ unsigned long long red[kT3 / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = red[0];
    for (int w = 1; w < kT3 / 32; ++w) m = red[w] > m ? red[w] : m;
    atomicMax(dst, m);
  }
}

__global__ void __launch_bounds__(kT3) k3_max_speed(const double* __restrict__ q, Dims3 d, Ctl3* ctl) {
  const int i = blockIdx.x * kT3 + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  unsigned long long s = 0;
  if (i < d.nx) s = speed_of(ld5(q, d.cell(k + 3, j + 3, i + 3)));
  block_max(s, &ctl->speed_bits);
}

// dt = cfl hmin / max speed (1e10 below 1e-15), clipped to t_end (solver.py:303-316); one thread.
__global__ void k3_step_begin(Ctl3* ctl, double* dts) {
  if (ctl->done) return;
  if (ctl->t == ctl->t_end || ctl->steps >= ctl->max_steps) {
    ctl->done = 1;
    return;
  }
  const double m = __longlong_as_double((long long)ctl->speed_bits);
  double dt = m < 1.0e-15 ? 1.0e10 : ctl->cfl * ctl->hmin / m;
  if (ctl->t + dt > ctl->t_end) dt = ctl->t_end - ctl->t;
  ctl->dt = dt;
  ctl->t = ctl->t + dt;
  if (dts) dts[ctl->steps] = dt;
  ctl->speed_bits = 0ull;
}

__global__ void k3_step_end(Ctl3* ctl) {
  if (!ctl->done) ctl->steps += 1;
}

// --- boundary (kernels.py:776-829) --------------------------------------------------------------------
template <int AXIS>
__global__ void __launch_bounds__(kT3) k3_bc(double* __restrict__ q, Dims3 d, Inflow in, const Ctl3* ctl) {
  if (ctl && ctl->done) return;
  const int a = blockIdx.x * kT3 + threadIdx.x, b = blockIdx.y;
  if constexpr (AXIS == 1) {  // (k, j) over (pz, py)
    if (a >= d.py) return;
    const int j = a, k = b;
    V5 lo = ld5(q, d.cell(k, j, 3)), hi = ld5(q, d.cell(k, j, d.nx + 2));
    if (in.on) lo = V5{{in.v[0], in.v[1], in.v[2], in.v[3], in.v[4]}};
    for (int g = 0; g < 3; ++g) {
      st5(q, d.cell(k, j, g), lo);
      st5(q, d.cell(k, j, d.nx + 3 + g), hi);
    }
  } else if constexpr (AXIS == 2) {  // (k, i) over (pz, px)
    if (a >= d.px) return;
    const int i = a, k = b;
    const V5 lo = ld5(q, d.cell(k, 3, i)), hi = ld5(q, d.cell(k, d.ny + 2, i));
    for (int g = 0; g < 3; ++g) {
      st5(q, d.cell(k, g, i), lo);
      st5(q, d.cell(k, d.ny + 3 + g, i), hi);
    }
  } else {  // (j, i) over (py, px)
    if (a >= d.px) return;
    const int i = a, j = b;
    const V5 lo = ld5(q, d.cell(3, j, i)), hi = ld5(q, d.cell(d.nz + 2, j, i));
    for (int g = 0; g < 3; ++g) {
      st5(q, d.cell(g, j, i), lo);
      st5(q, d.cell(d.nz + 3 + g, j, i), hi);
    }
  }
}

template <int DIR>
__device__ __forceinline__ int3 step_of() {
  return DIR == 1 ? make_int3(1, 0, 0) : (DIR == 2 ? make_int3(0, 1, 0) : make_int3(0, 0, 1));  // (i, j, k)
}

// Thread tiling of a 128-thread block for a kernel whose 5-point stencils run along axis AX (1 = i, 2 = j, 3 = k):
// 32 (i) x 4 tiles. When the stencil runs along j or k the four warp rows lie along that axis, so that a block's
// warps read 8 overlapping stencil rows through L1 instead of 20 rows that only neighbouring blocks share (through
// L2); when it runs along i they lie along j. 32-wide rows also fill the launch when a row is not a multiple of 128
// cells (224 faces: 7 full warps instead of two 128-thread blocks with 32 idle threads).
template <int AX>
struct Tile3 {
  static constexpr int kRows = AX == 1 ? 2 : AX;  // the axis of the tile's four warp rows
  static constexpr int bi = 32, bj = kRows == 2 ? kT3 / 32 : 1, bk = kRows == 3 ? kT3 / 32 : 1;
  __device__ static int i() { return (int)blockIdx.x * bi + (int)(threadIdx.x & 31); }
  __device__ static int j() { return (int)blockIdx.y * bj + (kRows == 2 ? (int)(threadIdx.x >> 5) : 0); }
  __device__ static int k() { return (int)blockIdx.z * bk + (kRows == 3 ? (int)(threadIdx.x >> 5) : 0); }
  static dim3 grid(int ni, int nj, int nk) { return dim3((ni + bi - 1) / bi, (nj + bj - 1) / bj, (nk + bk - 1) / bk); }
};

// --- normal reconstruction (kernels.py:869-927; mlp_normal_scalar.py) ---------------------------------
template <int M, int DIR>
__global__ void __launch_bounds__(kT3, 4) k3_normal(const double* __restrict__ q, double* __restrict__ nl,
                                                    double* __restrict__ nr, Dims3 d, int ni, int nj, int nk, int opts,
                                                    const Ctl3* ctl, unsigned long long* counters,
                                                    const __grid_constant__ typename ClosureParams<M>::type P) {
  if (ctl && ctl->done) return;
  using TL = Tile3<DIR>;
  const int i = TL::i(), j = TL::j(), k = TL::k();
  if (i >= ni || j >= nj || k >= nk) return;
  const int3 e = step_of<DIR>();
  Tally tally;
  V5 ch[5];
#pragma unroll
  for (int p = 0; p < 5; ++p) ch[p] = ld5(q, d.cell(k + p * e.z, j + p * e.y, i + p * e.x));
  Eig<DIR> E(roe(ch[1], ch[2]));
  const size_t o = d.cell(k, j, i);
  // side 0: the lr = 2 value (low face); side 1: the lr = 1 value (high face) of the stencil round-tripped
  // through side 0's eigenvectors. One loop, so the closure is inlined once.
#pragma unroll 1
  for (int side = 0; side < 2; ++side) {
    if (side == 1) {
#pragma unroll
      for (int p = 0; p < 5; ++p) ch[p] = E.right(ch[p]);
      E = Eig<DIR>(roe(ch[2], ch[3]));
    }
#pragma unroll
    for (int p = 0; p < 5; ++p) ch[p] = E.left(ch[p]);
    V5 cv;
#pragma unroll 1
    for (int c = 0; c < 5; ++c) {
      const double st[5] = {ch[0].v[c], ch[1].v[c], ch[2].v[c], ch[3].v[c], ch[4].v[c]};
      cv.v[c] = recon<M>(st, side == 0 ? 1 : 0, P, opts, tally);
    }
    V5 face = E.right(cv);
    if constexpr (M != M_JS && M != M_Z) {
      if ((opts & OPT_JS_FALLBACK) && !admissible5(face)) {
        // positivity fallback: the five characteristic values of this face again with WENO5-JS weights
#pragma unroll 1
        for (int c = 0; c < 5; ++c) {
          const double st[5] = {ch[0].v[c], ch[1].v[c], ch[2].v[c], ch[3].v[c], ch[4].v[c]};
          cv.v[c] = js3(st, side == 0 ? 1 : 0);
        }
        face = E.right(cv);
        ++tally.fallbacks;
      }
    }
    st5(side == 0 ? nl : nr, o, face);
  }

  if (counters && (opts & OPT_COUNT)) {
    if (tally.mlp) atomicAdd(&counters[0], (unsigned long long)tally.mlp);
    if (tally.plateau) atomicAdd(&counters[1], (unsigned long long)tally.plateau);
  }
  if (counters && tally.fallbacks) atomicAdd(&counters[6], (unsigned long long)tally.fallbacks);
}

// --- first transverse pass: both Gauss points of both normal arrays ------------------------------------
template <int M, int TA>
__global__ void __launch_bounds__(kT3) k3_trans(const double* __restrict__ nl, const double* __restrict__ nr,
                                                double* __restrict__ a_l1, double* __restrict__ a_l2,
                                                double* __restrict__ a_r1, double* __restrict__ a_r2, Dims3 d, int ni,
                                                int nj, int nk, int opts, const Ctl3* ctl,
                                                unsigned long long* counters,
                                                const __grid_constant__ typename ClosureParams<M>::type P) {
  if (ctl && ctl->done) return;
  using TL = Tile3<TA>;
  const int i = TL::i(), j = TL::j(), k = TL::k();
  if (i >= ni || j >= nj || k >= nk) return;
  const int3 e = step_of<TA>();
  Tally tally;
  const size_t o = d.cell(k, j, i);
  // items (side, component) in one loop, so the closure is inlined once; each stencil gives both Gauss points
#pragma unroll 1
  for (int item = 0; item < 10; ++item) {
    const int side = item / 5, c = item % 5;
    const double* src = side == 0 ? nl : nr;
    double st[5];
#pragma unroll
    for (int p = 0; p < 5; ++p) st[p] = src[d.cell(k + (p + 1) * e.z, j + (p + 1) * e.y, i + (p + 1) * e.x) * 5 + c];
    double v1, v2;
    recon_pair<M>(st, P, opts, tally, v1, v2);
    (side == 0 ? a_l1 : a_r1)[o * 5 + c] = v1;
    (side == 0 ? a_l2 : a_r2)[o * 5 + c] = v2;
  }
  if (counters && (opts & OPT_COUNT)) {
    if (tally.mlp) atomicAdd(&counters[2], (unsigned long long)tally.mlp);
    if (tally.plateau) atomicAdd(&counters[3], (unsigned long long)tally.plateau);
  }
  if (counters && tally.fallbacks) atomicAdd(&counters[6], (unsigned long long)tally.fallbacks);
}

// --- second transverse pass and face fluxes (kernels.py:1015-1076; solver.py:175-199) ------------------
template <int M, int DIR, int TB, int FLUX>
__global__ void __launch_bounds__(kT3, 4) k3_flux(const double* __restrict__ a_l1, const double* __restrict__ a_l2,
                                                  const double* __restrict__ a_r1, const double* __restrict__ a_r2,
                                                  double* __restrict__ flux, Dims3 d, int kf, int jf, int iff, double h,
                                                  int opts, const Ctl3* ctl, unsigned long long* counters,
                                                  const __grid_constant__ typename ClosureParams<M>::type P) {
  if (ctl->done) return;
  using TL = Tile3<TB>;
  const int i = TL::i(), j = TL::j(), k = TL::k();
  if (i >= iff || j >= jf || k >= kf) return;
  const double dt_h = ctl->dt / h;
  const int3 e = step_of<DIR>(), eb = step_of<TB>();
  Tally tally;
  // The four Gauss-point pairs (first, second) of the face: the stencils depend on the first point only (a_?1 or
  // a_?2 along TB), the head on the second, so each pass over the first point reconstructs both second points.
  // The reference sums the four fluxes in the order (1,1), (2,1), (1,2), (2,2); s3 holds the first pass's scaled
  // (1,2) flux until the sum reaches it, so that the sum keeps that order.
  V5 acc, s3;
#pragma unroll 1
  for (int first = 1; first <= 2; ++first) {
    const double* srcl = first == 1 ? a_l1 : a_l2;
    const double* srcr = first == 1 ? a_r1 : a_r2;
    V5 pl[2], pr[2];  // [second - 1]
    // items (side, component) in one loop, so the closure is inlined once
#pragma unroll 1
    for (int item = 0; item < 10; ++item) {
      const int side = item / 5, c = item % 5;
      double st[5];
#pragma unroll
      for (int p = 0; p < 5; ++p) {
        const int kk = k + (p + 1) * eb.z, jj = j + (p + 1) * eb.y, ii = i + (p + 1) * eb.x;
        st[p] = side == 0 ? srcl[d.cell(kk + e.z, jj + e.y, ii + e.x) * 5 + c] : srcr[d.cell(kk, jj, ii) * 5 + c];
      }
      double v1, v2;
      recon_pair<M>(st, P, opts, tally, v1, v2);
      if (side == 0) {
        pl[0].v[c] = v1;
        pl[1].v[c] = v2;
      } else {
        pr[0].v[c] = v1;
        pr[1].v[c] = v2;
      }
    }
#pragma unroll 1
    for (int second = 0; second < 2; ++second) {
      V5 f;
      if constexpr (FLUX == 1)
        f = hllc<DIR>(pr[second], pl[second]);
      else
        f = flux_pri<DIR>(con_to_pri(evilin<DIR>(pr[second], pl[second], dt_h)));
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const double scaled = f.v[c] * dt_h;
        if (first == 1) {
          if (second == 0)
            acc.v[c] = scaled;
          else
            s3.v[c] = scaled;
        } else if (second == 0) {
          acc.v[c] = acc.v[c] + scaled;  // (1,1) + (2,1)
        } else {
          acc.v[c] = (acc.v[c] + s3.v[c]) + scaled;  // + (1,2) + (2,2)
        }
      }
    }
  }
  st5(flux, ((size_t)k * jf + j) * iff + i, acc);
  if (counters && (opts & OPT_COUNT)) {
    if (tally.mlp) atomicAdd(&counters[4], (unsigned long long)tally.mlp);
    if (tally.plateau) atomicAdd(&counters[5], (unsigned long long)tally.plateau);
  }
  if (counters && tally.fallbacks) atomicAdd(&counters[6], (unsigned long long)tally.fallbacks);
}

// --- RK stage update (kernels.py:1079-1163) -----------------------------------------------------------
template <int STAGE>
__global__ void __launch_bounds__(kT3) k3_update(double* __restrict__ q, double* __restrict__ q0,
                                                 const double* __restrict__ fx, const double* __restrict__ fy,
                                                 const double* __restrict__ fz, Dims3 d, Ctl3* ctl) {
  if (ctl->done) return;
  const int i = blockIdx.x * kT3 + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  unsigned long long sp = 0;
  if (i < d.nx) {
    const int nx = d.nx, ny = d.ny;
    const size_t o = d.cell(k + 3, j + 3, i + 3);
    V5 val;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double xl = fx[(((size_t)k * ny + j) * (nx + 1) + i) * 5 + c];
      const double xr = fx[(((size_t)k * ny + j) * (nx + 1) + i + 1) * 5 + c];
      const double yl = fy[(((size_t)k * (ny + 1) + j) * nx + i) * 5 + c];
      const double yr = fy[(((size_t)k * (ny + 1) + j + 1) * nx + i) * 5 + c];
      const double zl = fz[(((size_t)k * ny + j) * nx + i) * 5 + c];
      const double zr = fz[(((size_t)(k + 1) * ny + j) * nx + i) * 5 + c];
      const double old = q[o * 5 + c];
      const double adv = old - 0.25 * (xr - xl) - 0.25 * (yr - yl) - 0.25 * (zr - zl);
      double v;
      if constexpr (STAGE == 1) {
        q0[o * 5 + c] = old;
        v = adv;
      } else if constexpr (STAGE == 2) {
        v = (3.0 / 4.0) * q0[o * 5 + c] + (1.0 / 4.0) * adv;
      } else {
        v = (1.0 / 3.0) * q0[o * 5 + c] + (2.0 / 3.0) * adv;
      }
      val.v[c] = v;
      q[o * 5 + c] = v;
    }
    if constexpr (STAGE == 3) sp = speed_of(val);
  }
  if constexpr (STAGE == 3) block_max(sp, &ctl->speed_bits);
}

// --- host side -----------------------------------------------------------------------------------------
struct Ws3 {
  Ctl3* ctl;
  unsigned long long* counters;  // [2c] MLP, [2c+1] plateau for normal, transverse, flux
  double *q0, *nl, *nr, *al1, *al2, *ar1, *ar2, *fx, *fy, *fz;
};

size_t padded5(int nx, int ny, int nz) { return (size_t)(nx + 6) * (ny + 6) * (nz + 6) * 5 * sizeof(double); }

size_t ws3_bytes(int nx, int ny, int nz) {
  return align_up(sizeof(Ctl3)) + align_up(8 * sizeof(unsigned long long)) + 7 * align_up(padded5(nx, ny, nz)) +
         align_up((size_t)nz * ny * (nx + 1) * 5 * sizeof(double)) +
         align_up((size_t)nz * (ny + 1) * nx * 5 * sizeof(double)) +
         align_up((size_t)(nz + 1) * ny * nx * 5 * sizeof(double));
}

Ws3 carve3(void* base, int nx, int ny, int nz) {
  char* p = static_cast<char*>(base);
  Ws3 w;
  w.ctl = reinterpret_cast<Ctl3*>(p);
  p += align_up(sizeof(Ctl3));
  w.counters = reinterpret_cast<unsigned long long*>(p);
  p += align_up(8 * sizeof(unsigned long long));
  double** arr[7] = {&w.q0, &w.nl, &w.nr, &w.al1, &w.al2, &w.ar1, &w.ar2};
  for (int a = 0; a < 7; ++a) {
    *arr[a] = reinterpret_cast<double*>(p);
    p += align_up(padded5(nx, ny, nz));
  }
  w.fx = reinterpret_cast<double*>(p);
  p += align_up((size_t)nz * ny * (nx + 1) * 5 * sizeof(double));
  w.fy = reinterpret_cast<double*>(p);
  p += align_up((size_t)nz * (ny + 1) * nx * 5 * sizeof(double));
  w.fz = reinterpret_cast<double*>(p);
  return w;
}

struct Run3 {
  double* q;
  Dims3 d;
  double dx, dy, dz;
  int flux, opts;
  Inflow in;
};

dim3 grid3(int ni, int nj, int nk) { return dim3((ni + kT3 - 1) / kT3, nj, nk); }

// Spacing of direction D (1 x, 2 y, 3 z).
template <int D>
double spacing_of(const Run3& r) {
  return D == 1 ? r.dx : (D == 2 ? r.dy : r.dz);
}

// Kernel parameters of method M for a reconstruction along direction D: the closure for SR, the WENO-Z
// epsilon h_D^2 for Z (the product the reference forms in each kernel, weno5_3d_kernels_z.py:550).
template <int M, int D>
typename ClosureParams<M>::type kparams(const wsr_ctx* ctx, const Run3& r) {
  if constexpr (M == M_Z) {
    const double h = spacing_of<D>(r);
    return ZEps{h * h, h * h};
  } else {
    return params_of<M>(ctx);
  }
}

template <int M, int DIR, int FLUX>
int sweep3(wsr_ctx* ctx, const Run3& r, const Ws3& w, double h, cudaStream_t st) {
  const Dims3& d = r.d;
  const int nx = d.nx, ny = d.ny, nz = d.nz, px = d.px, py = d.py, pz = d.pz;
  constexpr int TA = DIR == 1 ? 2 : (DIR == 2 ? 1 : 2);
  constexpr int TB = DIR == 3 ? 1 : 3;
  const int kn = DIR == 3 ? nz + 2 : pz, jn = DIR == 2 ? ny + 2 : py, in = DIR == 1 ? nx + 2 : px;
  k3_normal<M, DIR><<<Tile3<DIR>::grid(in, jn, kn), kT3, 0, st>>>(r.q, w.nl, w.nr, d, in, jn, kn, r.opts, w.ctl,
                                                                   w.counters, kparams<M, DIR>(ctx, r));
  WSR_LAUNCHED(ctx, "k3_normal");
  const int ka = TA == 3 ? nz : (DIR == 3 ? nz + 2 : pz);
  const int ja = TA == 2 ? ny : (DIR == 2 ? ny + 2 : py);
  const int ia = TA == 1 ? nx : (DIR == 1 ? nx + 2 : px);
  k3_trans<M, TA><<<Tile3<TA>::grid(ia, ja, ka), kT3, 0, st>>>(w.nl, w.nr, w.al1, w.al2, w.ar1, w.ar2, d, ia, ja, ka,
                                                                 r.opts, w.ctl, w.counters, kparams<M, TA>(ctx, r));
  WSR_LAUNCHED(ctx, "k3_trans");
  const int kf = DIR == 3 ? nz + 1 : nz, jf = DIR == 2 ? ny + 1 : ny, iff = DIR == 1 ? nx + 1 : nx;
  double* out = DIR == 1 ? w.fx : (DIR == 2 ? w.fy : w.fz);
  k3_flux<M, DIR, TB, FLUX><<<Tile3<TB>::grid(iff, jf, kf), kT3, 0, st>>>(
      w.al1, w.al2, w.ar1, w.ar2, out, d, kf, jf, iff, h, r.opts, w.ctl, w.counters, kparams<M, TB>(ctx, r));
  WSR_LAUNCHED(ctx, "k3_flux");
  return WSR_OK;
}

template <int M, int FLUX>
int stage3(wsr_ctx* ctx, const Run3& r, const Ws3& w, int stage, cudaStream_t st) {
  const Dims3& d = r.d;
  k3_bc<1><<<dim3((d.py + kT3 - 1) / kT3, d.pz), kT3, 0, st>>>(r.q, d, r.in, w.ctl);
  k3_bc<2><<<dim3((d.px + kT3 - 1) / kT3, d.pz), kT3, 0, st>>>(r.q, d, r.in, w.ctl);
  // WSR_OPT_Z_HALO: the z ghost planes were filled by the caller (a slab of a z-decomposed grid)
  if (!(r.opts & WSR_OPT_Z_HALO)) k3_bc<3><<<dim3((d.px + kT3 - 1) / kT3, d.py), kT3, 0, st>>>(r.q, d, r.in, w.ctl);
  WSR_LAUNCHED(ctx, "k3_bc");
  int rc;
  if ((rc = sweep3<M, 1, FLUX>(ctx, r, w, r.dx, st))) return rc;
  if ((rc = sweep3<M, 2, FLUX>(ctx, r, w, r.dy, st))) return rc;
  if ((rc = sweep3<M, 3, FLUX>(ctx, r, w, r.dz, st))) return rc;
  const dim3 g = grid3(d.nx, d.ny, d.nz);
  if (stage == 1)
    k3_update<1><<<g, kT3, 0, st>>>(r.q, w.q0, w.fx, w.fy, w.fz, d, w.ctl);
  else if (stage == 2)
    k3_update<2><<<g, kT3, 0, st>>>(r.q, w.q0, w.fx, w.fy, w.fz, d, w.ctl);
  else
    k3_update<3><<<g, kT3, 0, st>>>(r.q, w.q0, w.fx, w.fy, w.fz, d, w.ctl);
  WSR_LAUNCHED(ctx, "k3_update");
  return WSR_OK;
}

}  // namespace

// One SR stage (defined in the contracted object); the stage's run description as plain arguments.
int euler3d_sr_stage(wsr_ctx* ctx, int method, double* q, int nx, int ny, int nz, double dx, double dy, double dz,
                     int flux, int opts, const double* inflow, void* workspace, int stage, cudaStream_t st);

namespace {

#ifndef WSR_EULER3D_SR_UNIT
int stage_dispatch(wsr_ctx* ctx, int method, const Run3& r, const Ws3& w, int stage, cudaStream_t st) {
  if (method == WSR_METHOD_JS)
    return r.flux == 1 ? stage3<M_JS, 1>(ctx, r, w, stage, st) : stage3<M_JS, 0>(ctx, r, w, stage, st);
  if (method == WSR_METHOD_Z)
    return r.flux == 1 ? stage3<M_Z, 1>(ctx, r, w, stage, st) : stage3<M_Z, 0>(ctx, r, w, stage, st);
  return euler3d_sr_stage(ctx, method, r.q, r.d.nx, r.d.ny, r.d.nz, r.dx, r.dy, r.dz, r.flux, r.opts,
                          r.in.on ? r.in.v : nullptr, w.ctl, stage, st);
}
#else
int stage_dispatch_sr(wsr_ctx* ctx, int method, const Run3& r, const Ws3& w, int stage, cudaStream_t st) {
  const bool h = r.flux == 1;
  switch (method) {
    case WSR_METHOD_SR_F64:
      return h ? stage3<M_SR64, 1>(ctx, r, w, stage, st) : stage3<M_SR64, 0>(ctx, r, w, stage, st);
    case WSR_METHOD_SR_F32:
      return h ? stage3<M_SR32, 1>(ctx, r, w, stage, st) : stage3<M_SR32, 0>(ctx, r, w, stage, st);
    case WSR_METHOD_SR_BF16:
      return h ? stage3<M_SRBF16, 1>(ctx, r, w, stage, st) : stage3<M_SRBF16, 0>(ctx, r, w, stage, st);
    default:
      return fail(ctx, WSR_ERR_ARG, "bad SR method %d", method);
  }
}
#endif

int check3(wsr_ctx* ctx, const double* q, int nx, int ny, int nz, double dx, double dy, double dz, int method,
           int flux, void* ws, size_t wsb) {
  if (!ctx) return WSR_ERR_ARG;
  if (nx < 5 || ny < 5 || nz < 5) return fail(ctx, WSR_ERR_ARG, "nx, ny, nz must be >= 5 (got %d, %d, %d)", nx, ny, nz);
  if ((size_t)(nx + 6) * (ny + 6) > 65535u * kT3 || nz + 6 > 65535 || ny + 6 > 65535)
    return fail(ctx, WSR_ERR_ARG, "grid %d x %d x %d too large for one launch", nx, ny, nz);
  if (method < WSR_METHOD_JS || method > WSR_METHOD_Z) return fail(ctx, WSR_ERR_ARG, "bad method %d", method);
  if (flux != WSR_FLUX3_EVILIN && flux != WSR_FLUX3_HLLC) return fail(ctx, WSR_ERR_ARG, "bad 3D flux %d", flux);
  if (method != WSR_METHOD_JS && method != WSR_METHOD_Z && !ctx->have_closure)
    return fail(ctx, WSR_ERR_NO_CLOSURE, "SR method requested before wsr_closure_upload");
  if (!q) return fail(ctx, WSR_ERR_ARG, "null state");
  if (misaligned(q)) return fail(ctx, WSR_ERR_ARG, "state must be 16-byte aligned");
  if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0)) return fail(ctx, WSR_ERR_ARG, "dx, dy, dz must be positive");
  if (!ws) return fail(ctx, WSR_ERR_ARG, "workspace is NULL");
  if (reinterpret_cast<uintptr_t>(ws) % kAlign) return fail(ctx, WSR_ERR_ARG, "workspace must be 256-byte aligned");
  if (wsb < ws3_bytes(nx, ny, nz))
    return fail(ctx, WSR_ERR_ARG, "workspace too small: %zu < %zu bytes", wsb, ws3_bytes(nx, ny, nz));
  return WSR_OK;
}

Run3 make_run(double* q, int nx, int ny, int nz, double dx, double dy, double dz, int flux, int opts,
              const double* inflow) {
  Run3 r;
  r.q = q;
  r.d = Dims3{nx, ny, nz, nx + 6, ny + 6, nz + 6};
  r.dx = dx;
  r.dy = dy;
  r.dz = dz;
  r.flux = flux;
  r.opts = opts;
  r.in.on = inflow != nullptr;
  for (int c = 0; c < 5; ++c) r.in.v[c] = inflow ? inflow[c] : 0.0;
  return r;
}

__global__ void k3_init_ctl(Ctl3* ctl, double t, double t_end, double dt, double cfl, double hmin, int max_steps) {
  ctl->t = t;
  ctl->t_end = t_end;
  ctl->dt = dt;
  ctl->cfl = cfl;
  ctl->hmin = hmin;
  ctl->speed_bits = 0ull;
  ctl->steps = 0;
  ctl->done = 0;
  ctl->max_steps = max_steps;
}

}  // namespace

#ifdef WSR_EULER3D_SR_UNIT
int euler3d_sr_stage(wsr_ctx* ctx, int method, double* q, int nx, int ny, int nz, double dx, double dy, double dz,
                     int flux, int opts, const double* inflow, void* workspace, int stage, cudaStream_t st) {
  const Run3 r = make_run(q, nx, ny, nz, dx, dy, dz, flux, opts, inflow);
  return stage_dispatch_sr(ctx, method, r, carve3(workspace, nx, ny, nz), stage, st);
}
#else

extern "C" size_t wsr_euler3d_workspace_bytes(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) return 0;
  return ws3_bytes(nx, ny, nz);
}

extern "C" int wsr_euler3d_stage(wsr_ctx* ctx, double* q, int nx, int ny, int nz, double dx, double dy, double dz,
                                 double dt, int stage, int method, int flux, int opts, const double* inflow,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check3(ctx, q, nx, ny, nz, dx, dy, dz, method, flux, workspace, workspace_bytes);
  if (rc) return rc;
  if (stage < 1 || stage > 3) return fail(ctx, WSR_ERR_ARG, "stage must be 1, 2 or 3 (got %d)", stage);
  if (!(dt > 0.0)) return fail(ctx, WSR_ERR_ARG, "dt must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  const Ws3 w = carve3(workspace, nx, ny, nz);
  const Run3 r = make_run(q, nx, ny, nz, dx, dy, dz, flux, opts, inflow);
  k3_init_ctl<<<1, 1, 0, st>>>(w.ctl, 0.0, 1.0e300, dt, 1.0, 1.0, 1);
  if (opts & (OPT_COUNT | OPT_JS_FALLBACK))
    WSR_CUDA(ctx, cudaMemsetAsync(w.counters, 0, 8 * sizeof(unsigned long long), st));
  WSR_LAUNCHED(ctx, "k3_init_ctl");
  return stage_dispatch(ctx, method, r, w, stage, st);
}

extern "C" int wsr_euler3d_max_speed(wsr_ctx* ctx, const double* q, int nx, int ny, int nz, double* out_host,
                                     void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check3(ctx, q, nx, ny, nz, 1.0, 1.0, 1.0, WSR_METHOD_JS, WSR_FLUX3_EVILIN, workspace, workspace_bytes);
  if (rc) return rc;
  if (!out_host) return fail(ctx, WSR_ERR_ARG, "null output");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  const Ws3 w = carve3(workspace, nx, ny, nz);
  const Dims3 d{nx, ny, nz, nx + 6, ny + 6, nz + 6};
  k3_init_ctl<<<1, 1, 0, st>>>(w.ctl, 0.0, 1.0e300, 0.0, 1.0, 1.0, 1);
  k3_max_speed<<<grid3(nx, ny, nz), kT3, 0, st>>>(q, d, w.ctl);
  WSR_LAUNCHED(ctx, "k3_max_speed");
  unsigned long long bits = 0;
  WSR_CUDA(ctx, cudaMemcpyAsync(&bits, &w.ctl->speed_bits, sizeof(bits), cudaMemcpyDeviceToHost, st));
  WSR_CUDA(ctx, cudaStreamSynchronize(st));
  double v;
  memcpy(&v, &bits, sizeof(v));
  *out_host = v;
  return WSR_OK;
}

extern "C" int wsr_euler3d_run(wsr_ctx* ctx, double* q, int nx, int ny, int nz, double dx, double dy, double dz,
                               double cfl, double t_start, double t_end, int max_steps, int method, int flux, int opts,
                               const double* inflow, double* dts_host, int* steps_out, double* t_out, void* workspace,
                               size_t workspace_bytes, void* stream) {
  int rc = check3(ctx, q, nx, ny, nz, dx, dy, dz, method, flux, workspace, workspace_bytes);
  if (rc) return rc;
  if (max_steps < 1) return fail(ctx, WSR_ERR_ARG, "max_steps must be >= 1");
  if (opts & WSR_OPT_Z_HALO)
    return fail(ctx, WSR_ERR_ARG, "WSR_OPT_Z_HALO needs ghost planes refreshed between stages: use wsr_euler3d_stage");
  if (!(cfl > 0.0)) return fail(ctx, WSR_ERR_ARG, "cfl must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  const Ws3 w = carve3(workspace, nx, ny, nz);
  const Run3 r = make_run(q, nx, ny, nz, dx, dy, dz, flux, opts, inflow);
  const double hmin = fmin(dx, fmin(dy, dz));
  double* dts_dev = nullptr;
  if (dts_host) WSR_CUDA(ctx, cudaMallocAsync(&dts_dev, (size_t)max_steps * sizeof(double), st));
  k3_init_ctl<<<1, 1, 0, st>>>(w.ctl, t_start, t_end, 0.0, cfl, hmin, max_steps);
  if (opts & (OPT_COUNT | OPT_JS_FALLBACK))
    WSR_CUDA(ctx, cudaMemsetAsync(w.counters, 0, 8 * sizeof(unsigned long long), st));
  k3_max_speed<<<grid3(nx, ny, nz), kT3, 0, st>>>(q, r.d, w.ctl);
  WSR_LAUNCHED(ctx, "k3_max_speed");
  for (int s = 0; s < max_steps; ++s) {
    k3_step_begin<<<1, 1, 0, st>>>(w.ctl, dts_dev);
    WSR_LAUNCHED(ctx, "k3_step_begin");
    for (int stage = 1; stage <= 3; ++stage)
      if ((rc = stage_dispatch(ctx, method, r, w, stage, st))) return rc;
    k3_step_end<<<1, 1, 0, st>>>(w.ctl);
    WSR_LAUNCHED(ctx, "k3_step_end");
    // a run to t_end polls the control block every 16 steps; once done, the queued launches return at once
    if (t_end < 1.0e300 && (s & 15) == 15) {
      int done = 0;
      WSR_CUDA(ctx, cudaMemcpyAsync(&done, &w.ctl->done, sizeof(int), cudaMemcpyDeviceToHost, st));
      WSR_CUDA(ctx, cudaStreamSynchronize(st));
      if (done) break;
    }
  }
  Ctl3 h;
  WSR_CUDA(ctx, cudaMemcpyAsync(&h, w.ctl, sizeof(h), cudaMemcpyDeviceToHost, st));
  if (dts_dev) {
    WSR_CUDA(ctx, cudaMemcpyAsync(dts_host, dts_dev, (size_t)max_steps * sizeof(double), cudaMemcpyDeviceToHost, st));
    WSR_CUDA(ctx, cudaFreeAsync(dts_dev, st));
  }
  WSR_CUDA(ctx, cudaStreamSynchronize(st));
  if (steps_out) *steps_out = h.steps;
  if (t_out) *t_out = h.t;
  return WSR_OK;
}

extern "C" int wsr_euler3d_counters(wsr_ctx* ctx, void* workspace, size_t workspace_bytes, int nx, int ny, int nz,
                                    unsigned long long* out_host) {
  if (!ctx || !workspace || !out_host) return WSR_ERR_ARG;
  if (workspace_bytes < ws3_bytes(nx, ny, nz)) return fail(ctx, WSR_ERR_ARG, "workspace too small");
  const Ws3 w = carve3(workspace, nx, ny, nz);
  WSR_CUDA(ctx, cudaMemcpy(out_host, w.counters, 7 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return WSR_OK;
}
#endif  // WSR_EULER3D_SR_UNIT
