// 2D Euler WENO5 (JS / SR) finite-volume stage kernels, sm_100a.
//
// Data layout (the reference's, warp_weno5_helpers.py:66-87): padded row-major conserved state
// u[ny+6][nx+6][4] FP64, ghost width 3. Ghost cells are never materialised: stencil loads map a
// padded index to its source interior index (transmissive clamp or periodic wrap), which is what
// copy_transmissive_boundary_kernel / copy_periodic_boundary_kernel (DEPLOY:371-408) write.
//
// Per SSPRK3 stage (the reference launches 8 kernels: BC copy, x/y normal, 2+2 Gauss flux, update;
// REFSYM:298-435) this path launches four:
//   k_normal<DIR=1>  characteristic WENO5 of every cell along x -> face values xl (lr=2), xr (lr=1)
//   k_normal<DIR=2>  the same along y -> yl, yr
//   k_flux_x         per x face: transverse WENO5 at both Gauss points from one closure evaluation per
//                    stencil, HLLC/FORCE at each point, fx = (f1 + f2) dt/dx
//   k_flux_y_update  per cell: the two y faces it owns are shared with neighbours, so y fluxes are
//                    computed per face in k_flux_y, and k_update forms the flux divergence, the SSPRK3
//                    combination and (after the last stage) the max wave speed for the next dt.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "closure.cuh"
#include "euler_math.cuh"

namespace wsr {

constexpr int kGhost = 3;

enum Bc { BC_TRANSMISSIVE = 0, BC_PERIODIC = 1 };
enum Flux { FLUX_HLLC = 0, FLUX_FORCE = 1 };

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

// Device-resident time-step control block (one per run).
struct StepCtl {
  double t;          // simulated time reached
  double t_end;
  double dt;         // dt of the step in flight
  double dt_dx, dt_dy;
  unsigned long long max_speed_bits;  // max wave speed of the current u0 (non-negative double bits)
  int steps;         // completed steps
  int done;          // loop finished (t reached, non-finite dt, or failed health check)
  int health_bad;    // NaN or p <= 0 seen by the last stage-3 update
  int fallbacks;     // stencils re-evaluated with JS weights
  int check_health;  // stop when the state is unhealthy after step 1 or every check_interval steps
  int check_interval;
  int max_steps;     // capacity of the dts record
  double cfl, hmin;
};

__device__ __forceinline__ int map_index(int p, int n, int bc) {
  if (bc == BC_TRANSMISSIVE) return p < kGhost ? kGhost : (p >= n + kGhost ? n + kGhost - 1 : p);
  return p < kGhost ? p + n : (p >= n + kGhost ? p - n : p);
}

__device__ __forceinline__ d4 load_cell(const double* __restrict__ u, int nxt, int j, int i) {
  const double2* p = reinterpret_cast<const double2*>(u + ((size_t)j * nxt + i) * 4);
  double2 a = __ldg(p), b = __ldg(p + 1);
  d4 q;
  q.v[0] = a.x;
  q.v[1] = a.y;
  q.v[2] = b.x;
  q.v[3] = b.y;
  return q;
}

__device__ __forceinline__ void store_cell(double* __restrict__ u, size_t idx, const d4& q) {
  double2* p = reinterpret_cast<double2*>(u + idx * 4);
  p[0] = make_double2(q.v[0], q.v[1]);
  p[1] = make_double2(q.v[2], q.v[3]);
}

template <int M>
__device__ __forceinline__ bool stencil_weights(const double q[5], const typename ClosureParams<M>::type& P,
                                                StencilW& s) {
  if constexpr (M == M_JS) {
    s = js_stencil(q);
    return true;
  } else {
    return sr_stencil<M>(q, P, s);
  }
}

// Reconstruct one stencil at `head`, falling back to JS weights if the closure is not finite and the
// fallback option is set.
template <int M>
__device__ __forceinline__ double recon_one(const double q[5], int head, const typename ClosureParams<M>::type& P,
                                            int opts, Tally& tally) {
  StencilW s;
  bool ok = stencil_weights<M>(q, P, s);
  if (M != M_JS) {
    tally.mlp += s.linear ? 0 : 1;
    tally.plateau += s.linear ? 1 : 0;
  }
  double w[3], c[3];
  if (!ok && (opts & OPT_JS_FALLBACK)) {
    StencilW js = js_stencil(q);
    js_head_weights(js, linear_weights(head), w);
    ++tally.fallbacks;
  } else {
    head_weights<M>(s, head, (opts & OPT_ENO_CUTOFF) != 0, w);
  }
  candidates(q, head, c);
  return combine(w, c);
}

__device__ __forceinline__ bool admissible(const d4& q, double g) {
  double rho = q.v[0];
  if (!(rho > 0.0)) return false;
  double u = q.v[1] / rho, v = q.v[2] / rho;
  double p = (g - 1.0) * (q.v[3] - 0.5 * rho * (u * u + v * v));
  return p > 0.0;
}

// -------------------------------------------------------------------------------------------
// Normal (characteristic) reconstruction.
// DIR=1: cell (r, c), r in [1, ny+5), c in [0, nx+2): stencil padded (r, c..c+4), output xl/xr[r][c]
//        of a [ny+6][nx+2] cell array.
// DIR=2: cell (r, c), r in [0, ny+2), c in [1, nx+5): stencil padded (r..r+4, c), output yl/yr[r][c]
//        of a [ny+2][nx+6] cell array.
// The left face (lr=2, head 1) uses Roe(q1, q2); the right face (lr=1, head 0) uses Roe(q2, q3).
// -------------------------------------------------------------------------------------------
template <int M, int DIR>
__global__ void __launch_bounds__(128) k_normal(const double* __restrict__ u, double* __restrict__ out_l,
                                                double* __restrict__ out_r, int nx, int ny, int bc, double g,
                                                const StepCtl* __restrict__ ctl, int opts, int* __restrict__ fallbacks,
                                                unsigned long long* __restrict__ counters,
                                                const __grid_constant__ typename ClosureParams<M>::type P) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  const int nxt = nx + 2 * kGhost;
  int r0, r1, c0, c1, ncols;
  if (DIR == 1) {
    r0 = 1; r1 = ny + 5; c0 = 0; c1 = nx + 2; ncols = nx + 2;
  } else {
    r0 = 0; r1 = ny + 2; c0 = 1; c1 = nx + 5; ncols = nx + 6;
  }
  if (r < r0 || r >= r1 || c < c0 || c >= c1) return;
  if (ctl != nullptr && ctl->done) return;
  Tally tally;
  d4 q[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    int pj = DIR == 1 ? r : r + k;
    int pi = DIR == 1 ? c + k : c;
    q[k] = load_cell(u, nxt, map_index(pj, ny, bc), map_index(pi, nx, bc));
  }
  const size_t oidx = (size_t)r * ncols + c;
#pragma unroll 1
  for (int side = 0; side < 2; ++side) {
    const int head = side == 0 ? 1 : 0;
    d4 qa, qb;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      qa.v[k] = side == 0 ? q[1].v[k] : q[2].v[k];
      qb.v[k] = side == 0 ? q[2].v[k] : q[3].v[k];
    }
    RoeJ J = roe_jacobian(qa, qb, g);
    CharL L = char_left<DIR>(J, g);
    // ch[f][k]: characteristic field f of stencil cell k. The field loop below stays rolled (one
    // inlined closure) and rotates the rows so that every register-array index is a constant.
    double ch[4][5];
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
      for (int k = 0; k < 5; ++k) ch[f][k] = project<DIR>(L, f, q[k]);
    double cf[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
      double v = recon_one<M>(ch[0], head, P, opts, tally);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        cf[a] = cf[a + 1];
#pragma unroll
        for (int k = 0; k < 5; ++k) ch[a][k] = ch[a + 1][k];
      }
      cf[3] = v;
    }
    d4 face = char_to_con<DIR>(cf, J);
    if constexpr (M != M_JS) {
      if ((opts & OPT_JS_FALLBACK) && !admissible(face, g)) {
        // positivity fallback: redo this face with JS weights
        double jf[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          double s[5];
#pragma unroll
          for (int k = 0; k < 5; ++k) s[k] = project<DIR>(L, f, q[k]);
          StencilW js = js_stencil(s);
          double w[3], cc[3];
          js_head_weights(js, linear_weights(head), w);
          candidates(s, head, cc);
          jf[f] = combine(w, cc);
        }
        face = char_to_con<DIR>(jf, J);
        ++tally.fallbacks;
      }
    }
    store_cell(side == 0 ? out_l : out_r, oidx, face);
  }
  flush_tally(tally, opts, fallbacks, counters);
}

// Transverse reconstruction of one conserved component at both Gauss points (heads 2 and 3) from a
// single closure evaluation.
template <int M>
__device__ __forceinline__ void gauss_pair(const double q[5], const typename ClosureParams<M>::type& P, int opts,
                                           Tally& tally, double& g1, double& g2) {
  StencilW s;
  bool ok = stencil_weights<M>(q, P, s);
  if (M != M_JS) {
    tally.mlp += s.linear ? 0 : 1;
    tally.plateau += s.linear ? 1 : 0;
  }
  double w[3], c[3];
  const bool fb = !ok && (opts & OPT_JS_FALLBACK);
  if (fb) {
    s = js_stencil(q);
    ++tally.fallbacks;
  }
#pragma unroll
  for (int h = 2; h <= 3; ++h) {
    if (fb)
      js_head_weights(s, linear_weights(h), w);
    else
      head_weights<M>(s, h, (opts & OPT_ENO_CUTOFF) != 0, w);
    candidates(q, h, c);
    (h == 2 ? g1 : g2) = combine(w, c);
  }
}

template <int DIR>
__device__ __forceinline__ d4 riemann(const d4& ul, const d4& ur, int flux, double dt_h, double g) {
  return flux == FLUX_FORCE ? force_flux<DIR>(ul, ur, dt_h, g) : hllc_flux<DIR>(ul, ur, g);
}

// x faces: face (j, i), j in [0, ny), i in [0, nx]: u_R from xl[j+1..j+5][i+1], u_L from xr[j+1..j+5][i]
// (REFSYM:127-195). Output fx[j][i] of a [ny][nx+1] face array: (F(g1) + F(g2)) dt/dx.
// y faces: face (j, i), j in [0, ny], i in [0, nx): u_R from yl[j+1][i+1..i+5], u_L from yr[j][i+1..i+5]
// (REFSYM:198-266). Output fy[j][i] of a [ny+1][nx] face array.
template <int M, int DIR>
__global__ void __launch_bounds__(128) k_flux(const double* __restrict__ fl, const double* __restrict__ fr,
                                              double* __restrict__ fout, int nx, int ny, double g, int flux,
                                              const StepCtl* __restrict__ ctl, int opts, int* __restrict__ fallbacks,
                                              unsigned long long* __restrict__ counters,
                                              const __grid_constant__ typename ClosureParams<M>::type P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nfx = DIR == 1 ? nx + 1 : nx, nfy = DIR == 1 ? ny : ny + 1;
  if (i >= nfx || j >= nfy) return;
  if (ctl->done) return;
  const double dt_h = DIR == 1 ? ctl->dt_dx : ctl->dt_dy;
  Tally tally;
  // Eight stencils per face: n = 2*comp + side, side 0 -> u_R (from the lr=2 faces fl), side 1 -> u_L.
  // Results rotate through g1/g2 so that indices stay constant inside the rolled loop.
  double g1[8], g2[8];
#pragma unroll 1
  for (int n = 0; n < 8; ++n) {
    const int comp = n >> 1, side = n & 1;
    const double* src = side == 0 ? fl : fr;
    double s[5];
    if (DIR == 1) {
      const int ncols = nx + 2, col = side == 0 ? i + 1 : i;
#pragma unroll
      for (int k = 0; k < 5; ++k) s[k] = __ldg(src + ((size_t)(j + 1 + k) * ncols + col) * 4 + comp);
    } else {
      const int ncols = nx + 6, row = side == 0 ? j + 1 : j;
#pragma unroll
      for (int k = 0; k < 5; ++k) s[k] = __ldg(src + ((size_t)row * ncols + (i + 1 + k)) * 4 + comp);
    }
    double a, b;
    gauss_pair<M>(s, P, opts, tally, a, b);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      g1[k] = g1[k + 1];
      g2[k] = g2[k + 1];
    }
    g1[7] = a;
    g2[7] = b;
  }
  d4 ur1, ul1, ur2, ul2;
#pragma unroll
  for (int comp = 0; comp < 4; ++comp) {
    ur1.v[comp] = g1[2 * comp];
    ul1.v[comp] = g1[2 * comp + 1];
    ur2.v[comp] = g2[2 * comp];
    ul2.v[comp] = g2[2 * comp + 1];
  }
  d4 f1 = riemann<DIR>(ul1, ur1, flux, dt_h, g);
  d4 f2 = riemann<DIR>(ul2, ur2, flux, dt_h, g);
  d4 o;
#pragma unroll
  for (int k = 0; k < 4; ++k) o.v[k] = f1.v[k] * dt_h + f2.v[k] * dt_h;
  store_cell(fout, (size_t)j * nfx + i, o);
  flush_tally(tally, opts, fallbacks, counters);
}

__device__ __forceinline__ unsigned long long speed_bits(const d4& q, double g) {
  double rho = fmax(q.v[0], 1.0e-15), vx = q.v[1] / rho, vy = q.v[2] / rho;
  double p = (g - 1.0) * (q.v[3] - 0.5 * rho * (vx * vx + vy * vy));
  p = fmax(p, 1.0e-15);
  double a = sqrt(g * p / rho);
  double s = fmax(fabs(vx) + a, fabs(vy) + a);
  // non-negative doubles (and NaN, whose bits sort above +inf) order like their bit patterns
  return (unsigned long long)__double_as_longlong(s);
}

// Block-wide max of non-negative double bit patterns, one atomic per block (blockDim.x <= 1024).
__device__ __forceinline__ void block_max_to(unsigned long long v, unsigned long long* dst) {
  __shared__ unsigned long long red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < nw ? red[lane] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
      v = w > v ? w : v;
    }
    if (lane == 0) atomicMax(dst, v);
  }
}

// SSPRK3 update of the interior (DEPLOY:1027-1056) and, on stage 3, the max wave speed of the new
// state plus the health flags that the reference reads back on the host.
__global__ void __launch_bounds__(256) k_update(const double* __restrict__ u_stage, const double* __restrict__ u0,
                                                double* __restrict__ u_out, const double* __restrict__ fx,
                                                const double* __restrict__ fy, int nx, int ny, int rk, double g,
                                                StepCtl* __restrict__ ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (ctl->done) return;
  const bool active = i < nx && j < ny;
  const int nxt = nx + 2 * kGhost;
  unsigned long long sb = 0;
  int bad = 0;
  if (active) {
    const int jj = j + kGhost, ii = i + kGhost;
    d4 us = load_cell(u_stage, nxt, jj, ii);
    d4 fxl = load_cell(fx, nx + 1, j, i), fxr = load_cell(fx, nx + 1, j, i + 1);
    d4 fyb = load_cell(fy, nx, j, i), fyt = load_cell(fy, nx, j + 1, i);
    d4 o;
    d4 z = rk == 1 ? us : load_cell(u0, nxt, jj, ii);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double rhs = us.v[k] - 0.5 * (fxr.v[k] - fxl.v[k]) - 0.5 * (fyt.v[k] - fyb.v[k]);
      if (rk == 1)
        o.v[k] = rhs;
      else if (rk == 2)
        o.v[k] = 0.75 * z.v[k] + 0.25 * rhs;
      else
        o.v[k] = (1.0 / 3.0) * z.v[k] + (2.0 / 3.0) * rhs;
    }
    store_cell(u_out, (size_t)jj * nxt + ii, o);
    if (rk == 3) {
      sb = speed_bits(o, g);
      double rho = fmax(o.v[0], 1.0e-15), vx = o.v[1] / rho, vy = o.v[2] / rho;
      double p = (g - 1.0) * (o.v[3] - 0.5 * rho * (vx * vx + vy * vy));
      bad = isnan(o.v[0]) || isnan(o.v[1]) || isnan(o.v[2]) || isnan(o.v[3]) || p <= 0.0;
    }
  }
  if (rk == 3) {
    block_max_to(sb, &ctl->max_speed_bits);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&ctl->health_bad, 1);
  }
}

__global__ void __launch_bounds__(256) k_max_speed(const double* __restrict__ u, int nx, int ny, double g,
                                                   unsigned long long* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  unsigned long long sb = 0;
  if (i < nx && j < ny) sb = speed_bits(load_cell(u, nx + 2 * kGhost, j + kGhost, i + kGhost), g);
  block_max_to(sb, out);
}

// dt for the next step (REFSYM:477-483, wh:189-207), on one thread. Also resets the max-speed slot
// that the coming stage-3 update accumulates into. `dts` records each step's dt.
__global__ void k_step_begin(StepCtl* ctl, double* dts) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ctl->done) return;
  if (ctl->check_health && ctl->health_bad &&
      (ctl->steps == 1 || (ctl->check_interval > 0 && ctl->steps % ctl->check_interval == 0))) {
    ctl->done = 1;
    return;
  }
  if (!(ctl->t < ctl->t_end - 1.0e-14) || ctl->steps >= ctl->max_steps) {
    ctl->done = 1;
    return;
  }
  double ms = __longlong_as_double((long long)ctl->max_speed_bits);
  double dt = ms < 1.0e-15 ? 1.0e10 : ctl->cfl * ctl->hmin / ms;
  double rem = ctl->t_end - ctl->t;
  dt = dt < rem ? dt : rem;
  if (!isfinite(dt) || dt <= 0.0) {
    ctl->done = 1;
    return;
  }
  ctl->dt = dt;
  ctl->max_speed_bits = 0ull;
  ctl->health_bad = 0;
  dts[ctl->steps] = dt;
}

__global__ void k_set_dt_ratios(StepCtl* ctl, double dx, double dy) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ctl->done) return;
  ctl->dt_dx = ctl->dt / dx;
  ctl->dt_dy = ctl->dt / dy;
}

__global__ void k_step_end(StepCtl* ctl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ctl->done) return;
  ctl->t = ctl->t + ctl->dt;
  ctl->steps += 1;
}

}  // namespace wsr
