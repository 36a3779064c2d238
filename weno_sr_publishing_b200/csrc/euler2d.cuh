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
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "closure.cuh"
#include "closure_mma.cuh"
#include "euler_math.cuh"

namespace wsr {

constexpr int kGhost = 3;

enum Bc { BC_TRANSMISSIVE = 0, BC_PERIODIC = 1, BC_DOUBLE_MACH = 2 };

// Boundary of one stage. The double-Mach boundary is time dependent: it is evaluated at
// ctl->t + t_off * ctl->dt (the SSPRK3 stages use t, t + dt and t + dt/2, REFSYM:462-527), on the cell
// centres ((i - 3 + 1/2) dx, (j - 3 + 1/2) dy) of the padded grid.
// y_ext: the y ghost rows of the stage state are stored in the array (filled from neighbouring slabs of a
// y-decomposed grid, or by the caller) and read as they are; x ghosts are still derived from `kind`.
struct StageBc {
  int kind;
  double dx, dy, t_off;
  int y_ext;
};
enum Flux { FLUX_HLLC = 0, FLUX_FORCE = 1 };

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

// Double-Mach reflection (REFSYM:26-124): a Mach-10 shock through (1/6, 0) at 60 degrees to the wall.
// Exact pre/post-shock state at (x, y) and time t, with round-to-nearest operations in the reference's order.
static __device__ __noinline__ d4 double_mach_state(double x, double y, double t, double g) {
  const double r3 = __dsqrt_rn(3.0);
  const double shock_x = __dadd_rn(__dadd_rn(1.0 / 6.0, __ddiv_rn(y, r3)), __ddiv_rn(__dmul_rn(20.0, t), r3));
  double rho = 1.4, u = 0.0, v = 0.0, p = 1.0;
  if (x < shock_x) {
    rho = 8.0;
    u = __dmul_rn(__dmul_rn(8.25, r3), 0.5);
    v = -4.125;
    p = 116.5;
  }
  const double e = __dadd_rn(__dmul_rn(__dmul_rn(0.5, rho), __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v))),
                             __ddiv_rn(p, __dsub_rn(g, 1.0)));
  return d4{{rho, __dmul_rn(rho, u), __dmul_rn(rho, v), e}};
}

// Value of the ghost cell at padded (pj, pi) under the double-Mach boundary: the exact state on the top rows
// (all columns), the left columns and the bottom rows left of x = 1/6 (there at y = 0); a reflection of the
// interior (v negated, column clamped to the interior) on the bottom rows right of it; a copy of the last
// interior column on the right.
static __device__ __noinline__ d4 double_mach_ghost(const double* __restrict__ u, int nx, int ny, int pj, int pi,
                                             const StageBc& bc, double t, double g) {
  const int nxt = nx + 2 * kGhost;
  const double x = __dmul_rn((double)(pi - kGhost) + 0.5, bc.dx);
  const double y = __dmul_rn((double)(pj - kGhost) + 0.5, bc.dy);
  if (pj >= ny + kGhost) return double_mach_state(x, y, t, g);
  if (pj < kGhost) {
    if (x < 1.0 / 6.0) return double_mach_state(x, 0.0, t, g);
    const int si = pi < kGhost ? kGhost : (pi >= nx + kGhost ? nx + kGhost - 1 : pi);
    d4 q = load_cell(u, nxt, 2 * kGhost - 1 - pj, si);
    q.v[2] = -q.v[2];
    return q;
  }
  if (pi < kGhost) return double_mach_state(x, y, t, g);
  return load_cell(u, nxt, pj, nx + kGhost - 1);
}

__device__ __forceinline__ bool admissible(const d4& q, double g) {  // rho > 0 and p > 0
  double rho = q.v[0];
  if (!(rho > 0.0)) return false;
  double u = q.v[1] / rho, v = q.v[2] / rho;
  double p = (g - 1.0) * (q.v[3] - 0.5 * rho * (u * u + v * v));
  return p > 0.0;
}

// -------------------------------------------------------------------------------------------
// Closure work is compacted per block. Phase A: every thread forms its 8 stencils and the cheap
// plateau sensors; plateau stencils take the linear weights at once; the others push their stencil id
// (n * 128 + thread) onto a block queue in shared memory. Phase B: the 128 threads take queue entries
// in turn and, for each, evaluate features, the MLP pair, the weights and the reconstructed value(s),
// so the closure runs at full SIMT width wherever the wave fronts fall. Per-thread stencil state
// lives in shared memory, which keeps every loop rolled (a small instruction footprint) and the
// register count low.
// -------------------------------------------------------------------------------------------
#ifndef WSR_MIN_BLOCKS
#define WSR_MIN_BLOCKS 6
#endif
constexpr int kBlock = 128;
constexpr int kStencilsPerThread = 8;
// Resident blocks per SM the register budget targets: the FP64 MLP needs more registers.
// The FP64 closure kernels at 4 blocks per SM (128 registers): 16.3 ms per 2000^2 SR-FP64 step against 17.7 at
// 3 blocks and 17.3 at 5.
#ifndef WSR_SR64_MIN_BLOCKS
#define WSR_SR64_MIN_BLOCKS 4
#endif
template <int M>
constexpr int min_blocks() { return M == M_SR64 ? WSR_SR64_MIN_BLOCKS : WSR_MIN_BLOCKS; }

// Thread tiling of a 128-thread block: kernels whose stencils run along y use 32 x 4 tiles so that the
// rows a block reads are shared in L1; kernels whose stencils run along x use 128 x 1.
// yb0 is the first block row of the launch (a launch may cover a band of the rows).
template <bool TALL>
struct Tile {
  static constexpr int bx = TALL ? 32 : kBlock, by = TALL ? 4 : 1;
  __device__ static int x(int t) { return blockIdx.x * bx + (TALL ? (t & 31) : t); }
  __device__ static int y(int t, int yb0) { return ((int)blockIdx.y + yb0) * by + (TALL ? (t >> 5) : 0); }
};

// Pushes the stencils of this warp that need the closure onto the block queue (warp-aggregated).
__device__ __forceinline__ void queue_push(bool need, int id, unsigned short* q, int* count) {
  const unsigned m = __ballot_sync(0xffffffffu, need);
  if (m == 0u) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == __ffs(m) - 1) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
  if (need) q[base + __popc(m & ((1u << lane) - 1u))] = (unsigned short)id;
}


// -------------------------------------------------------------------------------------------
// Normal (characteristic) reconstruction, one thread per face: the Roe average of the two cells
// next to the face and its eigenvectors serve both face values that use them -- the lr=1 value of
// the cell on the left (stencil cells 0..4 of the six) and the lr=2 value of the cell on the right
// (cells 1..5) -- so each Roe average and projection is computed once (the reference computes each
// twice, once from each cell; DEPLOY:479-592).
// DIR=1: face thread (r, c), r in [1, ny+5), c in [0, nx]: padded row r, columns c..c+5; writes
//        out_r[r][c] (lr=1 of the cell centred at column c+2) and out_l[r][c+1] (lr=2 of column c+3),
//        arrays [ny+6][nx+2].
// DIR=2: face thread (r, c), r in [0, ny], c in [1, nx+5): padded column c, rows r..r+5; writes
//        out_r[r][c] and out_l[r+1][c], arrays [ny+2][nx+6].
// Stencil n = 2 f + side of a face: characteristic field f; side 0 -> cells 0..4 with head 0 (lr=1),
// side 1 -> cells 1..5 with head 1 (lr=2).
// FACES < kBlock (small grids): the block's first FACES threads take one face each (a row of FACES faces) and all
// kBlock threads share its closure queue, so a thread evaluates at most 8 FACES / kBlock closures instead of up to
// 8 (on a small grid the one-face-per-thread launch is latency bound by that serial chain). The face arithmetic
// is the same code either way.
// -------------------------------------------------------------------------------------------


// Phase A of one characteristic stencil with its side (= head) a compile-time constant, as in the unrolled pairs of
// the one-face-per-thread loop: the value at once, or true when the stencil needs the closure.
template <int M, int DIR, int SIDE>
__device__ __forceinline__ bool normal_stencil_a(const double s[5], const typename ClosureParams<M>::type& P,
                                                 double& val, Tally& tally) {
  if constexpr (M == M_JS) {
    val = js_value(s, SIDE);
    return false;
  } else if constexpr (M == M_Z) {
    val = z_value(s, SIDE, DIR == 1 ? P.ex : P.ey);  // eps = h^2 of the normal direction
    return false;
  } else {
    const bool need = !plateau5(s);
    if (!need) val = linear_value(s, SIDE);
    ++(need ? tally.mlp : tally.plateau);
    return need;
  }
}

template <int M, int DIR, int FACES = kBlock>
__global__ void __launch_bounds__(kBlock, min_blocks<M>()) k_normal(const double* __restrict__ u, double* __restrict__ out_l,
                                                      double* __restrict__ out_r, int nx, int ny, StageBc bc, Gas gas,
                                                      const StepCtl* __restrict__ ctl, int opts,
                                                      int* __restrict__ fallbacks,
                                                      unsigned long long* __restrict__ counters,
                                                      const __grid_constant__ typename ClosureParams<M>::type P,
                                                      int yb0) {
  __shared__ double s_ch[4][6][FACES];                  // characteristic values, [field][cell][face thread]
  __shared__ double s_val[kStencilsPerThread][FACES];   // reconstructed characteristic face values
  __shared__ unsigned short s_q[kStencilsPerThread * FACES];
  __shared__ int s_count;
  if (ctl != nullptr && ctl->done) return;  // uniform across the launch
  using TL = Tile<DIR == 2>;
  const int t = threadIdx.x;
  constexpr bool kAll = FACES == kBlock;
  const bool face_thread = kAll || t < FACES;
  const int c = kAll ? TL::x(t) : (int)blockIdx.x * FACES + t;
  const int r = kAll ? TL::y(t, yb0) : (int)blockIdx.y + yb0;
  const int nxt = nx + 2 * kGhost;
  const bool active =
      face_thread && (DIR == 1 ? (r >= 1 && r < ny + 5 && c <= nx) : (r <= ny && c >= 1 && c < nx + 5));
  if (t == 0) s_count = 0;
  Tally tally;
  RoeJ J;
  {
    // cells are loaded one at a time for the projection (L1 hits after the first touch), which keeps
    // the six-cell stencil out of the register budget
    const double bt = bc.kind == BC_DOUBLE_MACH ? ctl->t + bc.t_off * ctl->dt : 0.0;
    auto cell = [&](int k) {
      if (!active) return d4{{1.0, 0.0, 0.0, 2.5}};  // inert filler for threads past the edge
      const int pj = DIR == 1 ? r : r + k;
      const int pi = DIR == 1 ? c + k : c;
      if (bc.kind == BC_DOUBLE_MACH && (pj < kGhost || pj >= ny + kGhost || pi < kGhost || pi >= nx + kGhost))
        return double_mach_ghost(u, nx, ny, pj, pi, bc, bt, gas.g);
      return load_cell(u, nxt, bc.y_ext ? pj : map_index(pj, ny, bc.kind), map_index(pi, nx, bc.kind));
    };
    J = roe_jacobian(cell(2), cell(3), gas);
    const CharL L = char_left<DIR>(J, gas);
    if (face_thread) {
#pragma unroll 1
      for (int k = 0; k < 6; ++k) {
        const d4 qk = cell(k);
#pragma unroll
        for (int f = 0; f < 4; ++f) s_ch[f][k][t] = project<DIR>(L, f, qk);
      }
    }
  }
  const bool work = active;
  __syncthreads();
  if constexpr (!kAll) {
    // Phase A of the small-grid form: the kLanes lanes of face t / kLanes take its 8 stencils in turn (lane l:
    // stencils l, l + kLanes, ...; kLanes is even, so a lane keeps one side)
    constexpr int kLanes = kBlock / FACES;
    static_assert(kLanes % 2 == 0 && kStencilsPerThread % kLanes == 0, "lanes per face must be 2, 4 or 8");
    const int face = t / kLanes, lane = t % kLanes, side = lane & 1;
    const int fc = (int)blockIdx.x * FACES + face;
    const bool live = DIR == 1 ? (r >= 1 && r < ny + 5 && fc <= nx) : (r <= ny && fc >= 1 && fc < nx + 5);
#pragma unroll 1
    for (int n = lane; n < kStencilsPerThread; n += kLanes) {
      const int f = n >> 1;
      bool need = false;
      if (live) {
        double s[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) s[k] = s_ch[f][k + side][face];
        double v = 0.0;
        if (side == 0)
          need = normal_stencil_a<M, DIR, 0>(s, P, v, tally);
        else
          need = normal_stencil_a<M, DIR, 1>(s, P, v, tally);
        if (!need) s_val[n][face] = v;
      }
      if constexpr (has_mlp<M>()) queue_push(need, n * FACES + face, s_q, &s_count);
    }
  }
  // Phase A, two stencils per iteration (two independent dependency chains; unrolling by 4 or 8 spills)
#pragma unroll 2
  for (int n = 0; n < kStencilsPerThread; ++n) {
    if (!kAll) break;
    const int f = n >> 1, side = n & 1;
    bool need = false;
    if (work) {
      double s[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) s[k] = s_ch[f][k + side][t];
      if constexpr (M == M_JS) {
        s_val[n][t] = js_value(s, side);
      } else if constexpr (M == M_Z) {
        s_val[n][t] = z_value(s, side, DIR == 1 ? P.ex : P.ey);  // eps = h^2 of the normal direction
      } else {
        need = !plateau5(s);
        if (!need) s_val[n][t] = linear_value(s, side);
        ++(need ? tally.mlp : tally.plateau);
      }
    }
    if constexpr (has_mlp<M>()) queue_push(need, n * FACES + t, s_q, &s_count);
  }
  // Phase B
  if constexpr (M == M_SRBF16_TC && kAll) {
    // BF16 closure on the tensor cores: each warp takes 32 queue entries at a time (closure_mma.cuh)
    __syncthreads();
    const int count = s_count;
    if (count > 0) {
      const MmaW5 W = mma_weights(P.p, t & 31);
#pragma unroll 1
      for (int base = t & ~31; base < count; base += kBlock) {  // the same bound for every lane of a warp
        const int e = base + (t & 31);
        const bool valid = e < count;
        int n = 0, o = 0;
        double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        float x[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (valid) {
          const int id = s_q[e];
          n = id / kBlock;
          o = id % kBlock;
#pragma unroll
          for (int k = 0; k < 5; ++k) s[k] = s_ch[n >> 1][k + (n & 1)][o];
          sr_features32<M>(s, sensors5(s), x);
        }
        double a0, a1, a2;
        closure_bf16_mma(W, x, a0, a1, a2);
        if (valid) s_val[n][o] = sr_value<M>(s, n & 1, a0, a1, a2, opts, tally);
      }
    }
  } else if constexpr (has_mlp<M>()) {
    __syncthreads();
    const int count = s_count;
#pragma unroll 1
    for (int e = t; e < count; e += kBlock) {
      const int id = s_q[e];
      const int n = id / FACES, o = id % FACES, f = n >> 1, side = n & 1;
      double s[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) s[k] = s_ch[f][k + side][o];
      double a0, a1, a2;
      sr_betas<M>(s, P, a0, a1, a2);
      s_val[n][o] = sr_value<M>(s, side, a0, a1, a2, opts, tally);
    }
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      double cf[4] = {s_val[side][t], s_val[2 + side][t], s_val[4 + side][t], s_val[6 + side][t]};
      d4 face = char_to_con<DIR>(cf, J);
      if constexpr (has_mlp<M>()) {
        if ((opts & OPT_JS_FALLBACK) && !admissible(face, gas.g)) {
          // positivity fallback: redo this face value with JS weights
          double jf[4];
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            double s[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) s[k] = s_ch[f][k + side][t];
            jf[f] = js_value(s, side);
          }
          face = char_to_con<DIR>(jf, J);
          ++tally.fallbacks;
        }
      }
      size_t idx;
      if (DIR == 1)
        idx = (size_t)r * (nx + 2) + c + side;
      else
        idx = (size_t)(r + side) * (nx + 6) + c;
      store_cell(side == 0 ? out_r : out_l, idx, face);
    }
  }
  flush_tally(tally, opts, fallbacks, counters);
}

template <int DIR>
__device__ __forceinline__ d4 riemann(const d4& ul, const d4& ur, int flux, double dt_h, const Gas& gas) {
  return flux == FLUX_FORCE ? force_flux<DIR>(ul, ur, dt_h, gas.g) : hllc_flux<DIR>(ul, ur, gas);
}

// Transverse reconstruction and flux, one thread per face.
// x faces: face (j, i), j in [0, ny), i in [0, nx]: u_R from xl[j+1..j+5][i+1], u_L from xr[j+1..j+5][i]
// (REFSYM:127-195). Output fx[j][i] of a [ny][nx+1] face array: (F(g1) + F(g2)) dt/dx.
// y faces: face (j, i), j in [0, ny], i in [0, nx): u_R from yl[j+1][i+1..i+5], u_L from yr[j][i+1..i+5]
// (REFSYM:198-266). Output fy[j][i] of a [ny+1][nx] face array.
// Each of the 8 stencils (4 components x 2 sides) evaluates its closure once for both Gauss points.
// Stencil tiles of the transverse kernels, staged into shared memory by TMA (cp.async.bulk.tensor). A face-value
// array [rows][cols][4] FP64 is the 4D tensor {2 values, 2 pairs, cols, rows} (byte strides 16, 32, 32 cols), so a
// box holds one pair of components with a 16-byte inner extent and an x coordinate of 0 (every copy starts on a
// 16-byte boundary). Per block: x faces (32 x 4) read rows j0+1 .. j0+8 and columns i0 .. i0+32 of xl and xr;
// y faces (128 x 1) read row j+1 of yl and row j of yr, columns i0+1 .. i0+132. Boxes past the array's end are
// filled with zeros by the copy (those values belong to inactive faces).
template <int DIR>
struct FluxTile {
  static constexpr int cols = DIR == 1 ? 33 : 132, rows = DIR == 1 ? 8 : 1;
  static constexpr int box_doubles = 2 * cols * rows;
  static constexpr int stride = (box_doubles + 15) / 16 * 16;  // 128-byte aligned boxes
  static constexpr unsigned box_bytes = box_doubles * sizeof(double);
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tma_load_box(double* dst, const CUtensorMap* map, int pair, int col, int row,
                                             unsigned long long* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(0), "r"(pair), "r"(col), "r"(row), "r"(smem_u32(mbar))
      : "memory");
}

// Issues the block's four boxes (thread 0) and waits for them (every thread), at most about 2^22 polls; false
// when the copies did not complete in time.
template <int DIR>
__device__ __forceinline__ bool load_flux_tile(double* tile, unsigned long long* mbar, const CUtensorMap* map_l,
                                               const CUtensorMap* map_r, int i0, int j0) {
  using FT = FluxTile<DIR>;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)),
                 "r"(4u * FT::box_bytes)
                 : "memory");
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int side = b >> 1, pair = b & 1;
      const int col = DIR == 1 ? i0 : i0 + 1;
      const int row = DIR == 1 ? j0 + 1 : (side == 0 ? j0 + 1 : j0);
      tma_load_box(tile + b * FT::stride, side == 0 ? map_l : map_r, pair, col, row, mbar);
    }
  }
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(mbar))
        : "memory");
    if (done) return true;
  }
  return false;
}

// After a timed-out wait: wait once more (bounded) so that no copy is still writing the block's shared memory
// when it exits.
__device__ __forceinline__ void load_flux_tile_wait_again(unsigned long long* mbar) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(mbar))
        : "memory");
    if (done) return;
  }
}

// Stencil n = 2 comp + side of face (i, j) from the block's tile (i0, j0: the block's first face).
template <int DIR>
__device__ __forceinline__ void tile_transverse(const double* tile, int i, int j, int i0, int j0, int n, bool active,
                                                double s[5]) {
  using FT = FluxTile<DIR>;
  const int comp = n >> 1, side = n & 1;
  if (!active) {
#pragma unroll
    for (int k = 0; k < 5; ++k) s[k] = 0.0;
    return;
  }
  const double* box = tile + (side * 2 + (comp >> 1)) * FT::stride + (comp & 1);
  if (DIR == 1) {
    const int cc = side == 0 ? i - i0 + 1 : i - i0;
#pragma unroll
    for (int k = 0; k < 5; ++k) s[k] = box[((j - j0 + k) * FT::cols + cc) * 2];
  } else {
#pragma unroll
    for (int k = 0; k < 5; ++k) s[k] = box[(i - i0 + k) * 2];
  }
}

// Stencil n = 2 comp + side of face (i, j) read from the face-value arrays themselves (the small-grid form of
// k_flux, which stages no tile): the same values as tile_transverse.
template <int DIR>
__device__ __forceinline__ void global_transverse(const double* __restrict__ fl, const double* __restrict__ fr, int nx,
                                                  int i, int j, int n, bool active, double s[5]) {
  const int comp = n >> 1, side = n & 1;
  if (!active) {
#pragma unroll
    for (int k = 0; k < 5; ++k) s[k] = 0.0;
    return;
  }
  const double* src = side == 0 ? fl : fr;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const size_t cell = DIR == 1 ? (size_t)(j + 1 + k) * (nx + 2) + (side == 0 ? i + 1 : i)
                                 : (size_t)(side == 0 ? j + 1 : j) * (nx + 6) + i + 1 + k;
    s[k] = src[cell * 4 + comp];
  }
}

// Phase A of one transverse stencil: its values at the two Gauss points at once, or true when it needs the closure.
template <int M, int DIR>
__device__ __forceinline__ bool flux_stencil_a(const double s[5], const typename ClosureParams<M>::type& P, double& g0,
                                               double& g1, Tally& tally) {
  if constexpr (M == M_JS) {
    const StencilW js = js_stencil(s);
    double w[3], c[3];
    js_head_weights(js, linear_weights(2), w);
    candidates(s, 2, c);
    g0 = combine(w, c);
    js_head_weights(js, linear_weights(3), w);
    candidates(s, 3, c);
    g1 = combine(w, c);
    return false;
  } else if constexpr (M == M_Z) {
    const StencilW z = z_stencil(s, DIR == 1 ? P.ey : P.ex);  // eps = h^2 of the transverse direction
    g0 = z_value_w(z, s, 2);
    g1 = z_value_w(z, s, 3);
    return false;
  } else {
    const bool need = !plateau5(s);
    if (!need) {
      g0 = linear_value(s, 2);
      g1 = linear_value(s, 3);
    }
    ++(need ? tally.mlp : tally.plateau);
    return need;
  }
}

// FACES < kBlock: the small-grid form, as in k_normal (the block's first FACES threads take one face each, all
// kBlock threads share the closure queue); its stencils come from the face-value arrays directly.
template <int M, int DIR, int FACES = kBlock>
__global__ void __launch_bounds__(kBlock, min_blocks<M>()) k_flux(const double* __restrict__ fl, const double* __restrict__ fr,
                                                    double* __restrict__ fout, int nx, int ny, Gas gas, int flux,
                                                    const StepCtl* __restrict__ ctl, int opts,
                                                    int* __restrict__ fallbacks,
                                                    unsigned long long* __restrict__ counters,
                                                    const __grid_constant__ typename ClosureParams<M>::type P,
                                                    const __grid_constant__ CUtensorMap map_l,
                                                    const __grid_constant__ CUtensorMap map_r, int yb0) {
  constexpr bool kAll = FACES == kBlock;
  __shared__ double s_g[2][kStencilsPerThread][FACES];  // values at Gauss points 1 and 2
  __shared__ unsigned short s_q[kStencilsPerThread * FACES];
  __shared__ __align__(128) double s_tile[kAll ? 4 * FluxTile<DIR>::stride : 2];
  __shared__ unsigned long long s_mbar;
  __shared__ int s_count;
  if (ctl->done) return;  // uniform across the launch
  using TL = Tile<DIR == 1>;
  const int t = threadIdx.x;
  const bool face_thread = kAll || t < FACES;
  const int i = kAll ? TL::x(t) : (int)blockIdx.x * FACES + t;
  const int j = kAll ? TL::y(t, yb0) : (int)blockIdx.y + yb0;
  const int i0 = blockIdx.x * TL::bx, j0 = ((int)blockIdx.y + yb0) * TL::by;
  const int nfx = DIR == 1 ? nx + 1 : nx, nfy = DIR == 1 ? ny : ny + 1;
  const bool active = face_thread && i < nfx && j < nfy;
  const double dt_h = DIR == 1 ? ctl->dt_dx : ctl->dt_dy;
  if (t == 0) s_count = 0;
  if constexpr (kAll) {
    const bool tile_ok = load_flux_tile<DIR>(s_tile, &s_mbar, &map_l, &map_r, i0, j0);
    if (__syncthreads_or(!tile_ok)) {  // the same decision in every thread of the block
      if (t == 0) atomicExch(&fallbacks[1], 1);
      if (!tile_ok) load_flux_tile_wait_again(&s_mbar);
      return;
    }
  } else {
    __syncthreads();
  }
  Tally tally;
  const bool work = active;
  // Phase A of the small-grid form: lane n of the 8 lanes of face t / 8 takes stencil n
  if constexpr (!kAll) {
    // the kLanes lanes of face t / kLanes take its 8 stencils in turn
    constexpr int kLanes = kBlock / FACES;
    static_assert(kStencilsPerThread % kLanes == 0, "lanes per face must divide 8");
    const int face = t / kLanes, lane = t % kLanes;
    const int fi = (int)blockIdx.x * FACES + face;
    const bool live = fi < nfx && j < nfy;
#pragma unroll 1
    for (int n = lane; n < kStencilsPerThread; n += kLanes) {
      double s[5];
      global_transverse<DIR>(fl, fr, nx, fi, j, n, live, s);
      double g0 = 0.0, g1 = 0.0;
      const bool need = live && flux_stencil_a<M, DIR>(s, P, g0, g1, tally);
      if (live && !need) {
        s_g[0][n][face] = g0;
        s_g[1][n][face] = g1;
      }
      if constexpr (has_mlp<M>()) queue_push(need, n * FACES + face, s_q, &s_count);
    }
  }
  // Phase A, two stencils per iteration. Stencil n = 2 comp + side: side 0 -> u_R (lr=2 faces fl), side 1 -> u_L
  // (lr=1 faces fr).
#pragma unroll 2
  for (int n = 0; n < kStencilsPerThread; ++n) {
    if (!kAll) break;
    double s[5];
    tile_transverse<DIR>(s_tile, i, j, i0, j0, n, work, s);
    bool need = false;
    // the body of flux_stencil_a written out (measured 0.7% faster at 2000^2 than the call, same results)
    if (!work) {
      // nothing to reconstruct
    } else if constexpr (M == M_JS) {
      const StencilW js = js_stencil(s);
      double w[3], c[3];
      js_head_weights(js, linear_weights(2), w);
      candidates(s, 2, c);
      s_g[0][n][t] = combine(w, c);
      js_head_weights(js, linear_weights(3), w);
      candidates(s, 3, c);
      s_g[1][n][t] = combine(w, c);
    } else if constexpr (M == M_Z) {
      const StencilW z = z_stencil(s, DIR == 1 ? P.ey : P.ex);  // eps = h^2 of the transverse direction
      s_g[0][n][t] = z_value_w(z, s, 2);
      s_g[1][n][t] = z_value_w(z, s, 3);
    } else {
      need = !plateau5(s);
      if (!need) {
        s_g[0][n][t] = linear_value(s, 2);
        s_g[1][n][t] = linear_value(s, 3);
      }
      ++(need ? tally.mlp : tally.plateau);
    }
    if constexpr (has_mlp<M>()) queue_push(need, n * FACES + t, s_q, &s_count);
  }
  // Phase B: one closure evaluation per queued stencil serves both Gauss points.
  if constexpr (M == M_SRBF16_TC && kAll) {
    // BF16 closure on the tensor cores: each warp takes 32 queue entries at a time (closure_mma.cuh)
    __syncthreads();
    const int count = s_count;
    if (count > 0) {
      const MmaW5 W = mma_weights(P.p, t & 31);
#pragma unroll 1
      for (int base = t & ~31; base < count; base += kBlock) {  // the same bound for every lane of a warp
        const int e = base + (t & 31);
        const bool valid = e < count;
        int n = 0, o = 0;
        double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        float x[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (valid) {
          const int id = s_q[e];
          n = id / kBlock;
          o = id % kBlock;
          tile_transverse<DIR>(s_tile, TL::x(o), TL::y(o, yb0), i0, j0, n, true, s);
          sr_features32<M>(s, sensors5(s), x);
        }
        double a0, a1, a2;
        closure_bf16_mma(W, x, a0, a1, a2);
        if (valid) {
          s_g[0][n][o] = sr_value<M>(s, 2, a0, a1, a2, opts, tally);
          s_g[1][n][o] = sr_value<M>(s, 3, a0, a1, a2, opts, tally);
        }
      }
    }
  } else if constexpr (has_mlp<M>()) {
    __syncthreads();
    const int count = s_count;
#pragma unroll 1
    for (int e = t; e < count; e += kBlock) {
      const int id = s_q[e];
      const int n = id / FACES, o = id % FACES;
      double s[5];
      if constexpr (kAll)
        tile_transverse<DIR>(s_tile, TL::x(o), TL::y(o, yb0), i0, j0, n, true, s);
      else
        global_transverse<DIR>(fl, fr, nx, (int)blockIdx.x * FACES + o, (int)blockIdx.y + yb0, n, true, s);
      double a0, a1, a2;
      sr_betas<M>(s, P, a0, a1, a2);
      s_g[0][n][o] = sr_value<M>(s, 2, a0, a1, a2, opts, tally);
      s_g[1][n][o] = sr_value<M>(s, 3, a0, a1, a2, opts, tally);
    }
  }
  __syncthreads();
  if (active) {
    d4 ur1, ul1, ur2, ul2;
#pragma unroll
    for (int comp = 0; comp < 4; ++comp) {
      ur1.v[comp] = s_g[0][2 * comp][t];
      ul1.v[comp] = s_g[0][2 * comp + 1][t];
      ur2.v[comp] = s_g[1][2 * comp][t];
      ul2.v[comp] = s_g[1][2 * comp + 1][t];
    }
    const d4 f1 = riemann<DIR>(ul1, ur1, flux, dt_h, gas);
    const d4 f2 = riemann<DIR>(ul2, ur2, flux, dt_h, gas);
    d4 o;
#pragma unroll
    for (int k = 0; k < 4; ++k) o.v[k] = f1.v[k] * dt_h + f2.v[k] * dt_h;
    store_cell(fout, (size_t)j * nfx + i, o);
  }
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
static __global__ void __launch_bounds__(256) k_update(const double* __restrict__ u_stage, const double* __restrict__ u0,
                                                double* __restrict__ u_out, const double* __restrict__ fx,
                                                const double* __restrict__ fy, int nx, int ny, int rk, double g,
                                                StepCtl* __restrict__ ctl, int yb0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y + yb0;
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

static __global__ void __launch_bounds__(256) k_max_speed(const double* __restrict__ u, int nx, int ny, double g,
                                                   unsigned long long* __restrict__ out, int yb0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y + yb0;
  unsigned long long sb = 0;
  if (i < nx && j < ny) sb = speed_bits(load_cell(u, nx + 2 * kGhost, j + kGhost, i + kGhost), g);
  block_max_to(sb, out);
}

// dt for the next step (REFSYM:477-483, wh:189-207), on one thread. Also resets the max-speed slot
// that the coming stage-3 update accumulates into. `dts` records each step's dt.
static __global__ void k_step_begin(StepCtl* ctl, double* dts) {
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

static __global__ void k_set_dt_ratios(StepCtl* ctl, double dx, double dy) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ctl->done) return;
  ctl->dt_dx = ctl->dt / dx;
  ctl->dt_dy = ctl->dt / dy;
}

static __global__ void k_step_end(StepCtl* ctl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ctl->done) return;
  ctl->t = ctl->t + ctl->dt;
  ctl->steps += 1;
}

}  // namespace wsr
