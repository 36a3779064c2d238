// extern "C" entry points of libwsr.so for the 2D WENO5 path, the throughput probes and the no-allocation
// stage (declared in include/wsr.h); the 1D/training and WENO7 entry points are in wsr_api_1d.cu and wsr_api_w7.cu.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include <cuda.h>

#include "../../include/wsr.h"
#include "euler2d.cuh"
#include "wsr_ctx.cuh"

using namespace wsr;
using namespace wsr_detail;

namespace {

struct Ws2d {
  StepCtl* ctl;
  int* fallbacks;
  unsigned long long* counters;  // per kernel class k (normal x, normal y, flux x, flux y): [2k] MLP closure
                                 // evaluations, [2k+1] plateau stencils
  double* dts;  // ring of kDtsRing
  double *xl, *xr, *yl, *yr, *fx, *fy;
};

size_t ws_bytes(int nx, int ny) {
  size_t b = align_up(sizeof(StepCtl)) + align_up(sizeof(int)) + align_up(8 * sizeof(unsigned long long)) +
             align_up(kDtsRing * sizeof(double));
  b += 2 * cells_bytes((size_t)(ny + 6) * (nx + 2));
  b += 2 * cells_bytes((size_t)(ny + 2) * (nx + 6));
  b += cells_bytes((size_t)ny * (nx + 1));
  b += cells_bytes((size_t)(ny + 1) * nx);
  return b;
}

Ws2d carve(void* base, int nx, int ny) {
  char* p = static_cast<char*>(base);
  Ws2d w;
  w.ctl = reinterpret_cast<StepCtl*>(p);
  p += align_up(sizeof(StepCtl));
  w.fallbacks = reinterpret_cast<int*>(p);
  p += align_up(sizeof(int));
  w.counters = reinterpret_cast<unsigned long long*>(p);
  p += align_up(8 * sizeof(unsigned long long));
  w.dts = reinterpret_cast<double*>(p);
  p += align_up(kDtsRing * sizeof(double));
  w.xl = reinterpret_cast<double*>(p);
  p += cells_bytes((size_t)(ny + 6) * (nx + 2));
  w.xr = reinterpret_cast<double*>(p);
  p += cells_bytes((size_t)(ny + 6) * (nx + 2));
  w.yl = reinterpret_cast<double*>(p);
  p += cells_bytes((size_t)(ny + 2) * (nx + 6));
  w.yr = reinterpret_cast<double*>(p);
  p += cells_bytes((size_t)(ny + 2) * (nx + 6));
  w.fx = reinterpret_cast<double*>(p);
  p += cells_bytes((size_t)ny * (nx + 1));
  w.fy = reinterpret_cast<double*>(p);
  return w;
}

// Tensor maps of the four face-value arrays for the TMA tile loads of k_flux (euler2d.cuh FluxTile): each array
// [rows][cols][4] FP64 as the 4D tensor {2, 2, cols, rows}; boxes {2, 1, 33, 8} (x faces) and {2, 1, 132, 1}
// (y faces). cuTensorMapEncodeTiled comes through the runtime's driver entry point (no link to libcuda).
struct FaceMaps {
  CUtensorMap xl, xr, yl, yr;
};

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

bool face_map(CUtensorMap* m, double* base, int cols, int rows, int box_cols, int box_rows) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[4] = {2, 2, (cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[3] = {16, 32, (cuuint64_t)cols * 32};
  const cuuint32_t box[4] = {2, 1, (cuuint32_t)box_cols, (cuuint32_t)box_rows};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

bool face_maps(const Ws2d& w, int nx, int ny, FaceMaps* fm) {
  return face_map(&fm->xl, w.xl, nx + 2, ny + 6, FluxTile<1>::cols, FluxTile<1>::rows) &&
         face_map(&fm->xr, w.xr, nx + 2, ny + 6, FluxTile<1>::cols, FluxTile<1>::rows) &&
         face_map(&fm->yl, w.yl, nx + 6, ny + 2, FluxTile<2>::cols, FluxTile<2>::rows) &&
         face_map(&fm->yr, w.yr, nx + 6, ny + 2, FluxTile<2>::cols, FluxTile<2>::rows);
}

int check_2d(wsr_ctx* ctx, int nx, int ny, int method, int bc, int flux, void* ws, size_t wsb) {
  if (!ctx) return WSR_ERR_ARG;
  if (nx < 3 || ny < 3) return fail(ctx, WSR_ERR_ARG, "nx and ny must be >= 3 (got %d, %d)", nx, ny);
  if ((long long)(nx + 6) * (ny + 6) > (1ll << 31) / 4)
    return fail(ctx, WSR_ERR_ARG, "grid %d x %d too large for one launch", nx, ny);
  if (method < WSR_METHOD_JS || method > WSR_METHOD_SR_BF16_TC) return fail(ctx, WSR_ERR_ARG, "bad method %d", method);
  const int base = bc & ~WSR_BC_Y_HALO;
  if (base != WSR_BC_TRANSMISSIVE && base != WSR_BC_PERIODIC && base != WSR_BC_DOUBLE_MACH)
    return fail(ctx, WSR_ERR_ARG, "bad boundary %d", bc);
  if ((bc & WSR_BC_Y_HALO) && base == WSR_BC_DOUBLE_MACH)
    return fail(ctx, WSR_ERR_ARG, "WSR_BC_Y_HALO combines with WSR_BC_TRANSMISSIVE or WSR_BC_PERIODIC only");
  if (flux != WSR_FLUX_HLLC && flux != WSR_FLUX_FORCE) return fail(ctx, WSR_ERR_ARG, "bad flux %d", flux);
  if (method != WSR_METHOD_JS && method != WSR_METHOD_Z && !ctx->have_closure)
    return fail(ctx, WSR_ERR_NO_CLOSURE, "SR method requested before wsr_closure_upload");
  if (!ws) return fail(ctx, WSR_ERR_ARG, "workspace is NULL");
  if (reinterpret_cast<uintptr_t>(ws) % kAlign) return fail(ctx, WSR_ERR_ARG, "workspace must be 256-byte aligned");
  if (wsb < ws_bytes(nx, ny))
    return fail(ctx, WSR_ERR_ARG, "workspace too small: %zu < %zu bytes", wsb, ws_bytes(nx, ny));
  return WSR_OK;
}

int prof_flush(wsr_ctx* ctx) {
  if (ctx->n_ev == 0) return WSR_OK;
  WSR_CUDA(ctx, cudaEventSynchronize(ctx->ev_b[ctx->n_ev - 1]));
  for (int k = 0; k < ctx->n_ev; ++k) {
    float ms = 0.f;
    WSR_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev_a[k], ctx->ev_b[k]));
    ctx->prof_ms[ctx->ev_kind[k]] += ms;
    ctx->prof_count[ctx->ev_kind[k]] += 1;
  }
  ctx->n_ev = 0;
  return WSR_OK;
}

// Brackets one launch with events when profiling is on.
struct ProfScope {
  wsr_ctx* ctx;
  cudaStream_t st;
  int slot;
  ProfScope(wsr_ctx* c, cudaStream_t s, int kind) : ctx(c), st(s), slot(-1) {
    if (!ctx->prof_on) return;
    if (ctx->n_ev == kProfEvents && prof_flush(ctx) != WSR_OK) return;
    slot = ctx->n_ev++;
    ctx->ev_kind[slot] = kind;
    cudaEventRecord(ctx->ev_a[slot], st);
  }
  ~ProfScope() {
    if (slot >= 0) cudaEventRecord(ctx->ev_b[slot], st);
  }
};

struct StageArgs {
  const double* u_stage;
  const double* u0;
  double* u_out;
  int nx, ny, bc, flux, opts, rk;
  double dx, dy, g;
  double t_off;  // boundary time of the stage = ctl->t + t_off * ctl->dt
};

// One stage = 5 launches. dt/dx and dt/dy are read from ws.ctl on the device.
inline StageBc stage_bc(const StageArgs& a) {
  return StageBc{a.bc & ~WSR_BC_Y_HALO, a.dx, a.dy, a.t_off, (a.bc & WSR_BC_Y_HALO) ? 1 : 0};
}

// Kernel parameters of a method: the uploaded closure, or for WENO-Z the per-direction eps = h^2.
template <int M>
typename ClosureParams<M>::type stage_params(const wsr_ctx* ctx, const StageArgs& a) {
  if constexpr (M == M_Z)
    return ZEps{a.dx * a.dx, a.dy * a.dy};
  else
    return params_of<M>(ctx);
}

// ---- the five launches of a stage, whole or in row bands ---------------------------------------------------
// Two forms of the reconstruction kernels: 128 faces per block (one per thread), and on small grids 16 faces per
// block whose closure queue all 128 threads share (the FACES template argument of k_normal and k_flux).
// Faces per block of the small-grid forms by grid size (SR methods). Measured per step, seeded quadrant state, one
// thread per face / 16 / 32 / 64 faces per block, SR-FP32 (SR-FP64) in us: 100^2 227 / 149 / 159 / 193 (717 / 270 /
// 326 / 488); 200^2 288 / 259 / 235 / 304 (774 / 616 / 625 / 693); 300^2 359 / 431 / 359 / 365 (1028 / 1069 / 990 /
// 969); 400^2 527 / 643 / 495 / 482 (1422 / 1617 / 1472 / 1433).
constexpr long long kSmall16Cells = 128LL * 128;
constexpr long long kSmall32Cells = 256LL * 256;

// 0 for the one-face-per-thread form, else the faces per block of the small-grid form.
template <int M>
int small_faces(const StageArgs& a) {
  if constexpr (M == M_SRBF16_TC || !has_mlp<M>()) {
    // The tensor-core closure works on whole warps of queued stencils. JS and WENO-Z have no closure queue, so the
    // small forms gain them little, and their candidate arithmetic, once the side is not a compile-time constant,
    // compiles to differently rounded multiply-adds: one face per thread only.
    return 0;
  } else {
    if (a.opts & WSR_OPT_FACE_THREADS_1) return 0;
    if (a.opts & WSR_OPT_FACE_THREADS_8) return 16;
    if (a.opts & WSR_OPT_FACE_THREADS_4) return 32;
    const long long cells = (long long)a.nx * a.ny;
    return cells <= kSmall16Cells ? 16 : (cells <= kSmall32Cells ? 32 : 0);
  }
}

// Block rows of a stage's five launches, each in its kernel's own unit: normal x (1 padded row), normal y (g.ny
// face rows), flux x (g.fx face rows), flux y (1 face row), update (1 interior row); g is 4 and 4 for the
// 128-face form (32 x 4 tiles), 1 and 1 for the 16-face form. A stage can be issued in pieces: every launch covers
// the block rows from what was issued before up to a target, so no row is computed twice.
struct Rows5 {
  int nx, ny, fx, fy, up;
};
struct Gran {
  int ny, fx;
};
inline Gran gran_of(bool small) { return small ? Gran{1, 1} : Gran{4, 4}; }

inline Rows5 rows_total(int ny, Gran g) {
  return Rows5{ny + 5, (ny + 1 + g.ny - 1) / g.ny, (ny + g.fx - 1) / g.fx, ny + 1, ny};
}

// What update rows [0, U) need from the other four launches when the whole stage input is present: flux x face
// rows < U, flux y face rows <= U, the normal y face rows that flux y reads, and normal x rows up to 5 past the
// last flux x face row (its transverse stencils).
inline Rows5 rows_for_update(int ny, int U, Gran g) {
  const Rows5 T = rows_total(ny, g);
  Rows5 r;
  r.up = U;
  r.fx = std::min(T.fx, (U + g.fx - 1) / g.fx);
  r.fy = std::min(T.fy, U + 1);
  r.ny = std::min(T.ny, (r.fy + g.ny - 1) / g.ny);
  r.nx = std::min(T.nx, g.fx * r.fx + 5);
  return r;
}

// What the first A interior rows of a stage input allow of the two normal reconstructions under the transmissive
// boundary (ghost row p reads interior row clamp(p - 3, 0, ny - 1)): normal x row r reads padded row r, so
// r < A + 3; normal y face row r reads padded rows r .. r + 5, so a block of rows needs its last row r + 2 < A.
inline Rows5 normals_for_rows(int ny, int A, Rows5 done, Gran g) {
  const Rows5 T = rows_total(ny, g);
  Rows5 r = done;
  if (A >= ny) {
    r.nx = T.nx;
    r.ny = T.ny;
  } else {
    r.nx = std::max(done.nx, std::min(T.nx, A + 3));
    r.ny = std::max(done.ny, std::min(T.ny, A >= 2 ? (A - 2) / g.ny : 0));
  }
  return r;
}

template <int M, int FACES>
int launch_rows_form(wsr_ctx* ctx, const StageArgs& a, const Ws2d& w, const FaceMaps& fm, cudaStream_t st,
                     Rows5& done, const Rows5& want) {
  const auto P = stage_params<M>(ctx, a);
  const dim3 blk(kBlock);
  constexpr bool kAll = FACES == kBlock;
  if (want.nx > done.nx) {
    ProfScope ps(ctx, st, 0);
    k_normal<M, 1, FACES><<<dim3((a.nx + 1 + FACES - 1) / FACES, want.nx - done.nx), blk, 0, st>>>(
        a.u_stage, w.xl, w.xr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts, w.fallbacks, w.counters + 0, P,
        done.nx);
  }
  WSR_LAUNCHED(ctx, "k_normal<x>");
  done.nx = std::max(done.nx, want.nx);
  if (want.ny > done.ny) {
    ProfScope ps(ctx, st, 1);
    k_normal<M, 2, FACES><<<dim3(kAll ? (a.nx + 5 + 31) / 32 : (a.nx + 5 + FACES - 1) / FACES, want.ny - done.ny),
                            blk, 0, st>>>(a.u_stage, w.yl, w.yr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts,
                                          w.fallbacks, w.counters + 2, P, done.ny);
  }
  WSR_LAUNCHED(ctx, "k_normal<y>");
  done.ny = std::max(done.ny, want.ny);
  if (want.fx > done.fx) {
    ProfScope ps(ctx, st, 2);
    k_flux<M, 1, FACES><<<dim3(kAll ? (a.nx + 1 + 31) / 32 : (a.nx + 1 + FACES - 1) / FACES, want.fx - done.fx), blk,
                          0, st>>>(w.xl, w.xr, w.fx, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks,
                                   w.counters + 4, P, fm.xl, fm.xr, done.fx);
  }
  WSR_LAUNCHED(ctx, "k_flux<x>");
  done.fx = std::max(done.fx, want.fx);
  if (want.fy > done.fy) {
    ProfScope ps(ctx, st, 3);
    k_flux<M, 2, FACES><<<dim3((a.nx + FACES - 1) / FACES, want.fy - done.fy), blk, 0, st>>>(
        w.yl, w.yr, w.fy, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks, w.counters + 6, P, fm.yl,
        fm.yr, done.fy);
  }
  WSR_LAUNCHED(ctx, "k_flux<y>");
  done.fy = std::max(done.fy, want.fy);
  if (want.up > done.up) {
    ProfScope ps(ctx, st, 4);
    k_update<<<dim3((a.nx + 255) / 256, want.up - done.up), 256, 0, st>>>(a.u_stage, a.u0, a.u_out, w.fx, w.fy, a.nx,
                                                                          a.ny, a.rk, a.g, w.ctl, done.up);
  }
  WSR_LAUNCHED(ctx, "k_update");
  done.up = std::max(done.up, want.up);
  return WSR_OK;
}

template <int M>
int launch_rows(wsr_ctx* ctx, const StageArgs& a, const Ws2d& w, const FaceMaps& fm, cudaStream_t st, Rows5& done,
                const Rows5& want) {
  if constexpr (M == M_SRBF16_TC || !has_mlp<M>()) {
    return launch_rows_form<M, kBlock>(ctx, a, w, fm, st, done, want);
  } else {
    const int faces = small_faces<M>(a);
    if (faces == 16) return launch_rows_form<M, 16>(ctx, a, w, fm, st, done, want);
    if (faces == 32) return launch_rows_form<M, 32>(ctx, a, w, fm, st, done, want);
    return launch_rows_form<M, kBlock>(ctx, a, w, fm, st, done, want);
  }
}

int dispatch_rows(wsr_ctx* ctx, int method, const StageArgs& a, const Ws2d& w, const FaceMaps& fm, cudaStream_t st,
                  Rows5& done, const Rows5& want) {
  switch (method) {
    case WSR_METHOD_JS:
      return launch_rows<M_JS>(ctx, a, w, fm, st, done, want);
    case WSR_METHOD_SR_F64:
      return launch_rows<M_SR64>(ctx, a, w, fm, st, done, want);
    case WSR_METHOD_SR_F32:
      return launch_rows<M_SR32>(ctx, a, w, fm, st, done, want);
    case WSR_METHOD_Z:
      return launch_rows<M_Z>(ctx, a, w, fm, st, done, want);
    case WSR_METHOD_SR_BF16_TC:
      return launch_rows<M_SRBF16_TC>(ctx, a, w, fm, st, done, want);
    default:
      return launch_rows<M_SRBF16>(ctx, a, w, fm, st, done, want);
  }
}

// The row granularity the stage's launches use (which form dispatch_rows picks).
Gran stage_gran(int method, const StageArgs& a) {
  switch (method) {
    case WSR_METHOD_JS:
      return gran_of(small_faces<M_JS>(a) != 0);
    case WSR_METHOD_SR_F64:
      return gran_of(small_faces<M_SR64>(a) != 0);
    case WSR_METHOD_SR_F32:
      return gran_of(small_faces<M_SR32>(a) != 0);
    case WSR_METHOD_Z:
      return gran_of(small_faces<M_Z>(a) != 0);
    case WSR_METHOD_SR_BF16_TC:
      return gran_of(false);
    default:
      return gran_of(small_faces<M_SRBF16>(a) != 0);
  }
}

// One whole stage.
int dispatch_stage(wsr_ctx* ctx, int method, const StageArgs& a, const Ws2d& w, const FaceMaps& fm, cudaStream_t st) {
  Rows5 done{0, 0, 0, 0, 0};
  return dispatch_rows(ctx, method, a, w, fm, st, done, rows_total(a.ny, stage_gran(method, a)));
}

// Accumulates a host-buffer call's outcome for wsr_euler2d_host_wait: [0] stencil tile loads that timed out,
// [1] steps taken, [2] JS fallbacks.
__global__ void k_host_status(const StepCtl* ctl, const int* fallbacks, unsigned long long* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  status[0] += fallbacks[1] ? 1ull : 0ull;
  status[1] += (unsigned long long)ctl->steps;
  status[2] += (unsigned long long)fallbacks[0];
}

__global__ void k_init_ctl(StepCtl* ctl, int* fallbacks, unsigned long long* counters, double t_start, double t_end, double dt, double dx, double dy, double cfl,
                           double hmin, int check_health, int check_interval, int max_steps) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  ctl->t = t_start;
  ctl->t_end = t_end;
  ctl->dt = dt;
  ctl->dt_dx = dt / dx;
  ctl->dt_dy = dt / dy;
  ctl->max_speed_bits = 0ull;
  ctl->steps = 0;
  ctl->done = 0;
  ctl->health_bad = 0;
  ctl->fallbacks = 0;
  ctl->check_health = check_health;
  ctl->check_interval = check_interval;
  ctl->max_steps = max_steps;
  ctl->cfl = cfl;
  ctl->hmin = hmin;
  fallbacks[0] = 0;
  fallbacks[1] = 0;  // set by k_flux when a stencil tile load timed out
  for (int k = 0; k < 8; ++k) counters[k] = 0ull;
}

// Variant of k_step_begin that writes into a ring of kDtsRing records.
__global__ void k_step_begin_ring(StepCtl* ctl, double* ring) {
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
  ring[ctl->steps % kDtsRing] = dt;
}

}  // namespace

// Copy streams, band events and the status word of wsr_euler2d_advance_host, one per context. The bands are the
// interior rows cut into `nb` pieces; `pending` says that the last call's read-backs may still run.
constexpr int kHostBandsMax = 16;
struct wsr_host_pipe {
  cudaStream_t h2d, d2h;
  cudaEvent_t start, up[kHostBandsMax], ready[kHostBandsMax], down[kHostBandsMax], down_all, compute_end;
  unsigned long long* status;  // device: the k_host_status accumulators since the last wait
  const double* host;          // host array of the last call
  double* bufs[4];             // its device state buffers
  int nx, ny, nb;              // grid and band count of the last call
  bool pending;
};

namespace {

void destroy_pipe(wsr_host_pipe* p) {
  if (!p) return;
  if (p->status) cudaFree(p->status);
  cudaEventDestroy(p->start);
  cudaEventDestroy(p->down_all);
  cudaEventDestroy(p->compute_end);
  for (int k = 0; k < kHostBandsMax; ++k) {
    cudaEventDestroy(p->up[k]);
    cudaEventDestroy(p->ready[k]);
    cudaEventDestroy(p->down[k]);
  }
  cudaStreamDestroy(p->h2d);
  cudaStreamDestroy(p->d2h);
  delete p;
}

int make_pipe(wsr_ctx* ctx) {
  if (ctx->host) return WSR_OK;
  wsr_host_pipe* p = new (std::nothrow) wsr_host_pipe();
  if (!p) return fail(ctx, WSR_ERR_ARG, "out of host memory");
  std::memset(p, 0, sizeof(*p));
  const unsigned f = cudaEventDisableTiming;
  cudaError_t e = cudaStreamCreateWithFlags(&p->h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->start, f);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->down_all, f);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->compute_end, f);
  for (int k = 0; k < kHostBandsMax && e == cudaSuccess; ++k) {
    e = cudaEventCreateWithFlags(&p->up[k], f);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ready[k], f);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->down[k], f);
  }
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&p->status), 4 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(p->status, 0, 4 * sizeof(unsigned long long));
  if (e != cudaSuccess) {
    destroy_pipe(p);
    return fail(ctx, WSR_ERR_CUDA, "host pipe: %s", cudaGetErrorString(e));
  }
  ctx->host = p;
  return WSR_OK;
}

// Interior rows [band_lo(k), band_lo(k + 1)) of band k of nb. The first and last bands are half as high as the
// others (nb > 2): the first read-back starts sooner and the last upload ends sooner (at 2000^2 on the benchmark
// state 6.30-6.33 ms per call with 8 such bands against 6.36-6.37 with 7 equal ones). nb <= ny / 2 + 1 keeps every
// band at least one row high.
inline int band_lo(int ny, int nb, int k) {
  if (k <= 0) return 0;
  if (k >= nb) return ny;
  if (nb <= 2) return (int)((long long)ny * k / nb);
  return (int)(((double)k - 0.5) / (double)(nb - 1) * (double)ny);
}

}  // namespace

extern "C" {

// Message of the last wsr_ctx_create that failed on this thread (there is no context to hold it).
thread_local char g_create_err[256] = "";

int wsr_ctx_create(int device, wsr_ctx** out) {
  if (!out) {
    std::snprintf(g_create_err, sizeof(g_create_err), "wsr_ctx_create: null output pointer");
    return WSR_ERR_ARG;
  }
  *out = nullptr;
  wsr_ctx* ctx = new (std::nothrow) wsr_ctx();
  if (!ctx) {
    std::snprintf(g_create_err, sizeof(g_create_err), "wsr_ctx_create: out of host memory");
    return WSR_ERR_ARG;
  }
  std::memset(ctx, 0, sizeof(*ctx));
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  const char* what = "cudaSetDevice";
  if (e == cudaSuccess) {
    e = cudaMallocHost(reinterpret_cast<void**>(&ctx->host_pinned), 4096);
    what = "cudaMallocHost";
  }
  if (e != cudaSuccess) {
    std::snprintf(g_create_err, sizeof(g_create_err), "wsr_ctx_create(device %d): %s: %s", device, what,
                  cudaGetErrorString(e));
    delete ctx;
    return WSR_ERR_CUDA;
  }
  *out = ctx;
  return WSR_OK;
}

void wsr_ctx_destroy(wsr_ctx* ctx) {
  if (!ctx) return;
  if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
  if (ctx->host) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->host->h2d);
    cudaStreamSynchronize(ctx->host->d2h);
    destroy_pipe(ctx->host);
  }
  if (ctx->prof_created)
    for (int k = 0; k < kProfEvents; ++k) {
      cudaEventDestroy(ctx->ev_a[k]);
      cudaEventDestroy(ctx->ev_b[k]);
    }
  delete ctx;
}

const char* wsr_last_error(const wsr_ctx* ctx) {
  if (ctx) return ctx->err;
  return g_create_err[0] ? g_create_err : "null context";
}

int wsr_closure_upload(wsr_ctx* ctx, int kind, const double* packed, int n) {
  if (!ctx) return WSR_ERR_ARG;
  if (kind == 7) {
    if (!packed || n != kParams7) return fail(ctx, WSR_ERR_ARG, "expected %d WENO7 parameters, got %d", kParams7, n);
    for (int k = 0; k < kParams7; ++k) {
      ctx->q64.p[k] = packed[k];
      ctx->q32.p[k] = static_cast<float>(packed[k]);
      ctx->qbf16.p[k] = __bfloat162float(__float2bfloat16_rn(static_cast<float>(packed[k])));
    }
    ctx->have_closure7 = true;
    return WSR_OK;
  }
  if (kind != 5) return fail(ctx, WSR_ERR_ARG, "closure kind %d not supported (5 = WENO5, 7 = WENO7)", kind);
  if (!packed || n != kParams5) return fail(ctx, WSR_ERR_ARG, "expected %d WENO5 parameters, got %d", kParams5, n);
  for (int k = 0; k < kParams5; ++k) {
    ctx->p64.p[k] = packed[k];
    ctx->p32.p[k] = static_cast<float>(packed[k]);
    ctx->pbf16.p[k] = __bfloat162float(__float2bfloat16_rn(static_cast<float>(packed[k])));
  }
  ctx->p32.duplicate();
  ctx->pbf16.duplicate();
  ctx->have_closure = true;
  return WSR_OK;
}

size_t wsr_euler2d_workspace_bytes(int nx, int ny) {
  if (nx < 1 || ny < 1) return 0;
  return ws_bytes(nx, ny);
}

int wsr_euler2d_stage_at(wsr_ctx* ctx, const double* u_stage, const double* u0, double* u_out, int nx, int ny,
                         double dx, double dy, double gamma, double dt, int rk, int method, int bc, int flux, int opts,
                         double boundary_time, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_2d(ctx, nx, ny, method, bc, flux, workspace, workspace_bytes);
  if (rc) return rc;
  if (!u_stage || !u0 || !u_out) return fail(ctx, WSR_ERR_ARG, "null state pointer");
  if (misaligned(u_stage) || misaligned(u0) || misaligned(u_out))
    return fail(ctx, WSR_ERR_ARG, "state arrays must be 16-byte aligned");
  if (rk < 1 || rk > 3) return fail(ctx, WSR_ERR_ARG, "rk must be 1, 2 or 3 (got %d)", rk);
  if (!(dt > 0.0) || !(dx > 0.0) || !(dy > 0.0)) return fail(ctx, WSR_ERR_ARG, "dt, dx, dy must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((rc = wsr_euler2d_host_order(ctx, stream))) return rc;  // after host-buffer read-backs still in flight
  Ws2d w = carve(workspace, nx, ny);
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, boundary_time, 1.0e300, dt, dx, dy, 0.0, 0.0, 0, 0, 1);
  WSR_LAUNCHED(ctx, "k_init_ctl");
  FaceMaps fm;
  if (!face_maps(w, nx, ny, &fm)) return fail(ctx, WSR_ERR_CUDA, "encoding the face-value tensor maps failed");
  StageArgs a{u_stage, u0, u_out, nx, ny, bc, flux, opts, rk, dx, dy, gamma, 0.0};
  return dispatch_stage(ctx, method, a, w, fm, st);
}

int wsr_euler2d_stage(wsr_ctx* ctx, const double* u_stage, const double* u0, double* u_out, int nx, int ny,
                      double dx, double dy, double gamma, double dt, int rk, int method, int bc, int flux, int opts,
                      void* workspace, size_t workspace_bytes, void* stream) {
  return wsr_euler2d_stage_at(ctx, u_stage, u0, u_out, nx, ny, dx, dy, gamma, dt, rk, method, bc, flux, opts, 0.0,
                              workspace, workspace_bytes, stream);
}

int wsr_euler2d_max_speed(wsr_ctx* ctx, const double* u, int nx, int ny, double gamma, double* out_host,
                          void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_2d(ctx, nx, ny, WSR_METHOD_JS, WSR_BC_TRANSMISSIVE, WSR_FLUX_HLLC, workspace, workspace_bytes);
  if (rc) return rc;
  if (!u || !out_host) return fail(ctx, WSR_ERR_ARG, "null pointer");
  if (misaligned(u)) return fail(ctx, WSR_ERR_ARG, "state array must be 16-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws2d w = carve(workspace, nx, ny);
  WSR_CUDA(ctx, cudaMemsetAsync(&w.ctl->max_speed_bits, 0, sizeof(unsigned long long), st));
  k_max_speed<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(u, nx, ny, gamma, &w.ctl->max_speed_bits, 0);
  WSR_LAUNCHED(ctx, "k_max_speed");
  unsigned long long bits = 0;
  WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned, &w.ctl->max_speed_bits, sizeof(bits), cudaMemcpyDeviceToHost, st));
  WSR_CUDA(ctx, cudaStreamSynchronize(st));
  std::memcpy(&bits, ctx->host_pinned, sizeof(bits));
  double v;
  std::memcpy(&v, &bits, sizeof(v));
  *out_host = v;
  return WSR_OK;
}

int wsr_euler2d_run(wsr_ctx* ctx, double* const u[4], int nx, int ny, double dx, double dy, double gamma, double cfl,
                    double t_start, double t_end, int method, int bc, int flux, int opts, int check_health, int check_interval,
                    int fixed_steps, int max_steps, double* dts_host, int* steps_out, double* t_out, int* final_slot,
                    int* fallbacks_out, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_2d(ctx, nx, ny, method, bc, flux, workspace, workspace_bytes);
  if (rc) return rc;
  if (bc & WSR_BC_Y_HALO)
    return fail(ctx, WSR_ERR_ARG, "WSR_BC_Y_HALO needs ghost rows refreshed between stages: use wsr_euler2d_stage");
  if (!u || !u[0] || !u[1] || !u[2] || !u[3]) return fail(ctx, WSR_ERR_ARG, "null state buffer");
  if (misaligned(u[0]) || misaligned(u[1]) || misaligned(u[2]) || misaligned(u[3]))
    return fail(ctx, WSR_ERR_ARG, "state arrays must be 16-byte aligned");
  if (max_steps < 1) return fail(ctx, WSR_ERR_ARG, "max_steps must be >= 1");
  if (!(cfl > 0.0) || !(dx > 0.0) || !(dy > 0.0)) return fail(ctx, WSR_ERR_ARG, "cfl, dx, dy must be positive");
  if (fixed_steps > 0) {
    t_end = 1.0e300;
    max_steps = fixed_steps;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((rc = wsr_euler2d_host_order(ctx, stream))) return rc;  // after host-buffer read-backs still in flight
  Ws2d w = carve(workspace, nx, ny);
  const double hmin = dx < dy ? dx : dy;
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, fixed_steps > 0 ? 0.0 : t_start, t_end, 0.0, dx, dy, cfl, hmin,
                              check_health, check_interval,
                              max_steps);
  WSR_LAUNCHED(ctx, "k_init_ctl");
  k_max_speed<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(u[0], nx, ny, gamma, &w.ctl->max_speed_bits, 0);
  WSR_LAUNCHED(ctx, "k_max_speed");
  FaceMaps fm;
  if (!face_maps(w, nx, ny, &fm)) return fail(ctx, WSR_ERR_CUDA, "encoding the face-value tensor maps failed");
  const int batch = 16;  // steps launched between host polls (<= kDtsRing)
  int host_steps = 0;    // steps the host has launched
  int seen_steps = 0;    // steps whose dt has been copied out
  int done = 0;
  StepCtl snap;
  while (!done) {
    // a fixed-step run launches exactly its steps; a t_end run polls every `batch` steps
    const int nb = fixed_steps > 0 ? (max_steps - host_steps < batch ? max_steps - host_steps : batch) : batch;
    if (nb <= 0) break;
    for (int b = 0; b < nb; ++b) {
      const int s = host_steps + b;
      double* in = (s & 1) ? u[3] : u[0];
      double* out = (s & 1) ? u[0] : u[3];
      {
        ProfScope ps(ctx, st, 5);
        k_step_begin_ring<<<1, 1, 0, st>>>(w.ctl, w.dts);
        k_set_dt_ratios<<<1, 1, 0, st>>>(w.ctl, dx, dy);
      }
      WSR_LAUNCHED(ctx, "k_step_begin");
      StageArgs a1{in, in, u[1], nx, ny, bc, flux, opts, 1, dx, dy, gamma, 0.0};
      StageArgs a2{u[1], in, u[2], nx, ny, bc, flux, opts, 2, dx, dy, gamma, 1.0};
      StageArgs a3{u[2], in, out, nx, ny, bc, flux, opts, 3, dx, dy, gamma, 0.5};
      if ((rc = dispatch_stage(ctx, method, a1, w, fm, st))) return rc;
      if ((rc = dispatch_stage(ctx, method, a2, w, fm, st))) return rc;
      if ((rc = dispatch_stage(ctx, method, a3, w, fm, st))) return rc;
      {
        ProfScope ps(ctx, st, 5);
        k_step_end<<<1, 1, 0, st>>>(w.ctl);
      }
      WSR_LAUNCHED(ctx, "k_step_end");
    }
    host_steps += nb;
    WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned, w.ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
    WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned + 128, w.dts, kDtsRing * sizeof(double), cudaMemcpyDeviceToHost, st));
    WSR_CUDA(ctx, cudaStreamSynchronize(st));
    std::memcpy(&snap, ctx->host_pinned, sizeof(StepCtl));
    for (int s = seen_steps; s < snap.steps; ++s)
      if (dts_host && s < max_steps) dts_host[s] = ctx->host_pinned[128 + (s % kDtsRing)];
    seen_steps = snap.steps;
    done = snap.done;
  }
  int fb[2] = {0, 0};
  WSR_CUDA(ctx, cudaMemcpy(fb, w.fallbacks, sizeof(fb), cudaMemcpyDeviceToHost));
  if (fb[1]) return fail(ctx, WSR_ERR_CUDA, "a stencil tile load (TMA) did not complete in time");
  if (steps_out) *steps_out = snap.steps;
  if (t_out) *t_out = snap.t;
  if (final_slot) *final_slot = (snap.steps & 1) ? 3 : 0;
  if (fallbacks_out) *fallbacks_out = fb[0];
  return WSR_OK;
}

// Queues one host-buffer call (wsr_euler2d_advance_host); on success the call's copies and kernels are in flight.
static int advance_host_enqueue(wsr_ctx* ctx, double* u_host, double* const u[4], int nx, int ny, double dx,
                                double dy, double gamma, double cfl, int steps, int method, int bc, int flux, int opts,
                                int flags, int bands, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_2d(ctx, nx, ny, method, bc, flux, workspace, workspace_bytes);
  if (rc) return rc;
  if (bc & WSR_BC_Y_HALO) return fail(ctx, WSR_ERR_ARG, "WSR_BC_Y_HALO is for wsr_euler2d_stage");
  if (!u_host) return fail(ctx, WSR_ERR_ARG, "null host array");
  if (!u || !u[0] || !u[1] || !u[2] || !u[3]) return fail(ctx, WSR_ERR_ARG, "null state buffer");
  if (misaligned(u[0]) || misaligned(u[1]) || misaligned(u[2]) || misaligned(u[3]))
    return fail(ctx, WSR_ERR_ARG, "state arrays must be 16-byte aligned");
  if (steps < 1) return fail(ctx, WSR_ERR_ARG, "steps must be >= 1");
  if (!(cfl > 0.0) || !(dx > 0.0) || !(dy > 0.0)) return fail(ctx, WSR_ERR_ARG, "cfl, dx, dy must be positive");
  if (flags & ~WSR_HOST_ASYNC) return fail(ctx, WSR_ERR_ARG, "bad flags %d", flags);
  if (bands < 0) return fail(ctx, WSR_ERR_ARG, "bands must be >= 0");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  if ((rc = make_pipe(ctx))) return rc;
  wsr_host_pipe* p = ctx->host;
  cudaPointerAttributes attr;
  WSR_CUDA(ctx, cudaPointerGetAttributes(&attr, u_host));
  // pageable memory copies synchronously: one band, no overlap
  // one band per 250 rows: on the 2000^2 benchmark state 4 / 7 / 10 / 14 / 20 equal bands took 7.01 / 6.70 / 6.74 /
  // 7.15 / 7.42 ms per call (more bands start the copies sooner but cut the heavy stage kernels into more tails)
  int nb = bands > 0 ? bands : ny / 250;
  nb = attr.type == cudaMemoryTypeHost ? std::max(1, std::min(std::min(nb, kHostBandsMax), ny / 2 + 1)) : 1;
  Ws2d w = carve(workspace, nx, ny);
  FaceMaps fm;
  if (!face_maps(w, nx, ny, &fm)) return fail(ctx, WSR_ERR_CUDA, "encoding the face-value tensor maps failed");
  const size_t pitch = (size_t)(nx + 6) * 4 * sizeof(double), width = (size_t)nx * 4 * sizeof(double);
  auto row_at = [&](double* base, int row) { return base + ((size_t)(row + kGhost) * (nx + 6) + kGhost) * 4; };

  // uploads of the interior rows, band by band. Chained on one host array, band k waits for the previous call's
  // read-back of band k (which came after that call's last use of those rows of u[0]); otherwise for earlier work
  // on the stream and every read-back still running.
  const bool chained = p->pending && p->host == u_host && p->nx == nx && p->ny == ny && p->nb == nb &&
                       p->bufs[0] == u[0] && p->bufs[1] == u[1] && p->bufs[2] == u[2] && p->bufs[3] == u[3];
  if (!chained) {
    WSR_CUDA(ctx, cudaEventRecord(p->start, st));
    WSR_CUDA(ctx, cudaStreamWaitEvent(p->h2d, p->start, 0));
    if (p->pending) WSR_CUDA(ctx, cudaStreamWaitEvent(p->h2d, p->down_all, 0));
  }
  for (int k = 0; k < nb; ++k) {
    const int r0 = band_lo(ny, nb, k), r1 = band_lo(ny, nb, k + 1);
    if (chained) WSR_CUDA(ctx, cudaStreamWaitEvent(p->h2d, p->down[k], 0));
    WSR_CUDA(ctx, cudaMemcpy2DAsync(row_at(u[0], r0), pitch, row_at(u_host, r0), pitch, width, r1 - r0,
                                    cudaMemcpyHostToDevice, p->h2d));
    WSR_CUDA(ctx, cudaEventRecord(p->up[k], p->h2d));
  }

  const double hmin = dx < dy ? dx : dy;
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, 0.0, 1.0e300, 0.0, dx, dy, cfl, hmin, 0, 0, steps);
  WSR_LAUNCHED(ctx, "k_init_ctl");
  // the first stage's normal reconstructions follow the upload band by band (transmissive: every row they read is
  // an interior row near their own); the wave speed, and with it dt, needs every band
  const bool overlap = bc == WSR_BC_TRANSMISSIVE;
  for (int s = 0; s < steps; ++s) {
    double* in = (s & 1) ? u[3] : u[0];
    double* out = (s & 1) ? u[0] : u[3];
    const StageArgs a1{in, in, u[1], nx, ny, bc, flux, opts, 1, dx, dy, gamma, 0.0};
    const StageArgs a2{u[1], in, u[2], nx, ny, bc, flux, opts, 2, dx, dy, gamma, 1.0};
    const StageArgs a3{u[2], in, out, nx, ny, bc, flux, opts, 3, dx, dy, gamma, 0.5};
    const Gran g = stage_gran(method, a1);
    Rows5 done{0, 0, 0, 0, 0};
    if (s == 0) {
      for (int k = 0; k < nb; ++k) {
        const int r0 = band_lo(ny, nb, k), r1 = band_lo(ny, nb, k + 1);
        WSR_CUDA(ctx, cudaStreamWaitEvent(st, p->up[k], 0));
        k_max_speed<<<dim3((nx + 255) / 256, r1 - r0), 256, 0, st>>>(u[0], nx, ny, gamma, &w.ctl->max_speed_bits, r0);
        WSR_LAUNCHED(ctx, "k_max_speed");
        if (overlap && (rc = dispatch_rows(ctx, method, a1, w, fm, st, done, normals_for_rows(ny, r1, done, g))))
          return rc;
      }
    }
    k_step_begin_ring<<<1, 1, 0, st>>>(w.ctl, w.dts);
    k_set_dt_ratios<<<1, 1, 0, st>>>(w.ctl, dx, dy);
    WSR_LAUNCHED(ctx, "k_step_begin");
    if ((rc = dispatch_rows(ctx, method, a1, w, fm, st, done, rows_total(ny, g)))) return rc;
    if ((rc = dispatch_stage(ctx, method, a2, w, fm, st))) return rc;
    if (s == steps - 1) {
      // the last stage band by band, each band's read-back as soon as its rows are final
      Rows5 d3{0, 0, 0, 0, 0};
      for (int k = 0; k < nb; ++k) {
        const int r0 = band_lo(ny, nb, k), r1 = band_lo(ny, nb, k + 1);
        if ((rc = dispatch_rows(ctx, method, a3, w, fm, st, d3, rows_for_update(ny, r1, g)))) return rc;
        WSR_CUDA(ctx, cudaEventRecord(p->ready[k], st));
        WSR_CUDA(ctx, cudaStreamWaitEvent(p->d2h, p->ready[k], 0));
        WSR_CUDA(ctx, cudaMemcpy2DAsync(row_at(u_host, r0), pitch, row_at(out, r0), pitch, width, r1 - r0,
                                        cudaMemcpyDeviceToHost, p->d2h));
        WSR_CUDA(ctx, cudaEventRecord(p->down[k], p->d2h));
      }
    } else if ((rc = dispatch_stage(ctx, method, a3, w, fm, st))) {
      return rc;
    }
    k_step_end<<<1, 1, 0, st>>>(w.ctl);
    WSR_LAUNCHED(ctx, "k_step_end");
  }
  k_host_status<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, p->status);
  WSR_LAUNCHED(ctx, "k_host_status");
  WSR_CUDA(ctx, cudaEventRecord(p->compute_end, st));
  WSR_CUDA(ctx, cudaEventRecord(p->down_all, p->d2h));
  p->host = u_host;
  for (int k = 0; k < 4; ++k) p->bufs[k] = u[k];
  p->nx = nx;
  p->ny = ny;
  p->nb = nb;
  p->pending = true;
  return WSR_OK;
}

int wsr_euler2d_advance_host(wsr_ctx* ctx, double* u_host, double* const u[4], int nx, int ny, double dx, double dy,
                             double gamma, double cfl, int steps, int method, int bc, int flux, int opts, int flags,
                             int bands, void* workspace, size_t workspace_bytes, void* stream) {
  const int rc = advance_host_enqueue(ctx, u_host, u, nx, ny, dx, dy, gamma, cfl, steps, method, bc, flux, opts, flags,
                                      bands, workspace, workspace_bytes, stream);
  if (rc != WSR_OK) {
    // copies of this call may already be queued: let them finish before the caller can release u_host, and start
    // the next call afresh
    if (ctx && ctx->host) {
      cudaStreamSynchronize(ctx->host->h2d);
      cudaStreamSynchronize(ctx->host->d2h);
      ctx->host->pending = false;
      ctx->host->host = nullptr;
    }
    return rc;
  }
  if (flags & WSR_HOST_ASYNC) return WSR_OK;
  return wsr_euler2d_host_wait(ctx, nullptr, nullptr);
}

int wsr_euler2d_host_order(wsr_ctx* ctx, void* stream) {
  if (!ctx) return WSR_ERR_ARG;
  wsr_host_pipe* p = ctx->host;
  if (!p || !p->pending) return WSR_OK;
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  WSR_CUDA(ctx, cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), p->down_all, 0));
  WSR_CUDA(ctx, cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), p->compute_end, 0));
  return WSR_OK;
}

int wsr_euler2d_host_wait(wsr_ctx* ctx, int* steps_out, int* fallbacks_out) {
  if (!ctx) return WSR_ERR_ARG;
  if (steps_out) *steps_out = 0;
  if (fallbacks_out) *fallbacks_out = 0;
  wsr_host_pipe* p = ctx->host;
  if (!p) return WSR_OK;
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  WSR_CUDA(ctx, cudaEventSynchronize(p->compute_end));
  WSR_CUDA(ctx, cudaStreamWaitEvent(p->d2h, p->compute_end, 0));
  WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned, p->status, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                p->d2h));
  WSR_CUDA(ctx, cudaMemsetAsync(p->status, 0, 4 * sizeof(unsigned long long), p->d2h));
  WSR_CUDA(ctx, cudaStreamSynchronize(p->d2h));
  unsigned long long h[4];
  std::memcpy(h, ctx->host_pinned, sizeof(h));
  p->pending = false;
  if (steps_out) *steps_out = (int)h[1];
  if (fallbacks_out) *fallbacks_out = (int)h[2];
  if (h[0]) return fail(ctx, WSR_ERR_CUDA, "a stencil tile load (TMA) did not complete in time");
  return WSR_OK;
}

int wsr_profile_enable(wsr_ctx* ctx, int on) {
  if (!ctx) return WSR_ERR_ARG;
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  if (on && !ctx->prof_created) {
    for (int k = 0; k < kProfEvents; ++k) {
      WSR_CUDA(ctx, cudaEventCreate(&ctx->ev_a[k]));
      WSR_CUDA(ctx, cudaEventCreate(&ctx->ev_b[k]));
    }
    ctx->prof_created = true;
  }
  if (ctx->prof_on) {
    int rc = prof_flush(ctx);
    if (rc) return rc;
  }
  ctx->prof_on = on != 0;
  ctx->n_ev = 0;
  for (int k = 0; k < kProfKinds; ++k) {
    ctx->prof_ms[k] = 0.0;
    ctx->prof_count[k] = 0;
  }
  return WSR_OK;
}

int wsr_profile_read(wsr_ctx* ctx, double* ms, long long* launches) {
  if (!ctx || !ms || !launches) return WSR_ERR_ARG;
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  int rc = prof_flush(ctx);
  if (rc) return rc;
  for (int k = 0; k < kProfKinds; ++k) {
    ms[k] = ctx->prof_ms[k];
    launches[k] = ctx->prof_count[k];
  }
  return WSR_OK;
}

// ---- device-resident time loop of a y-slab (one slab of a decomposed grid per rank) ----
// The control block of the workspace carries t, dt and the stop flag as in wsr_euler2d_run; between these calls
// the caller exchanges the halo rows and all-reduces (MAX) the 64-bit wave-speed slot, all on the device.
int wsr_euler2d_slab_begin(wsr_ctx* ctx, const double* u, int nx, int ny, double dx, double dy, double gamma,
                           double cfl, double t_start, double t_end, int max_steps, void* workspace,
                           size_t workspace_bytes, void* stream) {
  int rc = check_2d(ctx, nx, ny, WSR_METHOD_JS, WSR_BC_TRANSMISSIVE, WSR_FLUX_HLLC, workspace, workspace_bytes);
  if (rc) return rc;
  if (!u || misaligned(u)) return fail(ctx, WSR_ERR_ARG, "state must be a 16-byte aligned device array");
  if (max_steps < 1 || !(cfl > 0.0) || !(dx > 0.0) || !(dy > 0.0))
    return fail(ctx, WSR_ERR_ARG, "max_steps, cfl, dx, dy must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws2d w = carve(workspace, nx, ny);
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, t_start, t_end, 0.0, dx, dy, cfl, dx < dy ? dx : dy, 0,
                              0, max_steps);
  WSR_LAUNCHED(ctx, "k_init_ctl");
  k_max_speed<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(u, nx, ny, gamma, &w.ctl->max_speed_bits, 0);
  WSR_LAUNCHED(ctx, "k_max_speed");
  return WSR_OK;
}

int wsr_euler2d_slab_speed_slot(wsr_ctx* ctx, void* workspace, size_t workspace_bytes, int nx, int ny,
                                unsigned long long** slot) {
  if (!ctx || !workspace || !slot) return WSR_ERR_ARG;
  if (workspace_bytes < ws_bytes(nx, ny)) return fail(ctx, WSR_ERR_ARG, "workspace too small");
  *slot = &carve(workspace, nx, ny).ctl->max_speed_bits;
  return WSR_OK;
}

int wsr_euler2d_slab_step(wsr_ctx* ctx, int phase, int nx, int ny, double dx, double dy, void* workspace,
                          size_t workspace_bytes, void* stream) {
  if (!ctx || !workspace || (phase != 0 && phase != 1)) return WSR_ERR_ARG;
  if (workspace_bytes < ws_bytes(nx, ny)) return fail(ctx, WSR_ERR_ARG, "workspace too small");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws2d w = carve(workspace, nx, ny);
  if (phase == 0) {
    k_step_begin_ring<<<1, 1, 0, st>>>(w.ctl, w.dts);
    k_set_dt_ratios<<<1, 1, 0, st>>>(w.ctl, dx, dy);
  } else {
    k_step_end<<<1, 1, 0, st>>>(w.ctl);
  }
  WSR_LAUNCHED(ctx, "slab step control");
  return WSR_OK;
}

int wsr_euler2d_slab_stage(wsr_ctx* ctx, const double* u_stage, const double* u0, double* u_out, int nx, int ny,
                           double dx, double dy, double gamma, int rk, int method, int bc, int flux, int opts,
                           void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_2d(ctx, nx, ny, method, bc, flux, workspace, workspace_bytes);
  if (rc) return rc;
  if ((bc & ~WSR_BC_Y_HALO) == WSR_BC_DOUBLE_MACH) return fail(ctx, WSR_ERR_ARG, "slabs take no double-Mach boundary");
  if (!u_stage || !u0 || !u_out || misaligned(u_stage) || misaligned(u0) || misaligned(u_out))
    return fail(ctx, WSR_ERR_ARG, "state arrays must be 16-byte aligned device arrays");
  if (rk < 1 || rk > 3) return fail(ctx, WSR_ERR_ARG, "rk must be 1, 2 or 3 (got %d)", rk);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws2d w = carve(workspace, nx, ny);
  FaceMaps fm;
  if (!face_maps(w, nx, ny, &fm)) return fail(ctx, WSR_ERR_CUDA, "encoding the face-value tensor maps failed");
  StageArgs a{u_stage, u0, u_out, nx, ny, bc, flux, opts, rk, dx, dy, gamma, rk == 1 ? 0.0 : (rk == 2 ? 1.0 : 0.5)};
  return dispatch_stage(ctx, method, a, w, fm, st);
}

int wsr_euler2d_slab_status(wsr_ctx* ctx, void* workspace, size_t workspace_bytes, int nx, int ny, int* steps,
                            double* t, int* done, double* dts_ring, void* stream) {
  if (!ctx || !workspace) return WSR_ERR_ARG;
  if (workspace_bytes < ws_bytes(nx, ny)) return fail(ctx, WSR_ERR_ARG, "workspace too small");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws2d w = carve(workspace, nx, ny);
  WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned, w.ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
  WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned + 128, w.dts, kDtsRing * sizeof(double), cudaMemcpyDeviceToHost, st));
  WSR_CUDA(ctx, cudaStreamSynchronize(st));
  StepCtl snap;
  std::memcpy(&snap, ctx->host_pinned, sizeof(StepCtl));
  if (steps) *steps = snap.steps;
  if (t) *t = snap.t;
  if (done) *done = snap.done;
  if (dts_ring) std::memcpy(dts_ring, ctx->host_pinned + 128, kDtsRing * sizeof(double));
  int fb[2] = {0, 0};
  WSR_CUDA(ctx, cudaMemcpy(fb, w.fallbacks, sizeof(fb), cudaMemcpyDeviceToHost));
  if (fb[1]) return fail(ctx, WSR_ERR_CUDA, "a stencil tile load (TMA) did not complete in time");
  return WSR_OK;
}

int wsr_euler2d_counters(wsr_ctx* ctx, void* workspace, size_t workspace_bytes, int nx, int ny,
                         unsigned long long* out_host) {
  if (!ctx || !workspace || !out_host) return WSR_ERR_ARG;
  if (workspace_bytes < ws_bytes(nx, ny)) return fail(ctx, WSR_ERR_ARG, "workspace too small");
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws2d w = carve(workspace, nx, ny);
  WSR_CUDA(ctx, cudaMemcpy(out_host, w.counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return WSR_OK;
}

}  // extern "C"

namespace {
// Independent FMA chains for the peak-throughput probe (8 per thread).
template <typename T>
__global__ void __launch_bounds__(256) k_fma_probe(T* out, int iters, T a, T b) {
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-12345.678)) out[blockIdx.x] = s;  // keeps the chains live
}
}  // namespace

extern "C" int wsr_probe_peak_flops(wsr_ctx* ctx, int bits, double* tflops, void* stream) {
  if (!ctx || !tflops || (bits != 32 && bits != 64)) return WSR_ERR_ARG;
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int sms = 0;
  WSR_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  const int blocks = sms * 8, threads = 256, iters = bits == 32 ? 4096 : 2048;
  void* out = nullptr;
  WSR_CUDA(ctx, cudaMallocAsync(&out, blocks * sizeof(double), st));
  cudaEvent_t e0, e1;
  WSR_CUDA(ctx, cudaEventCreate(&e0));
  WSR_CUDA(ctx, cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    WSR_CUDA(ctx, cudaEventRecord(e0, st));
    if (bits == 32)
      k_fma_probe<float><<<blocks, threads, 0, st>>>(static_cast<float*>(out), iters, 0.9999f, 1e-4f);
    else
      k_fma_probe<double><<<blocks, threads, 0, st>>>(static_cast<double*>(out), iters, 0.9999, 1e-4);
    WSR_CUDA(ctx, cudaEventRecord(e1, st));
    WSR_CUDA(ctx, cudaEventSynchronize(e1));
    float ms = 0.f;
    WSR_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
    double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    double tf = flops / (ms * 1e-3) / 1e12;
    if (rep > 0 && tf > best) best = tf;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  WSR_CUDA(ctx, cudaFreeAsync(out, st));
  WSR_CUDA(ctx, cudaStreamSynchronize(st));
  *tflops = best;
  return WSR_OK;
}


// ---------------------------------------------------------------------------------------------
// No-allocation stage (wsr_euler2d_stage_noalloc).
//
// Some callers cannot call cudaMalloc: a host application that owns every byte of device memory
// through its own pool, or a solver step that must not pay cudaMalloc's implicit device
// synchronisation. For them the stage's scratch (face values, fluxes, step-control block) lives in
// the file-scope array below instead of a caller workspace. Every GPU that loads libwsr.so holds
// these WSR_NOALLOC_SCRATCH_BYTES until the process exits. All calls on a device share the array and
// it keeps the previous call's contents: the control block and counters are re-initialised by every
// call, and every face/flux value a call reads is written earlier in the same call, so nothing
// carries over; but calls that overlap on the GPU (e.g. on two streams at once) race on the array
// and must be serialised by the caller. The device address of the array is looked up once per device and
// cached for the life of the process; it does not survive cudaDeviceReset on that device.
// ---------------------------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[WSR_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoallocMaxDevices = 128;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoallocMaxDevices];  // device address of g_noalloc_scratch, per device

// Host code may not pass &g_noalloc_scratch to a kernel (it is a host-side stand-in, not a device
// address): the device address is looked up once per device, with that device current.
int noalloc_scratch_for(int dev, void** out) {
  if (dev < 0 || dev >= kNoallocMaxDevices) return WSR_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_addr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return WSR_ERR_CUDA;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return WSR_OK;
}

template <int M>
int noalloc_launch(const typename ClosureParams<M>::type& P, const StageArgs& a, const Ws2d& w, const FaceMaps& fm,
                   cudaStream_t st) {
  const dim3 blk(128);
  k_normal<M, 1><<<dim3((a.nx + 1 + 127) / 128, a.ny + 5), blk, 0, st>>>(
      a.u_stage, w.xl, w.xr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts, w.fallbacks, w.counters + 0, P, 0);
  k_normal<M, 2><<<dim3((a.nx + 5 + 31) / 32, (a.ny + 1 + 3) / 4), blk, 0, st>>>(
      a.u_stage, w.yl, w.yr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts, w.fallbacks, w.counters + 2, P, 0);
  k_flux<M, 1><<<dim3((a.nx + 1 + 31) / 32, (a.ny + 3) / 4), blk, 0, st>>>(
      w.xl, w.xr, w.fx, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks, w.counters + 4, P, fm.xl,
      fm.xr, 0);
  k_flux<M, 2><<<dim3((a.nx + 127) / 128, a.ny + 1), blk, 0, st>>>(
      w.yl, w.yr, w.fy, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks, w.counters + 6, P, fm.yl,
      fm.yr, 0);
  k_update<<<dim3((a.nx + 255) / 256, a.ny), 256, 0, st>>>(a.u_stage, a.u0, a.u_out, w.fx, w.fy, a.nx, a.ny, a.rk,
                                                          a.g, w.ctl, 0);
  // the error state was drained on entry, so an error here comes from these launches
  return cudaPeekAtLastError() == cudaSuccess ? WSR_OK : WSR_ERR_CUDA;
}

}  // namespace

extern "C" int wsr_euler2d_stage_noalloc(const double* u_stage, const double* u0, double* u_out, int nx, int ny,
                                         double dx, double dy, double gamma, double dt, int rk, int method, int bc,
                                         int flux, int opts, const double* closure_params, void* stream) {
  if (nx < 3 || ny < 3) return WSR_ERR_ARG;
  if (ws_bytes(nx, ny) > (size_t)WSR_NOALLOC_SCRATCH_BYTES) return WSR_ERR_SCRATCH_LIMIT;
  if (method < WSR_METHOD_JS || method > WSR_METHOD_Z) return WSR_ERR_ARG;
  if (bc != WSR_BC_TRANSMISSIVE && bc != WSR_BC_PERIODIC) return WSR_ERR_ARG;
  if (flux != WSR_FLUX_HLLC && flux != WSR_FLUX_FORCE) return WSR_ERR_ARG;
  if (rk < 1 || rk > 3 || !(dt > 0.0) || !(dx > 0.0) || !(dy > 0.0)) return WSR_ERR_ARG;
  if (!u_stage || !u0 || !u_out || misaligned(u_stage) || misaligned(u0) || misaligned(u_out)) return WSR_ERR_ARG;
  if (method != WSR_METHOD_JS && method != WSR_METHOD_Z && !closure_params) return WSR_ERR_NO_CLOSURE;
  // Drain a launch error left in this thread's error state by earlier, unrelated work, so that the checks below
  // report only this call's launches (an error that made the context unusable is sticky and still reported).
  (void)cudaGetLastError();
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return WSR_ERR_CUDA;
  void* scratch = nullptr;
  int rc = noalloc_scratch_for(dev, &scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Ws2d w = carve(scratch, nx, ny);
  FaceMaps fm;
  if (!face_maps(w, nx, ny, &fm)) return WSR_ERR_CUDA;
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, 0.0, 1.0, dt, dx, dy, 0.0, 0.0, 0, 0, 1);
  if (cudaPeekAtLastError() != cudaSuccess) return WSR_ERR_CUDA;
  StageArgs a{u_stage, u0, u_out, nx, ny, bc, flux, opts, rk, dx, dy, gamma, 0.0};
  switch (method) {
    case WSR_METHOD_JS:
      return noalloc_launch<M_JS>(NoParams{}, a, w, fm, st);
    case WSR_METHOD_Z:
      return noalloc_launch<M_Z>(ZEps{dx * dx, dy * dy}, a, w, fm, st);
    case WSR_METHOD_SR_F64: {
      Mlp5d P;
      for (int k = 0; k < kParams5; ++k) P.p[k] = closure_params[k];
      return noalloc_launch<M_SR64>(P, a, w, fm, st);
    }
    case WSR_METHOD_SR_F32: {
      Mlp5f P;
      for (int k = 0; k < kParams5; ++k) P.p[k] = static_cast<float>(closure_params[k]);
      P.duplicate();
      return noalloc_launch<M_SR32>(P, a, w, fm, st);
    }
    default: {
      Mlp5f P;
      for (int k = 0; k < kParams5; ++k)
        P.p[k] = __bfloat162float(__float2bfloat16_rn(static_cast<float>(closure_params[k])));
      P.duplicate();
      return noalloc_launch<M_SRBF16>(P, a, w, fm, st);
    }
  }
}
