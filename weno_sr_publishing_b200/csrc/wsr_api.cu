// extern "C" entry points of libwsr.so (declared in include/wsr.h).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include "../../include/wsr.h"
#include "adv1d.cuh"
#include "euler2d.cuh"
#include "euler2d_w7.cuh"
#include "train1d.cuh"
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

size_t cells_bytes(size_t n) { return align_up(n * 4 * sizeof(double)); }

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

int check_2d(wsr_ctx* ctx, int nx, int ny, int method, int bc, int flux, void* ws, size_t wsb) {
  if (!ctx) return WSR_ERR_ARG;
  if (nx < 3 || ny < 3) return fail(ctx, WSR_ERR_ARG, "nx and ny must be >= 3 (got %d, %d)", nx, ny);
  if ((long long)(nx + 6) * (ny + 6) > (1ll << 31) / 4)
    return fail(ctx, WSR_ERR_ARG, "grid %d x %d too large for one launch", nx, ny);
  if (method < WSR_METHOD_JS || method > WSR_METHOD_Z) return fail(ctx, WSR_ERR_ARG, "bad method %d", method);
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

template <int M>
int launch_stage(wsr_ctx* ctx, const StageArgs& a, const Ws2d& w, cudaStream_t st) {
  const auto P = stage_params<M>(ctx, a);
  const dim3 blk(128);  // the reconstruction kernels compact closure work per warp of a 128-thread block
  {
    ProfScope ps(ctx, st, 0);
    dim3 grd((a.nx + 1 + 127) / 128, a.ny + 5);
    k_normal<M, 1><<<grd, blk, 0, st>>>(a.u_stage, w.xl, w.xr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts, w.fallbacks,
                                        w.counters + 0, P);
  }
  WSR_LAUNCHED(ctx, "k_normal<x>");
  {
    ProfScope ps(ctx, st, 1);
    dim3 grd((a.nx + 5 + 31) / 32, (a.ny + 1 + 3) / 4);
    k_normal<M, 2><<<grd, blk, 0, st>>>(a.u_stage, w.yl, w.yr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts, w.fallbacks,
                                        w.counters + 2, P);
  }
  WSR_LAUNCHED(ctx, "k_normal<y>");
  {
    ProfScope ps(ctx, st, 2);
    dim3 grd((a.nx + 1 + 31) / 32, (a.ny + 3) / 4);
    k_flux<M, 1><<<grd, blk, 0, st>>>(w.xl, w.xr, w.fx, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks,
                                      w.counters + 4, P);
  }
  WSR_LAUNCHED(ctx, "k_flux<x>");
  {
    ProfScope ps(ctx, st, 3);
    dim3 grd((a.nx + 127) / 128, a.ny + 1);
    k_flux<M, 2><<<grd, blk, 0, st>>>(w.yl, w.yr, w.fy, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks,
                                      w.counters + 6, P);
  }
  WSR_LAUNCHED(ctx, "k_flux<y>");
  {
    ProfScope ps(ctx, st, 4);
    dim3 grd((a.nx + 255) / 256, a.ny);
    k_update<<<grd, 256, 0, st>>>(a.u_stage, a.u0, a.u_out, w.fx, w.fy, a.nx, a.ny, a.rk, a.g, w.ctl);
  }
  WSR_LAUNCHED(ctx, "k_update");
  return WSR_OK;
}

int dispatch_stage(wsr_ctx* ctx, int method, const StageArgs& a, const Ws2d& w, cudaStream_t st) {
  switch (method) {
    case WSR_METHOD_JS:
      return launch_stage<M_JS>(ctx, a, w, st);
    case WSR_METHOD_SR_F64:
      return launch_stage<M_SR64>(ctx, a, w, st);
    case WSR_METHOD_SR_F32:
      return launch_stage<M_SR32>(ctx, a, w, st);
    case WSR_METHOD_Z:
      return launch_stage<M_Z>(ctx, a, w, st);
    default:
      return launch_stage<M_SRBF16>(ctx, a, w, st);
  }
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
  *fallbacks = 0;
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

extern "C" {

int wsr_ctx_create(int device, wsr_ctx** out) {
  if (!out) return WSR_ERR_ARG;
  *out = nullptr;
  wsr_ctx* ctx = new (std::nothrow) wsr_ctx();
  if (!ctx) return WSR_ERR_ARG;
  std::memset(ctx, 0, sizeof(*ctx));
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&ctx->host_pinned), 4096);
  if (e != cudaSuccess) {
    delete ctx;
    return WSR_ERR_CUDA;
  }
  *out = ctx;
  return WSR_OK;
}

void wsr_ctx_destroy(wsr_ctx* ctx) {
  if (!ctx) return;
  if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
  if (ctx->prof_created)
    for (int k = 0; k < kProfEvents; ++k) {
      cudaEventDestroy(ctx->ev_a[k]);
      cudaEventDestroy(ctx->ev_b[k]);
    }
  delete ctx;
}

const char* wsr_last_error(const wsr_ctx* ctx) { return ctx ? ctx->err : "null context"; }

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
  Ws2d w = carve(workspace, nx, ny);
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, boundary_time, 1.0e300, dt, dx, dy, 0.0, 0.0, 0, 0, 1);
  WSR_LAUNCHED(ctx, "k_init_ctl");
  StageArgs a{u_stage, u0, u_out, nx, ny, bc, flux, opts, rk, dx, dy, gamma, 0.0};
  return dispatch_stage(ctx, method, a, w, st);
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
  k_max_speed<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(u, nx, ny, gamma, &w.ctl->max_speed_bits);
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
  Ws2d w = carve(workspace, nx, ny);
  const double hmin = dx < dy ? dx : dy;
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, fixed_steps > 0 ? 0.0 : t_start, t_end, 0.0, dx, dy, cfl, hmin,
                              check_health, check_interval,
                              max_steps);
  WSR_LAUNCHED(ctx, "k_init_ctl");
  k_max_speed<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(u[0], nx, ny, gamma, &w.ctl->max_speed_bits);
  WSR_LAUNCHED(ctx, "k_max_speed");
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
      if ((rc = dispatch_stage(ctx, method, a1, w, st))) return rc;
      if ((rc = dispatch_stage(ctx, method, a2, w, st))) return rc;
      if ((rc = dispatch_stage(ctx, method, a3, w, st))) return rc;
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
  int fb = 0;
  WSR_CUDA(ctx, cudaMemcpy(&fb, w.fallbacks, sizeof(int), cudaMemcpyDeviceToHost));
  if (steps_out) *steps_out = snap.steps;
  if (t_out) *t_out = snap.t;
  if (final_slot) *final_slot = (snap.steps & 1) ? 3 : 0;
  if (fallbacks_out) *fallbacks_out = fb;
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

// ---------------------------------------------------------------------------------------------
// Batched 1D advection
// ---------------------------------------------------------------------------------------------
namespace {

template <int SCHEME, int M>
const typename AdvParams<SCHEME, M>::type& adv_params_of(const wsr_ctx* ctx);
template <>
const NoParams& adv_params_of<5, M_JS>(const wsr_ctx*) {
  static const NoParams np{};
  return np;
}
template <>
const NoParams& adv_params_of<7, M_JS>(const wsr_ctx*) {
  static const NoParams np{};
  return np;
}
template <>
const Mlp5d& adv_params_of<5, M_SR64>(const wsr_ctx* c) { return c->p64; }
template <>
const Mlp5f& adv_params_of<5, M_SR32>(const wsr_ctx* c) { return c->p32; }
template <>
const Mlp5f& adv_params_of<5, M_SRBF16>(const wsr_ctx* c) { return c->pbf16; }
template <>
const Mlp7d& adv_params_of<7, M_SR64>(const wsr_ctx* c) { return c->q64; }
template <>
const Mlp7f& adv_params_of<7, M_SR32>(const wsr_ctx* c) { return c->q32; }
template <>
const Mlp7f& adv_params_of<7, M_SRBF16>(const wsr_ctx* c) { return c->qbf16; }

struct AdvArgs {
  double* u;
  const long long* offsets;
  const int* order;
  const double *vel, *dx;
  const int* nfull;
  const double *dtf, *dtl;
  int B, nmax, opts;
  int *fallbacks, *errors;
  unsigned long long* counters;
};

template <int SCHEME, int M, int INTEG>
int adv_launch(wsr_ctx* ctx, const AdvArgs& a, cudaStream_t st) {
  const size_t smem = adv_smem_bytes<INTEG>(a.nmax);
  auto kern = k_adv1d<SCHEME, M, INTEG>;
  WSR_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<a.B, kAdvThreads, smem, st>>>(a.u, a.offsets, a.order, a.vel, a.dx, a.nfull, a.dtf, a.dtl, a.B, a.nmax,
                                        a.opts, a.fallbacks, a.errors, a.counters, adv_params_of<SCHEME, M>(ctx));
  WSR_LAUNCHED(ctx, "k_adv1d");
  return WSR_OK;
}

template <int SCHEME, int INTEG>
int adv_dispatch_m(wsr_ctx* ctx, int method, const AdvArgs& a, cudaStream_t st) {
  switch (method) {
    case WSR_METHOD_JS:
      return adv_launch<SCHEME, M_JS, INTEG>(ctx, a, st);
    case WSR_METHOD_SR_F64:
      return adv_launch<SCHEME, M_SR64, INTEG>(ctx, a, st);
    case WSR_METHOD_SR_F32:
      return adv_launch<SCHEME, M_SR32, INTEG>(ctx, a, st);
    default:
      return adv_launch<SCHEME, M_SRBF16, INTEG>(ctx, a, st);
  }
}

}  // namespace

extern "C" size_t wsr_adv1d_workspace_bytes(void) { return 256; }

extern "C" int wsr_adv1d_run(wsr_ctx* ctx, double* u, const long long* offsets, const int* order,
                             const double* velocity, const double* dx, const int* n_full, const double* dt_full,
                             const double* dt_last, int B, int nmax, int scheme, int method, int integrator, int opts,
                             int* fallbacks_out, int* errors_out, unsigned long long* counters_out, void* workspace,
                             size_t workspace_bytes, void* stream) {
  if (!ctx) return WSR_ERR_ARG;
  if (B < 1) return fail(ctx, WSR_ERR_ARG, "B must be >= 1");
  if (scheme != 5 && scheme != 7) return fail(ctx, WSR_ERR_ARG, "scheme must be 5 or 7 (got %d)", scheme);
  if (integrator != WSR_INTEG_SSPRK3 && integrator != WSR_INTEG_SHU_RK4)
    return fail(ctx, WSR_ERR_ARG, "bad integrator %d", integrator);
  if (method < WSR_METHOD_JS || method > WSR_METHOD_SR_BF16) return fail(ctx, WSR_ERR_ARG, "bad method %d", method);
  if (nmax < (scheme == 5 ? 5 : 7) || nmax > kAdvNmax)
    return fail(ctx, WSR_ERR_ARG, "nmax must be in [%d, %d] (got %d)", scheme == 5 ? 5 : 7, kAdvNmax, nmax);
  if (method != WSR_METHOD_JS && !(scheme == 5 ? ctx->have_closure : ctx->have_closure7))
    return fail(ctx, WSR_ERR_NO_CLOSURE, "SR method requested before uploading a WENO%d closure", scheme);
  if (!u || !offsets || !velocity || !dx || !n_full || !dt_full || !dt_last)
    return fail(ctx, WSR_ERR_ARG, "null array argument");
  if (!workspace || workspace_bytes < wsr_adv1d_workspace_bytes())
    return fail(ctx, WSR_ERR_ARG, "workspace too small");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  int* fb = static_cast<int*>(workspace);
  int* err = fb + 1;
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(static_cast<char*>(workspace) + 16);
  WSR_CUDA(ctx, cudaMemsetAsync(workspace, 0, 32, st));
  AdvArgs a{u, offsets, order, velocity, dx, n_full, dt_full, dt_last, B, nmax, opts, fb, err, cnt};
  int rc;
  if (scheme == 5)
    rc = integrator == WSR_INTEG_SSPRK3 ? adv_dispatch_m<5, 0>(ctx, method, a, st) : adv_dispatch_m<5, 1>(ctx, method, a, st);
  else
    rc = integrator == WSR_INTEG_SSPRK3 ? adv_dispatch_m<7, 0>(ctx, method, a, st) : adv_dispatch_m<7, 1>(ctx, method, a, st);
  if (rc) return rc;
  if (fallbacks_out || errors_out || counters_out) {
    int host[4];
    unsigned long long hc[2];
    WSR_CUDA(ctx, cudaMemcpyAsync(host, workspace, 16, cudaMemcpyDeviceToHost, st));
    WSR_CUDA(ctx, cudaMemcpyAsync(hc, cnt, 16, cudaMemcpyDeviceToHost, st));
    WSR_CUDA(ctx, cudaStreamSynchronize(st));
    if (fallbacks_out) *fallbacks_out = host[0];
    if (errors_out) *errors_out = host[1];
    if (counters_out) {
      counters_out[0] = hc[0];
      counters_out[1] = hc[1];
    }
    if (host[1]) return fail(ctx, WSR_ERR_ARG, "%d trajectories had fewer cells than the stencil or more than nmax", host[1]);
  }
  return WSR_OK;
}

namespace {

struct WsTrain {
  double* ck;         // B x K x n checkpoint states (every ckpt_every-th step)
  double* seg;        // B x min(every, steps) x 3 x n stage states of the segment being reversed
  unsigned* signs;    // B x steps x ceil(n/32) x 2 ballot words of sign(u - e)
  double* loss_part;  // B
  double* grad_part;  // B x 189
};

size_t train_ws_bytes(int B, int n, int steps, int every) {
  const size_t K = (size_t)(steps + every - 1) / every, seg = (size_t)(every < steps ? every : steps);
  const size_t words = (size_t)(n + 31) / 32;
  return align_up((size_t)B * K * n * sizeof(double)) + align_up((size_t)B * seg * 3 * n * sizeof(double)) +
         align_up((size_t)B * steps * words * 2 * sizeof(unsigned)) + align_up((size_t)B * sizeof(double)) +
         align_up((size_t)B * kP5 * sizeof(double));
}

WsTrain carve_train(void* base, int B, int n, int steps, int every) {
  const size_t K = (size_t)(steps + every - 1) / every, seg = (size_t)(every < steps ? every : steps);
  const size_t words = (size_t)(n + 31) / 32;
  char* p = static_cast<char*>(base);
  WsTrain w;
  w.ck = reinterpret_cast<double*>(p);
  p += align_up((size_t)B * K * n * sizeof(double));
  w.seg = reinterpret_cast<double*>(p);
  p += align_up((size_t)B * seg * 3 * n * sizeof(double));
  w.signs = reinterpret_cast<unsigned*>(p);
  p += align_up((size_t)B * steps * words * 2 * sizeof(unsigned));
  w.loss_part = reinterpret_cast<double*>(p);
  p += align_up((size_t)B * sizeof(double));
  w.grad_part = reinterpret_cast<double*>(p);
  return w;
}

int check_train(wsr_ctx* ctx, const double* velocity, int B, int n, double dx, double dt, int steps, int every,
                int method, void* ws, size_t wsb) {
  if (!ctx) return WSR_ERR_ARG;
  if (B < 1) return fail(ctx, WSR_ERR_ARG, "B must be >= 1");
  if (n < 5 || n > kTrainNmax) return fail(ctx, WSR_ERR_ARG, "n must be in [5, %d] (got %d)", kTrainNmax, n);
  if (steps < 1 || every < 1) return fail(ctx, WSR_ERR_ARG, "steps and ckpt_every must be >= 1");
  if (!(dx > 0.0) || !(dt > 0.0)) return fail(ctx, WSR_ERR_ARG, "dx and dt must be positive");
  if (method != WSR_METHOD_SR_F64 && method != WSR_METHOD_SR_F32)
    return fail(ctx, WSR_ERR_ARG, "training needs WSR_METHOD_SR_F64 or WSR_METHOD_SR_F32 (got %d)", method);
  if (!ctx->have_closure) return fail(ctx, WSR_ERR_NO_CLOSURE, "training called before wsr_closure_upload");
  if (!velocity) return fail(ctx, WSR_ERR_ARG, "null velocity array");
  if (!ws) return fail(ctx, WSR_ERR_ARG, "workspace is NULL");
  if (reinterpret_cast<uintptr_t>(ws) % kAlign) return fail(ctx, WSR_ERR_ARG, "workspace must be 256-byte aligned");
  if (wsb < train_ws_bytes(B, n, steps, every))
    return fail(ctx, WSR_ERR_ARG, "workspace too small: %zu < %zu bytes", wsb, train_ws_bytes(B, n, steps, every));
  return WSR_OK;
}

template <int M>
int train_fwd_launch(wsr_ctx* ctx, const double* u0, const double* desc, const double* vel, int B, int n, double dx,
                     double dt, int steps, int every, double* loss_out, double* u_final, const WsTrain& w,
                     cudaStream_t st) {
  const size_t smem = train_fwd_smem(n);
  auto kern = k_train_fwd<M>;
  WSR_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<B, kTrainThreads, smem, st>>>(u0, desc, vel, n, dx, dt, steps, every, w.ck, w.signs, w.loss_part, u_final,
                                       params_of<M>(ctx));
  WSR_LAUNCHED(ctx, "k_train_fwd");
  k_train_reduce<<<1, 256, 0, st>>>(w.loss_part, nullptr, B, 1.0 / ((double)B * (double)steps * (double)n),
                                    loss_out, nullptr);
  WSR_LAUNCHED(ctx, "k_train_reduce");
  return WSR_OK;
}

template <int M>
int train_bwd_launch(wsr_ctx* ctx, const double* vel, int B, int n, double dx, double dt, int steps, int every,
                     double* grad_out, double* grad_u0, const WsTrain& w, cudaStream_t st) {
  const size_t smem = train_bwd_smem<M>(n);
  auto kern = k_train_bwd<M>;
  WSR_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const double gscale = 1.0 / ((double)B * (double)steps * (double)n);
  kern<<<B, kTrainThreads, smem, st>>>(w.ck, w.signs, vel, n, dx, dt, steps, every, gscale, w.seg, w.grad_part,
                                       grad_u0, params_of<M>(ctx));
  WSR_LAUNCHED(ctx, "k_train_bwd");
  k_train_reduce<<<1, 256, 0, st>>>(nullptr, w.grad_part, B, 0.0, nullptr, grad_out);
  WSR_LAUNCHED(ctx, "k_train_reduce");
  return WSR_OK;
}

}  // namespace

extern "C" size_t wsr_train1d_workspace_bytes(int B, int n, int steps, int ckpt_every) {
  if (B < 1 || n < 1 || steps < 1 || ckpt_every < 1) return 0;
  return train_ws_bytes(B, n, steps, ckpt_every);
}

extern "C" int wsr_train1d_forward(wsr_ctx* ctx, const double* u0, const double* desc, const double* velocity, int B,
                                   int n, double dx, double dt, int steps, int ckpt_every, int method,
                                   double* loss_out, double* u_final, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  const int rc = check_train(ctx, velocity, B, n, dx, dt, steps, ckpt_every, method, workspace, workspace_bytes);
  if (rc) return rc;
  if (!desc || !loss_out) return fail(ctx, WSR_ERR_ARG, "null desc or loss_out");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  const WsTrain w = carve_train(workspace, B, n, steps, ckpt_every);
  return method == WSR_METHOD_SR_F64
             ? train_fwd_launch<M_SR64>(ctx, u0, desc, velocity, B, n, dx, dt, steps, ckpt_every, loss_out, u_final, w, st)
             : train_fwd_launch<M_SR32>(ctx, u0, desc, velocity, B, n, dx, dt, steps, ckpt_every, loss_out, u_final, w, st);
}

extern "C" int wsr_train1d_backward(wsr_ctx* ctx, const double* velocity, int B, int n, double dx, double dt,
                                    int steps, int ckpt_every, int method, double* grad_out, double* grad_u0,
                                    void* workspace, size_t workspace_bytes, void* stream) {
  const int rc = check_train(ctx, velocity, B, n, dx, dt, steps, ckpt_every, method, workspace, workspace_bytes);
  if (rc) return rc;
  if (!grad_out) return fail(ctx, WSR_ERR_ARG, "null grad_out");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  const WsTrain w = carve_train(workspace, B, n, steps, ckpt_every);
  return method == WSR_METHOD_SR_F64
             ? train_bwd_launch<M_SR64>(ctx, velocity, B, n, dx, dt, steps, ckpt_every, grad_out, grad_u0, w, st)
             : train_bwd_launch<M_SR32>(ctx, velocity, B, n, dx, dt, steps, ckpt_every, grad_out, grad_u0, w, st);
}

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

// ---------------------------------------------------------------------------------------------
// 2D Euler WENO7 (JS, Z, SR-FP64) with Shu RK4 (weno7_point_rk4_shu/point_rk4.py, weno7_point_rk4_z.py,
// teacherfree_lab_weno7_rk4_distance_balanced_fast/warp_sod/point_rk4_mlp.py).
// ---------------------------------------------------------------------------------------------
namespace {

struct Ws7 {
  StepCtl* ctl;
  double* dts;                     // ring of kDtsRing
  unsigned long long* counters;    // SR closure evaluations: normal x, normal y, flux x, flux y
  double *xl, *xr, *yl, *yr, *fx, *fy;
  double *u1, *u2, *u3;
  double* rhs[6];  // rhs0, rhs_t0, rhs1, rhs_t1, rhs2, rhs3 (interior)
};

size_t ws7_bytes(int nx, int ny) {
  const size_t np = (size_t)(nx + 8) * (ny + 8), ni = (size_t)nx * ny;
  return align_up(sizeof(StepCtl)) + align_up(kDtsRing * sizeof(double)) + align_up(4 * sizeof(unsigned long long)) +
         2 * cells_bytes((size_t)(ny + 8) * (nx + 2)) + 2 * cells_bytes((size_t)(ny + 2) * (nx + 8)) +
         cells_bytes((size_t)ny * (nx + 1)) + cells_bytes((size_t)(ny + 1) * nx) + 3 * cells_bytes(np) +
         6 * cells_bytes(ni);
}

Ws7 carve7(void* base, int nx, int ny) {
  char* p = static_cast<char*>(base);
  auto take = [&](size_t bytes) {
    char* q = p;
    p += bytes;
    return reinterpret_cast<double*>(q);
  };
  Ws7 w;
  w.ctl = reinterpret_cast<StepCtl*>(take(align_up(sizeof(StepCtl))));
  w.dts = take(align_up(kDtsRing * sizeof(double)));
  w.counters = reinterpret_cast<unsigned long long*>(take(align_up(4 * sizeof(unsigned long long))));
  w.xl = take(cells_bytes((size_t)(ny + 8) * (nx + 2)));
  w.xr = take(cells_bytes((size_t)(ny + 8) * (nx + 2)));
  w.yl = take(cells_bytes((size_t)(ny + 2) * (nx + 8)));
  w.yr = take(cells_bytes((size_t)(ny + 2) * (nx + 8)));
  w.fx = take(cells_bytes((size_t)ny * (nx + 1)));
  w.fy = take(cells_bytes((size_t)(ny + 1) * nx));
  const size_t np = (size_t)(nx + 8) * (ny + 8);
  w.u1 = take(cells_bytes(np));
  w.u2 = take(cells_bytes(np));
  w.u3 = take(cells_bytes(np));
  for (int k = 0; k < 6; ++k) w.rhs[k] = take(cells_bytes((size_t)nx * ny));
  return w;
}

int check7(wsr_ctx* ctx, int nx, int ny, int bc, int method, void* ws, size_t wsb) {
  if (!ctx) return WSR_ERR_ARG;
  if (method != WSR_METHOD_JS && method != WSR_METHOD_Z && method != WSR_METHOD_SR_F64)
    return fail(ctx, WSR_ERR_ARG, "WENO7 2D method must be WSR_METHOD_JS, WSR_METHOD_Z or WSR_METHOD_SR_F64 (got %d)",
                method);
  if (method == WSR_METHOD_SR_F64 && !ctx->have_closure7)
    return fail(ctx, WSR_ERR_NO_CLOSURE, "WSR_METHOD_SR_F64 needs the WENO7 closure (wsr_closure_upload, scheme 7)");
  if (nx < 4 || ny < 4) return fail(ctx, WSR_ERR_ARG, "nx and ny must be >= 4 (got %d, %d)", nx, ny);
  if ((long long)(nx + 8) * (ny + 8) > (1ll << 31) / 4)
    return fail(ctx, WSR_ERR_ARG, "grid %d x %d too large for one launch", nx, ny);
  if (bc != WSR_BC_TRANSMISSIVE && bc != WSR_BC_PERIODIC) return fail(ctx, WSR_ERR_ARG, "bad boundary %d", bc);
  if (!ws) return fail(ctx, WSR_ERR_ARG, "workspace is NULL");
  if (reinterpret_cast<uintptr_t>(ws) % kAlign) return fail(ctx, WSR_ERR_ARG, "workspace must be 256-byte aligned");
  if (wsb < ws7_bytes(nx, ny))
    return fail(ctx, WSR_ERR_ARG, "workspace too small: %zu < %zu bytes", wsb, ws7_bytes(nx, ny));
  return WSR_OK;
}

// One right-hand side L(src) (reverse = 0) or L~(src) (reverse = 1) into rhs: 5 launches. z: WENO-Z
// weights with eps = dx^3 along x and dy^3 along y.
template <bool Z>
int launch_rhs7_t(wsr_ctx* ctx, const double* src, double* rhs, int nx, int ny, double dx, double dy, double g,
                  int bc, int reverse, const Ws7& w, cudaStream_t st) {
  const Gas gas = make_gas(g);
  const double ex = dx * dx * dx, ey = dy * dy * dy;
  w7::k7_normal<1, Z><<<dim3((nx + 1 + 127) / 128, ny + 7), 128, 0, st>>>(src, w.xl, w.xr, nx, ny, bc, gas, ex, w.ctl);
  WSR_LAUNCHED(ctx, "k7_normal<x>");
  w7::k7_normal<2, Z><<<dim3((nx + 7 + 31) / 32, (ny + 1 + 3) / 4), 128, 0, st>>>(src, w.yl, w.yr, nx, ny, bc, gas, ey,
                                                                                w.ctl);
  WSR_LAUNCHED(ctx, "k7_normal<y>");
  w7::k7_flux<1, Z><<<dim3((nx + 1 + 31) / 32, (ny + 3) / 4), 128, 0, st>>>(w.xl, w.xr, w.fx, nx, ny, gas, reverse,
                                                                           ey, w.ctl);
  WSR_LAUNCHED(ctx, "k7_flux<x>");
  w7::k7_flux<2, Z><<<dim3((nx + 127) / 128, ny + 1), 128, 0, st>>>(w.yl, w.yr, w.fy, nx, ny, gas, reverse, ex, w.ctl);
  WSR_LAUNCHED(ctx, "k7_flux<y>");
  w7::k7_rhs<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(w.fx, w.fy, rhs, nx, ny, 1.0 / dx, 1.0 / dy, w.ctl);
  WSR_LAUNCHED(ctx, "k7_rhs");
  return WSR_OK;
}

// The same right-hand side with the FP64 WENO7 closure.
int launch_rhs7_sr(wsr_ctx* ctx, const double* src, double* rhs, int nx, int ny, double dx, double dy, double g,
                   int bc, int reverse, const Ws7& w, cudaStream_t st) {
  const Gas gas = make_gas(g);
  const Mlp7d& P = ctx->q64;
  w7::k7s_normal<1><<<dim3((nx + 1 + 127) / 128, ny + 7), 128, 0, st>>>(src, w.xl, w.xr, nx, ny, bc, gas, w.ctl,
                                                                       w.counters + 0, P);
  WSR_LAUNCHED(ctx, "k7s_normal<x>");
  w7::k7s_normal<2><<<dim3((nx + 7 + 31) / 32, (ny + 1 + 3) / 4), 128, 0, st>>>(src, w.yl, w.yr, nx, ny, bc, gas,
                                                                               w.ctl, w.counters + 1, P);
  WSR_LAUNCHED(ctx, "k7s_normal<y>");
  w7::k7s_flux<1><<<dim3((nx + 1 + 31) / 32, (ny + 3) / 4), 128, 0, st>>>(w.xl, w.xr, w.fx, nx, ny, gas, reverse,
                                                                         w.ctl, w.counters + 2, P);
  WSR_LAUNCHED(ctx, "k7s_flux<x>");
  w7::k7s_flux<2><<<dim3((nx + 127) / 128, ny + 1), 128, 0, st>>>(w.yl, w.yr, w.fy, nx, ny, gas, reverse, w.ctl,
                                                                 w.counters + 3, P);
  WSR_LAUNCHED(ctx, "k7s_flux<y>");
  w7::k7_rhs<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(w.fx, w.fy, rhs, nx, ny, 1.0 / dx, 1.0 / dy, w.ctl);
  WSR_LAUNCHED(ctx, "k7_rhs");
  return WSR_OK;
}

int launch_rhs7(wsr_ctx* ctx, const double* src, double* rhs, int nx, int ny, double dx, double dy, double g, int bc,
                int reverse, int method, const Ws7& w, cudaStream_t st) {
  if (method == WSR_METHOD_SR_F64) return launch_rhs7_sr(ctx, src, rhs, nx, ny, dx, dy, g, bc, reverse, w, st);
  return method == WSR_METHOD_Z ? launch_rhs7_t<true>(ctx, src, rhs, nx, ny, dx, dy, g, bc, reverse, w, st)
                                : launch_rhs7_t<false>(ctx, src, rhs, nx, ny, dx, dy, g, bc, reverse, w, st);
}

template <int S>
int launch_shu7(wsr_ctx* ctx, const w7::ShuArgs& a, int nx, int ny, const Ws7& w, cudaStream_t st) {
  w7::k7_shu<S><<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(a, nx, ny, w.ctl);
  WSR_LAUNCHED(ctx, "k7_shu");
  return WSR_OK;
}

// One Shu RK4 step of u (in place): L(u), L~(u), L(u1), L~(u1), L(u2), L(u3) and four combinations
// (point_rk4.py:514-538).
int shu_step7(wsr_ctx* ctx, double* u, int nx, int ny, double dx, double dy, double g, int bc, int method, const Ws7& w,
              cudaStream_t st) {
  int rc;
  double* const* R = w.rhs;
  w7::ShuArgs a{u, w.u1, w.u2, w.u3, R[0], R[1], R[2], R[3], R[4], R[5], nullptr};
  if ((rc = launch_rhs7(ctx, u, R[0], nx, ny, dx, dy, g, bc, 0, method, w, st))) return rc;
  a.out = w.u1;
  if ((rc = launch_shu7<1>(ctx, a, nx, ny, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, u, R[1], nx, ny, dx, dy, g, bc, 1, method, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u1, R[2], nx, ny, dx, dy, g, bc, 0, method, w, st))) return rc;
  a.out = w.u2;
  if ((rc = launch_shu7<2>(ctx, a, nx, ny, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u1, R[3], nx, ny, dx, dy, g, bc, 1, method, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u2, R[4], nx, ny, dx, dy, g, bc, 0, method, w, st))) return rc;
  a.out = w.u3;
  if ((rc = launch_shu7<3>(ctx, a, nx, ny, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u3, R[5], nx, ny, dx, dy, g, bc, 0, method, w, st))) return rc;
  a.out = u;
  return launch_shu7<4>(ctx, a, nx, ny, w, st);
}

__global__ void k7_init(StepCtl* ctl, unsigned long long* counters, double t_start, double t_end, double cfl,
                        double hmin, int max_steps) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < 4; ++k) counters[k] = 0ull;
  ctl->t = t_start;
  ctl->t_end = t_end;
  ctl->dt = 0.0;
  ctl->max_speed_bits = 0ull;
  ctl->steps = 0;
  ctl->done = 0;
  ctl->health_bad = 0;
  ctl->fallbacks = 0;
  ctl->check_health = 0;
  ctl->check_interval = 0;
  ctl->max_steps = max_steps;
  ctl->cfl = cfl;
  ctl->hmin = hmin;
}

}  // namespace

extern "C" size_t wsr_euler2d_w7_workspace_bytes(int nx, int ny) {
  if (nx < 4 || ny < 4) return 0;
  return ws7_bytes(nx, ny);
}

extern "C" int wsr_euler2d_w7_rhs(wsr_ctx* ctx, const double* u, double* rhs, int nx, int ny, double dx, double dy,
                                  double gamma, int bc, int method, int reverse, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  int rc = check7(ctx, nx, ny, bc, method, workspace, workspace_bytes);
  if (rc) return rc;
  if (!u || !rhs) return fail(ctx, WSR_ERR_ARG, "null pointer");
  if (misaligned(u) || misaligned(rhs)) return fail(ctx, WSR_ERR_ARG, "arrays must be 16-byte aligned");
  if (!(dx > 0.0) || !(dy > 0.0)) return fail(ctx, WSR_ERR_ARG, "dx, dy must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws7 w = carve7(workspace, nx, ny);
  k7_init<<<1, 1, 0, st>>>(w.ctl, w.counters, 0.0, 1.0, 0.0, 0.0, 1);
  WSR_LAUNCHED(ctx, "k7_init");
  return launch_rhs7(ctx, u, rhs, nx, ny, dx, dy, gamma, bc, reverse != 0, method, w, st);
}

extern "C" int wsr_euler2d_w7_run(wsr_ctx* ctx, double* u, int nx, int ny, double dx, double dy, double gamma,
                                  double cfl, double t_start, double t_end, int bc, int method, int max_steps,
                                  double* dts_host, int* steps_out, double* t_out, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  int rc = check7(ctx, nx, ny, bc, method, workspace, workspace_bytes);
  if (rc) return rc;
  if (!u) return fail(ctx, WSR_ERR_ARG, "null state");
  if (misaligned(u)) return fail(ctx, WSR_ERR_ARG, "state must be 16-byte aligned");
  if (max_steps < 1) return fail(ctx, WSR_ERR_ARG, "max_steps must be >= 1");
  if (!(cfl > 0.0) || !(dx > 0.0) || !(dy > 0.0)) return fail(ctx, WSR_ERR_ARG, "cfl, dx, dy must be positive");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws7 w = carve7(workspace, nx, ny);
  k7_init<<<1, 1, 0, st>>>(w.ctl, w.counters, t_start, t_end, cfl, dx < dy ? dx : dy, max_steps);
  WSR_LAUNCHED(ctx, "k7_init");
  const int batch = 16;  // steps launched between host polls (<= kDtsRing)
  int host_steps = 0, seen = 0, done = 0;
  StepCtl snap;
  std::memset(&snap, 0, sizeof(snap));
  while (!done) {
    const int nb = max_steps - host_steps < batch ? max_steps - host_steps : batch;
    if (nb <= 0) break;
    for (int b = 0; b < nb; ++b) {
      w7::k7_max_speed<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(u, nx, ny, gamma, w.ctl);
      w7::k7_step_begin<<<1, 1, 0, st>>>(w.ctl, w.dts, kDtsRing);
      WSR_LAUNCHED(ctx, "k7_step_begin");
      if ((rc = shu_step7(ctx, u, nx, ny, dx, dy, gamma, bc, method, w, st))) return rc;
      k_step_end<<<1, 1, 0, st>>>(w.ctl);
      WSR_LAUNCHED(ctx, "k_step_end");
    }
    host_steps += nb;
    WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned, w.ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, st));
    WSR_CUDA(ctx, cudaMemcpyAsync(ctx->host_pinned + 128, w.dts, kDtsRing * sizeof(double), cudaMemcpyDeviceToHost, st));
    WSR_CUDA(ctx, cudaStreamSynchronize(st));
    std::memcpy(&snap, ctx->host_pinned, sizeof(StepCtl));
    for (int s = seen; s < snap.steps; ++s)
      if (dts_host && s < max_steps) dts_host[s] = ctx->host_pinned[128 + (s % kDtsRing)];
    seen = snap.steps;
    done = snap.done;
  }
  if (steps_out) *steps_out = snap.steps;
  if (t_out) *t_out = snap.t;
  return WSR_OK;
}

extern "C" int wsr_euler2d_w7_counters(wsr_ctx* ctx, void* workspace, size_t workspace_bytes, int nx, int ny,
                                       unsigned long long* out_host) {
  if (!ctx || !workspace || !out_host) return WSR_ERR_ARG;
  if (nx < 4 || ny < 4 || workspace_bytes < ws7_bytes(nx, ny))
    return fail(ctx, WSR_ERR_ARG, "workspace does not hold a %d x %d WENO7 grid", nx, ny);
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  Ws7 w = carve7(workspace, nx, ny);
  WSR_CUDA(ctx, cudaMemcpy(out_host, w.counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return WSR_OK;
}

extern "C" int wsr_probe_exp_tab(wsr_ctx* ctx, const double* x, double* out, int n, void* stream) {
  if (!ctx || !x || !out || n < 0) return WSR_ERR_ARG;
  if (n == 0) return WSR_OK;
  WSR_CUDA(ctx, cudaSetDevice(ctx->device));
  w7::k_probe_exp_tab<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(x, out, n);
  WSR_LAUNCHED(ctx, "k_probe_exp_tab");
  return WSR_OK;
}

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
// and must be serialised by the caller.
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
int noalloc_launch(const typename ClosureParams<M>::type& P, const StageArgs& a, const Ws2d& w, cudaStream_t st) {
  const dim3 blk(128);
  k_normal<M, 1><<<dim3((a.nx + 1 + 127) / 128, a.ny + 5), blk, 0, st>>>(
      a.u_stage, w.xl, w.xr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts, w.fallbacks, w.counters + 0, P);
  k_normal<M, 2><<<dim3((a.nx + 5 + 31) / 32, (a.ny + 1 + 3) / 4), blk, 0, st>>>(
      a.u_stage, w.yl, w.yr, a.nx, a.ny, stage_bc(a), make_gas(a.g), w.ctl, a.opts, w.fallbacks, w.counters + 2, P);
  k_flux<M, 1><<<dim3((a.nx + 1 + 31) / 32, (a.ny + 3) / 4), blk, 0, st>>>(
      w.xl, w.xr, w.fx, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks, w.counters + 4, P);
  k_flux<M, 2><<<dim3((a.nx + 127) / 128, a.ny + 1), blk, 0, st>>>(
      w.yl, w.yr, w.fy, a.nx, a.ny, make_gas(a.g), a.flux, w.ctl, a.opts, w.fallbacks, w.counters + 6, P);
  k_update<<<dim3((a.nx + 255) / 256, a.ny), 256, 0, st>>>(a.u_stage, a.u0, a.u_out, w.fx, w.fy, a.nx, a.ny, a.rk,
                                                          a.g, w.ctl);
  return cudaGetLastError() == cudaSuccess ? WSR_OK : WSR_ERR_CUDA;
}

}  // namespace

extern "C" int wsr_euler2d_stage_noalloc(const double* u_stage, const double* u0, double* u_out, int nx, int ny,
                                         double dx, double dy, double gamma, double dt, int rk, int method, int bc,
                                         int flux, int opts, const double* closure_params, void* stream) {
  if (nx < 3 || ny < 3) return WSR_ERR_ARG;
  if (ws_bytes(nx, ny) > (size_t)WSR_NOALLOC_SCRATCH_BYTES) return WSR_ERR_SCRATCH_LIMIT;
  if (method < WSR_METHOD_JS || method > WSR_METHOD_SR_BF16) return WSR_ERR_ARG;
  if (bc != WSR_BC_TRANSMISSIVE && bc != WSR_BC_PERIODIC) return WSR_ERR_ARG;
  if (flux != WSR_FLUX_HLLC && flux != WSR_FLUX_FORCE) return WSR_ERR_ARG;
  if (rk < 1 || rk > 3 || !(dt > 0.0) || !(dx > 0.0) || !(dy > 0.0)) return WSR_ERR_ARG;
  if (!u_stage || !u0 || !u_out || misaligned(u_stage) || misaligned(u0) || misaligned(u_out)) return WSR_ERR_ARG;
  if (method != WSR_METHOD_JS && !closure_params) return WSR_ERR_NO_CLOSURE;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return WSR_ERR_CUDA;
  void* scratch = nullptr;
  int rc = noalloc_scratch_for(dev, &scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Ws2d w = carve(scratch, nx, ny);
  k_init_ctl<<<1, 1, 0, st>>>(w.ctl, w.fallbacks, w.counters, 0.0, 1.0, dt, dx, dy, 0.0, 0.0, 0, 0, 1);
  if (cudaGetLastError() != cudaSuccess) return WSR_ERR_CUDA;
  StageArgs a{u_stage, u0, u_out, nx, ny, bc, flux, opts, rk, dx, dy, gamma, 0.0};
  switch (method) {
    case WSR_METHOD_JS:
      return noalloc_launch<M_JS>(NoParams{}, a, w, st);
    case WSR_METHOD_SR_F64: {
      Mlp5d P;
      for (int k = 0; k < kParams5; ++k) P.p[k] = closure_params[k];
      return noalloc_launch<M_SR64>(P, a, w, st);
    }
    case WSR_METHOD_SR_F32: {
      Mlp5f P;
      for (int k = 0; k < kParams5; ++k) P.p[k] = static_cast<float>(closure_params[k]);
      P.duplicate();
      return noalloc_launch<M_SR32>(P, a, w, st);
    }
    default: {
      Mlp5f P;
      for (int k = 0; k < kParams5; ++k)
        P.p[k] = __bfloat162float(__float2bfloat16_rn(static_cast<float>(closure_params[k])));
      P.duplicate();
      return noalloc_launch<M_SRBF16>(P, a, w, st);
    }
  }
}
