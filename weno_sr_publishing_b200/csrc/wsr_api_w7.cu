// extern "C" entry points of libwsr.so for the 2D WENO7 path (declared in include/wsr.h).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/wsr.h"
#include "euler2d.cuh"
#include "euler2d_w7.cuh"
#include "wsr_ctx.cuh"

using namespace wsr;
using namespace wsr_detail;

// ---------------------------------------------------------------------------------------------
// 2D Euler WENO7 (JS, Z, SR-FP64) with Shu RK4 (weno7_point_rk4_shu/point_rk4.py, weno7_point_rk4_z.py,
// teacherfree_lab_weno7_rk4_distance_balanced_fast/warp_sod/point_rk4_mlp.py).
// ---------------------------------------------------------------------------------------------
namespace {

struct Ws7 {
  StepCtl* ctl;
  double* dts;                     // ring of kDtsRing
  unsigned long long* counters;    // SR closure evaluations: normal x, normal y, flux x, flux y; [4] JS fallbacks
  double *xl, *xr, *yl, *yr, *fx, *fy;
  double *u1, *u2, *u3;
  double* rhs[6];  // rhs0, rhs_t0, rhs1, rhs_t1, rhs2, rhs3 (interior)
};

size_t ws7_bytes(int nx, int ny) {
  const size_t np = (size_t)(nx + 8) * (ny + 8), ni = (size_t)nx * ny;
  return align_up(sizeof(StepCtl)) + align_up(kDtsRing * sizeof(double)) + align_up(8 * sizeof(unsigned long long)) +
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
  w.counters = reinterpret_cast<unsigned long long*>(take(align_up(8 * sizeof(unsigned long long))));
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
                   int bc, int reverse, int opts, const Ws7& w, cudaStream_t st) {
  const Gas gas = make_gas(g);
  const Mlp7d& P = ctx->q64;
  w7::k7s_normal<1><<<dim3((nx + 1 + 127) / 128, ny + 7), 128, 0, st>>>(src, w.xl, w.xr, nx, ny, bc, gas, w.ctl,
                                                                       w.counters + 0, opts, w.counters + 4, P);
  WSR_LAUNCHED(ctx, "k7s_normal<x>");
  w7::k7s_normal<2><<<dim3((nx + 7 + 31) / 32, (ny + 1 + 3) / 4), 128, 0, st>>>(src, w.yl, w.yr, nx, ny, bc, gas,
                                                                               w.ctl, w.counters + 1, opts,
                                                                               w.counters + 4, P);
  WSR_LAUNCHED(ctx, "k7s_normal<y>");
  w7::k7s_flux<1><<<dim3((nx + 1 + 31) / 32, (ny + 3) / 4), 128, 0, st>>>(w.xl, w.xr, w.fx, nx, ny, gas, reverse,
                                                                         w.ctl, w.counters + 2, opts, w.counters + 4,
                                                                         P);
  WSR_LAUNCHED(ctx, "k7s_flux<x>");
  w7::k7s_flux<2><<<dim3((nx + 127) / 128, ny + 1), 128, 0, st>>>(w.yl, w.yr, w.fy, nx, ny, gas, reverse, w.ctl,
                                                                 w.counters + 3, opts, w.counters + 4, P);
  WSR_LAUNCHED(ctx, "k7s_flux<y>");
  w7::k7_rhs<<<dim3((nx + 255) / 256, ny), 256, 0, st>>>(w.fx, w.fy, rhs, nx, ny, 1.0 / dx, 1.0 / dy, w.ctl);
  WSR_LAUNCHED(ctx, "k7_rhs");
  return WSR_OK;
}

int launch_rhs7(wsr_ctx* ctx, const double* src, double* rhs, int nx, int ny, double dx, double dy, double g, int bc,
                int reverse, int method, int opts, const Ws7& w, cudaStream_t st) {
  if (method == WSR_METHOD_SR_F64) return launch_rhs7_sr(ctx, src, rhs, nx, ny, dx, dy, g, bc, reverse, opts, w, st);
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
int shu_step7(wsr_ctx* ctx, double* u, int nx, int ny, double dx, double dy, double g, int bc, int method, int opts,
              const Ws7& w, cudaStream_t st) {
  int rc;
  double* const* R = w.rhs;
  w7::ShuArgs a{u, w.u1, w.u2, w.u3, R[0], R[1], R[2], R[3], R[4], R[5], nullptr};
  if ((rc = launch_rhs7(ctx, u, R[0], nx, ny, dx, dy, g, bc, 0, method, opts, w, st))) return rc;
  a.out = w.u1;
  if ((rc = launch_shu7<1>(ctx, a, nx, ny, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, u, R[1], nx, ny, dx, dy, g, bc, 1, method, opts, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u1, R[2], nx, ny, dx, dy, g, bc, 0, method, opts, w, st))) return rc;
  a.out = w.u2;
  if ((rc = launch_shu7<2>(ctx, a, nx, ny, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u1, R[3], nx, ny, dx, dy, g, bc, 1, method, opts, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u2, R[4], nx, ny, dx, dy, g, bc, 0, method, opts, w, st))) return rc;
  a.out = w.u3;
  if ((rc = launch_shu7<3>(ctx, a, nx, ny, w, st))) return rc;
  if ((rc = launch_rhs7(ctx, w.u3, R[5], nx, ny, dx, dy, g, bc, 0, method, opts, w, st))) return rc;
  a.out = u;
  return launch_shu7<4>(ctx, a, nx, ny, w, st);
}

__global__ void k7_init(StepCtl* ctl, unsigned long long* counters, double t_start, double t_end, double cfl,
                        double hmin, int max_steps) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < 8; ++k) counters[k] = 0ull;
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
                                  double gamma, int bc, int method, int reverse, int opts, void* workspace,
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
  return launch_rhs7(ctx, u, rhs, nx, ny, dx, dy, gamma, bc, reverse != 0, method, opts, w, st);
}

extern "C" int wsr_euler2d_w7_run(wsr_ctx* ctx, double* u, int nx, int ny, double dx, double dy, double gamma,
                                  double cfl, double t_start, double t_end, int bc, int method, int opts, int max_steps,
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
      if ((rc = shu_step7(ctx, u, nx, ny, dx, dy, gamma, bc, method, opts, w, st))) return rc;
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
  WSR_CUDA(ctx, cudaMemcpy(out_host, w.counters, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
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
