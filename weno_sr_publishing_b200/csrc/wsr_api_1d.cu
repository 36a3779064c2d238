// extern "C" entry points of libwsr.so for the batched 1D advection path and closure training
// (declared in include/wsr.h).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/wsr.h"
#include "adv1d.cuh"
#include "train1d.cuh"
#include "wsr_ctx.cuh"

using namespace wsr;
using namespace wsr_detail;

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
const ZEps& adv_params_of<5, M_Z>(const wsr_ctx*) {
  static const ZEps unused{};  // WENO-Z takes eps from each trajectory's dx
  return unused;
}
template <>
const ZEps& adv_params_of<7, M_Z>(const wsr_ctx*) {
  static const ZEps unused{};
  return unused;
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
    case WSR_METHOD_Z:
      return adv_launch<SCHEME, M_Z, INTEG>(ctx, a, st);
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
  if (method < WSR_METHOD_JS || method > WSR_METHOD_Z) return fail(ctx, WSR_ERR_ARG, "bad method %d", method);
  if (nmax < (scheme == 5 ? 5 : 7) || nmax > kAdvNmax)
    return fail(ctx, WSR_ERR_ARG, "nmax must be in [%d, %d] (got %d)", scheme == 5 ? 5 : 7, kAdvNmax, nmax);
  if (method != WSR_METHOD_JS && method != WSR_METHOD_Z && !(scheme == 5 ? ctx->have_closure : ctx->have_closure7))
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
