// The libwsr context (closure parameters, error text, profiling events) and the helpers that every
// translation unit of the library shares.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "../../include/wsr.h"
#include "closure.cuh"
#include "adv1d.cuh"

constexpr int kProfKinds = 6;  // normal x, normal y, flux x, flux y, update, control
constexpr int kProfEvents = 512;

struct wsr_host_pipe;  // copy streams and band events of wsr_euler2d_advance_host (wsr_api.cu)

struct wsr_ctx {
  int device;
  bool have_closure;
  wsr::Mlp5d p64;
  wsr::Mlp5f p32;
  wsr::Mlp5f pbf16;
  bool have_closure7;
  wsr::Mlp7d q64;
  wsr::Mlp7f q32;
  wsr::Mlp7f qbf16;
  char err[512];
  double* host_pinned;  // small pinned mailbox for control-block reads
  // per-kernel CUDA-event timing (off unless wsr_profile_enable)
  bool prof_on;
  bool prof_created;
  cudaEvent_t ev_a[kProfEvents], ev_b[kProfEvents];
  int ev_kind[kProfEvents];
  int n_ev;
  double prof_ms[kProfKinds];
  long long prof_count[kProfKinds];
  wsr_host_pipe* host;  // created by the first host-buffer call
};

namespace wsr_detail {

using namespace wsr;

inline int fail(wsr_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define WSR_CUDA(ctx, call)                                                                    \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail(ctx, WSR_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

#define WSR_LAUNCHED(ctx, what)                                                                \
  do {                                                                                         \
    cudaError_t e_ = cudaGetLastError();                                                       \
    if (e_ != cudaSuccess) return fail(ctx, WSR_ERR_CUDA, "launch %s: %s", what, cudaGetErrorString(e_)); \
  } while (0)

constexpr size_t kAlign = 256;
constexpr int kDtsRing = 64;  // dt records kept on the device between host polls

inline size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// bytes of an array of n cells of 4 FP64 values, padded to the workspace alignment
inline size_t cells_bytes(size_t n) { return align_up(n * 4 * sizeof(double)); }

inline bool misaligned(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) != 0; }


template <int M>
const typename ClosureParams<M>::type& params_of(const wsr_ctx* ctx);
template <>
inline const NoParams& params_of<M_JS>(const wsr_ctx*) {
  static const NoParams np{};
  return np;
}
template <>
inline const Mlp5d& params_of<M_SR64>(const wsr_ctx* ctx) {
  return ctx->p64;
}
template <>
inline const Mlp5f& params_of<M_SR32>(const wsr_ctx* ctx) {
  return ctx->p32;
}
template <>
inline const Mlp5f& params_of<M_SRBF16>(const wsr_ctx* ctx) {
  return ctx->pbf16;
}
template <>
inline const Mlp5f& params_of<M_SRBF16_TC>(const wsr_ctx* ctx) {
  return ctx->pbf16;
}

}  // namespace wsr_detail
