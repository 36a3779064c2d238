// BF16 closure MLP on the tensor cores: the closure of 32 queued stencils at once, per warp.
//
// The BF16 closure (BF16 inputs, parameters and activations, FP32 accumulation) is an exact fit for the warp
// tensor-core instruction mma.sync.m16n8k16 .bf16 x .bf16 -> .f32: a layer of the MLP 5->10->6->6->3 is
// Z = X W + b with X the [rows x inputs] activations and W the [inputs x outputs] weights. One warp holds 32
// queued stencils; their direct and reflected inputs are 64 rows, four 16-row tiles (tiles 0, 1: direct rows of
// stencils 0..15, 16..31; tiles 2, 3: the reflected rows of the same stencils). Inputs are padded to K = 16 and
// outputs to N = 16 (first layer) or 8 (the others) with zero weights and biases.
//
// Fragment layouts (PTX ISA, mma.m16n8k16 with 16-bit operands; g = lane / 4, q = lane % 4):
//   A (16 x 16, row): {a0a1, a2a3, a4a5, a6a7} = (row g, cols 2q, 2q+1), (row g+8, cols 2q, 2q+1),
//                     (row g, cols 8+2q, 9+2q), (row g+8, cols 8+2q, 9+2q)
//   B (16 x 8, col):  {b0b1, b2b3} = (rows 2q, 2q+1; col g), (rows 8+2q, 9+2q; col g)
//   C/D (16 x 8):     {c0, c1, c2, c3} = (row g, cols 2q, 2q+1), (row g+8, cols 2q, 2q+1)
// A layer's output fragment for output columns 0..15 (two 8-column tiles), after the activation and the
// rounding to bfloat16, IS the next layer's A fragment register for register, so the four layers chain inside
// each lane without data exchange. Only the inputs (shuffled from the lanes that formed the features) and the
// three outputs per row (gathered across the four lanes of a quad, then handed back to the lanes that own the
// stencils) cross lanes.
//
// Same arithmetic as mlp_pair<float, true> up to the order of the FP32 accumulation inside the tensor core.
#pragma once
#include <cuda_runtime.h>

#include "closure.cuh"

namespace wsr {

// bfloat16 pair with `lo` in the low half (the lower column of a fragment register). The values are already
// representable in bfloat16, so the conversion is exact.
__device__ __forceinline__ unsigned bf16pair(float lo, float hi) {
  unsigned r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

__device__ __forceinline__ void mma_bf16(const unsigned a[4], unsigned b0, unsigned b1, float c0, float c1, float c2,
                                         float c3, float d[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%10, %11, %12, %13};"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(c0), "f"(c1), "f"(c2), "f"(c3));
}

// Per-lane weight and bias fragments of the four layers, formed once per block from the (bfloat16-rounded)
// packed parameters.
struct MmaW5 {
  unsigned w1[2][2], w2[2], w3[2], w4[2];  // [n tile][register] for the first layer
  float b1[2][2], b2[2], b3[2], b4[2];     // bias of output columns 2q, 2q+1 (of each n tile)
};

__device__ __forceinline__ MmaW5 mma_weights(const float* __restrict__ P, int lane) {
  const int g = lane >> 2, q = lane & 3;
  auto w = [&](int base, int ni, int no, int k, int n) -> float {
    return (k < ni && n < no) ? P[base + k * no + n] : 0.0f;
  };
  auto bias = [&](int base, int no, int n) -> float { return n < no ? P[base + n] : 0.0f; };
  MmaW5 m;
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    const int n = 8 * nt + g;
    m.w1[nt][0] = bf16pair(w(kW1, 5, 10, 2 * q, n), w(kW1, 5, 10, 2 * q + 1, n));
    m.w1[nt][1] = bf16pair(w(kW1, 5, 10, 8 + 2 * q, n), w(kW1, 5, 10, 9 + 2 * q, n));
    m.b1[nt][0] = bias(kB1, 10, 8 * nt + 2 * q);
    m.b1[nt][1] = bias(kB1, 10, 8 * nt + 2 * q + 1);
  }
  m.w2[0] = bf16pair(w(kW2, 10, 6, 2 * q, g), w(kW2, 10, 6, 2 * q + 1, g));
  m.w2[1] = bf16pair(w(kW2, 10, 6, 8 + 2 * q, g), w(kW2, 10, 6, 9 + 2 * q, g));
  m.w3[0] = bf16pair(w(kW3, 6, 6, 2 * q, g), w(kW3, 6, 6, 2 * q + 1, g));
  m.w3[1] = 0u;
  m.w4[0] = bf16pair(w(kW4, 6, 3, 2 * q, g), w(kW4, 6, 3, 2 * q + 1, g));
  m.w4[1] = 0u;
  m.b2[0] = bias(kB2, 6, 2 * q);
  m.b2[1] = bias(kB2, 6, 2 * q + 1);
  m.b3[0] = bias(kB3, 6, 2 * q);
  m.b3[1] = bias(kB3, 6, 2 * q + 1);
  m.b4[0] = bias(kB4, 3, 2 * q);
  m.b4[1] = bias(kB4, 3, 2 * q + 1);
  return m;
}

__device__ __forceinline__ float swish_bf16(float z) { return bf16r(swish<float>(z)); }

// Softmax of 6 tanh(z / 6) over three outputs (mlp_pair's head).
__device__ __forceinline__ void ratio_head(float z0, float z1, float z2, float r[3]) {
  const float b0 = 6.0f * tanh_t(div6(z0)), b1 = 6.0f * tanh_t(div6(z1)), b2 = 6.0f * tanh_t(div6(z2));
  float m = b0 > b1 ? b0 : b1;
  m = m > b2 ? m : b2;
  const float e0 = exp_t(b0 - m), e1 = exp_t(b1 - m), e2 = exp_t(b2 - m);
  const float inv = rcp_t(e0 + e1 + e2);
  r[0] = e0 * inv;
  r[1] = e1 * inv;
  r[2] = e2 * inv;
}

// The BF16 closure of the warp's 32 stencils. x: this lane's bfloat16-rounded features (zeros for a lane
// without a stencil). Every lane of the warp must call it (it synchronises the warp). Returns this lane's
// reflection-averaged ratios' reciprocal scaled betas, as closure_from_features<M_SRBF16> does.
__device__ __forceinline__ void closure_bf16_mma(const MmaW5& W, const float x[5], double& a0, double& a1,
                                                 double& a2) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  // feature pairs of this lane's stencil: direct (x0 x1 | x2 x3 | x4 0) and reflected (x2 x1 | x0 x3 | x4 0)
  const unsigned dir[3] = {bf16pair(x[0], x[1]), bf16pair(x[2], x[3]), bf16pair(x[4], 0.0f)};
  const unsigned ref[3] = {bf16pair(x[2], x[1]), bf16pair(x[0], x[3]), dir[2]};
  float z[4][4];  // layer-4 outputs of tile mt: (row g: cols 2q, 2q+1), (row g+8: cols 2q, 2q+1)
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int h = mt & 1, o = mt >> 1;
    unsigned a[4];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int src = 16 * h + g + 8 * r;
      const unsigned p0 = __shfl_sync(full, o ? ref[0] : dir[0], src);
      const unsigned p1 = __shfl_sync(full, o ? ref[1] : dir[1], src);
      const unsigned p2 = __shfl_sync(full, o ? ref[2] : dir[2], src);
      a[r] = q == 0 ? p0 : (q == 1 ? p1 : (q == 2 ? p2 : 0u));  // input columns 2q, 2q+1 (>= 5 are zero)
    }
    a[2] = a[3] = 0u;  // input columns 8..15
    // layer 1: 5 -> 10, two 8-column tiles
    float d0[4], d1[4];
    mma_bf16(a, W.w1[0][0], W.w1[0][1], W.b1[0][0], W.b1[0][1], W.b1[0][0], W.b1[0][1], d0);
    mma_bf16(a, W.w1[1][0], W.w1[1][1], W.b1[1][0], W.b1[1][1], W.b1[1][0], W.b1[1][1], d1);
    a[0] = bf16pair(swish_bf16(d0[0]), swish_bf16(d0[1]));
    a[1] = bf16pair(swish_bf16(d0[2]), swish_bf16(d0[3]));
    a[2] = bf16pair(swish_bf16(d1[0]), swish_bf16(d1[1]));
    a[3] = bf16pair(swish_bf16(d1[2]), swish_bf16(d1[3]));
    // layer 2: 10 -> 6
    mma_bf16(a, W.w2[0], W.w2[1], W.b2[0], W.b2[1], W.b2[0], W.b2[1], d0);
    a[0] = bf16pair(swish_bf16(d0[0]), swish_bf16(d0[1]));
    a[1] = bf16pair(swish_bf16(d0[2]), swish_bf16(d0[3]));
    a[2] = a[3] = 0u;
    // layer 3: 6 -> 6
    mma_bf16(a, W.w3[0], W.w3[1], W.b3[0], W.b3[1], W.b3[0], W.b3[1], d0);
    a[0] = bf16pair(swish_bf16(d0[0]), swish_bf16(d0[1]));
    a[1] = bf16pair(swish_bf16(d0[2]), swish_bf16(d0[3]));
    // layer 4: 6 -> 3 (raw outputs)
    mma_bf16(a, W.w4[0], W.w4[1], W.b4[0], W.b4[1], W.b4[0], W.b4[1], z[mt]);
  }
  // the heads: lane q of a quad takes the two rows of tile q (outputs 0, 1 from quad lane 0, output 2 from
  // quad lane 1), so each lane evaluates two heads, as one thread of the scalar closure does
  float zz[2][3];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const float u0 = __shfl_sync(full, z[mt][0], 4 * g), u1 = __shfl_sync(full, z[mt][1], 4 * g);
    const float u2 = __shfl_sync(full, z[mt][0], 4 * g + 1);
    const float v0 = __shfl_sync(full, z[mt][2], 4 * g), v1 = __shfl_sync(full, z[mt][3], 4 * g);
    const float v2 = __shfl_sync(full, z[mt][2], 4 * g + 1);
    if (q == mt) {
      zz[0][0] = u0, zz[0][1] = u1, zz[0][2] = u2;
      zz[1][0] = v0, zz[1][1] = v1, zz[1][2] = v2;
    }
  }
  float rat[2][3];  // lane (g, q): ratios of orientation q >> 1 of stencils 16 (q & 1) + g + 8 r
  ratio_head(zz[0][0], zz[0][1], zz[0][2], rat[0]);
  ratio_head(zz[1][0], zz[1][1], zz[1][2], rat[1]);
  // stencil s = 16 h + 8 r + g' (lane s): direct ratios in lane 4 g' + h, reflected in lane 4 g' + h + 2
  const int gs = lane & 7, h = lane >> 4, r = (lane >> 3) & 1;
  float ra[3], rb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float d_r0 = __shfl_sync(full, rat[0][k], 4 * gs + h), d_r1 = __shfl_sync(full, rat[1][k], 4 * gs + h);
    const float f_r0 = __shfl_sync(full, rat[0][k], 4 * gs + h + 2), f_r1 = __shfl_sync(full, rat[1][k], 4 * gs + h + 2);
    ra[k] = r ? d_r1 : d_r0;
    rb[k] = r ? f_r1 : f_r0;
  }
  const double r0 = 0.5 * ((double)ra[0] + (double)rb[2]);
  const double r1 = 0.5 * ((double)ra[1] + (double)rb[1]);
  const double r2 = 0.5 * ((double)ra[2] + (double)rb[0]);
  a0 = rcp64(3.0 * r0 + 1.0e-12);
  a1 = rcp64(3.0 * r1 + 1.0e-12);
  a2 = rcp64(3.0 * r2 + 1.0e-12);
}

}  // namespace wsr
