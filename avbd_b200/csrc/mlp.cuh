// Tensor-core inference of the learned warm-start network (20 -> 64 -> 64
// -> 4, SiLU): BF16 operands, FP32 accumulation, one warp per 16-contact
// tile.  Shared by the solve kernels (the warm start runs inside the
// prelude phase) and the stand-alone avbd_mlp_infer entry point.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace avbd {
namespace {

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);  // .x (low half) = lo
  return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// Copies the packed block into shared memory (whole block participates).
__device__ __forceinline__ void stage_weights(const float* __restrict__ w, float* sw) {
  for (int k = threadIdx.x; k < AVBD_MLP_FLOATS; k += blockDim.x) sw[k] = w[k];
  __syncthreads();
}

// Forward pass of one 16-row tile by one warp.  `feat` points at row 0 of
// the tile (MLP_IN raw floats per row), `rows` valid rows (1..16).  On
// return lanes with (lane & 3) < 2 hold the denormalised outputs of rows
// g = lane >> 2 and g + 8 at columns 2t, 2t+1 (t = lane & 3): y[0..1] for
// row g, y[2..3] for row g + 8.
__device__ __forceinline__ void mlp_tile(const float* sw, const float* __restrict__ feat, int rows, float (&y)[4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t* W1 = reinterpret_cast<const uint32_t*>(sw + MLPO_W1);
  const uint32_t* W2 = reinterpret_cast<const uint32_t*>(sw + MLPO_W2);
  const uint32_t* W3 = reinterpret_cast<const uint32_t*>(sw + MLPO_W3);
  // Layer-1 A fragments: rows g and g+8, columns {2t, 2t+1, 2t+8, 2t+9} of
  // both 16-wide k-steps; normalised, zero beyond MLP_IN and beyond `rows`.
  uint32_t a[2][4];
#pragma unroll
  for (int kk = 0; kk < 2; ++kk) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {      // h: column half (+0 / +8)
#pragma unroll
      for (int r = 0; r < 2; ++r) {    // r: row g / g+8
        int row = g + 8 * r;
        int col = 16 * kk + 8 * h + 2 * t;
        float v0 = 0.0f, v1 = 0.0f;
        if (row < rows) {
          if (col < MLP_IN) v0 = (feat[row * MLP_IN + col] - sw[MLPO_FMEAN + col]) * sw[MLPO_FISTD + col];
          if (col + 1 < MLP_IN)
            v1 = (feat[row * MLP_IN + col + 1] - sw[MLPO_FMEAN + col + 1]) * sw[MLPO_FISTD + col + 1];
        }
        a[kk][2 * h + r] = bf16x2(v0, v1);
      }
    }
  }
  // Layer 1: 8 n-tiles of 8 hidden units.
  float h1[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float b0 = sw[MLPO_B1 + 8 * j + 2 * t], b1 = sw[MLPO_B1 + 8 * j + 2 * t + 1];
    h1[j][0] = b0; h1[j][1] = b1; h1[j][2] = b0; h1[j][3] = b1;
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
      const uint32_t* wr = W1 + (8 * j + g) * 16 + 8 * kk + t;
      mma_bf16(h1[j], a[kk][0], a[kk][1], a[kk][2], a[kk][3], wr[0], wr[4]);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) h1[j][e] = silu(h1[j][e]);
  }
  // Layer 2: the accumulator tiles 2kk, 2kk+1 are the A fragment of k-step kk.
  float h2[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float b0 = sw[MLPO_B2 + 8 * j + 2 * t], b1 = sw[MLPO_B2 + 8 * j + 2 * t + 1];
    h2[j][0] = b0; h2[j][1] = b1; h2[j][2] = b0; h2[j][3] = b1;
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t a0 = bf16x2(h1[2 * kk][0], h1[2 * kk][1]), a1 = bf16x2(h1[2 * kk][2], h1[2 * kk][3]);
    uint32_t a2 = bf16x2(h1[2 * kk + 1][0], h1[2 * kk + 1][1]), a3 = bf16x2(h1[2 * kk + 1][2], h1[2 * kk + 1][3]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t* wr = W2 + (8 * j + g) * 32 + 8 * kk + t;
      mma_bf16(h2[j], a0, a1, a2, a3, wr[0], wr[4]);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) h2[j][e] = silu(h2[j][e]);
  // Layer 3: one n-tile (outputs 0..3 used, 4..7 zero weights).
  float o[4];
  {
    float b0 = sw[MLPO_B3 + 2 * t], b1 = sw[MLPO_B3 + 2 * t + 1];
    o[0] = b0; o[1] = b1; o[2] = b0; o[3] = b1;
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t a0 = bf16x2(h2[2 * kk][0], h2[2 * kk][1]), a1 = bf16x2(h2[2 * kk][2], h2[2 * kk][3]);
    uint32_t a2 = bf16x2(h2[2 * kk + 1][0], h2[2 * kk + 1][1]), a3 = bf16x2(h2[2 * kk + 1][2], h2[2 * kk + 1][3]);
    const uint32_t* wr = W3 + g * 32 + 8 * kk + t;
    mma_bf16(o, a0, a1, a2, a3, wr[0], wr[4]);
  }
  int c = 2 * (t & 1);  // output columns of this lane (t = 0: 0,1; t = 1: 2,3)
  float m0 = sw[MLPO_OMEAN + c], m1 = sw[MLPO_OMEAN + c + 1];
  float s0 = sw[MLPO_OSTD + c], s1 = sw[MLPO_OSTD + c + 1];
  y[0] = o[0] * s0 + m0;
  y[1] = o[1] * s1 + m1;
  y[2] = o[2] * s0 + m0;
  y[3] = o[3] * s1 + m1;
}

// Gathers the 4 outputs of rows g and g+8 into lane 4g: out_g[4], out_g8[4].
__device__ __forceinline__ void gather_rows(const float (&y)[4], float (&og)[4], float (&og8)[4]) {
  float n0 = __shfl_down_sync(0xffffffffu, y[0], 1), n1 = __shfl_down_sync(0xffffffffu, y[1], 1);
  float n2 = __shfl_down_sync(0xffffffffu, y[2], 1), n3 = __shfl_down_sync(0xffffffffu, y[3], 1);
  og[0] = y[0]; og[1] = y[1]; og[2] = n0; og[3] = n1;
  og8[0] = y[2]; og8[1] = y[3]; og8[2] = n2; og8[3] = n3;
}

// Targets -> warm-start state (forces scaled by zeta).  Returns false when
// the contact must keep the zero start: separated (depth <= 0), non-finite,
// or a predicted friction force outside the static cone
// (|lambda_t| > mu_s |lambda_n|).
__device__ __forceinline__ bool decode_start(const float (&y)[4], float depth, float mus, float zeta, float4& lam,
                                             float& kn) {
  float ln0 = -expm1f(fmaxf(y[0], 0.0f));
  float sc = fabsf(ln0) + 1.0f;
  float ln = zeta * ln0;
  float lt = zeta * (y[1] * sc), lb = zeta * (y[2] * sc);
  kn = fminf(fmaxf(expf(y[3]), PEN_MIN), PEN_MAX);
  lam = make_float4(ln, lt, lb, 0.0f);
  if (!(depth > 0.0f)) return false;
  if (!isfinite(ln) || !isfinite(lt) || !isfinite(lb) || !isfinite(kn)) return false;
  if (sqrtf(lt * lt + lb * lb) > mus * fabsf(ln)) return false;
  return true;
}

}  // namespace
}  // namespace avbd
