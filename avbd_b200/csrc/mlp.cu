// Learned warm start for new contacts: a 20 -> 64 -> 64 -> 4 SiLU network
// that predicts the cached state (lambda_n, lambda_t1, lambda_t2, k_n) a
// contact would have had, in place of the cache-miss defaults of the
// emission (kernels_6dof.py:2864-2879).  No counterpart in the reference.
//
//  * Inference (mlp.cuh; the solver runs it inside the prelude phase of
//    the solve kernel): one warp per 16-contact tile on the tensor cores,
//    mma.sync.m16n8k16 with BF16 operands and FP32 accumulation; the packed
//    weights are staged once per block in shared memory; hidden activations
//    stay in registers (an m16n8 accumulator tile is, lane for lane, the A
//    fragment of the next layer's m16n8k16).  avbd_mlp_infer runs the same
//    tile code stand-alone.
//  * Training: FP32 forward/backward over 32-sample tiles in shared memory,
//    per-block gradient partials in registers, a fixed-order reduction
//    across blocks (bit-reproducible), and a bias-corrected Adam step.
#include "kernels.cuh"
#include "mlp.cuh"

namespace avbd {

namespace {

constexpr int P_W1 = 0, P_B1 = 1280, P_W2 = 1344, P_B2 = 5440, P_W3 = 5504, P_B3 = 5760;
static_assert(P_B3 + 4 == AVBD_MLP_PARAMS, "master parameter count");

__global__ void __launch_bounds__(128) k_mlp_infer(const float* __restrict__ packed, const float* __restrict__ feat,
                                                   int n, float* __restrict__ out) {
  __shared__ float sw[AVBD_MLP_FLOATS];
  stage_weights(packed, sw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int tile = blockIdx.x * nw + warp; tile * 16 < n; tile += gridDim.x * nw) {
    int r0 = tile * 16, rows = min(16, n - r0);
    float y[4], og[4], og8[4];
    mlp_tile(sw, feat + (size_t)r0 * MLP_IN, rows, y);
    gather_rows(y, og, og8);
    if ((lane & 3) == 0) {
      int g = lane >> 2;
      if (g < rows) *reinterpret_cast<float4*>(out + 4 * (size_t)(r0 + g)) = make_float4(og[0], og[1], og[2], og[3]);
      if (g + 8 < rows)
        *reinterpret_cast<float4*>(out + 4 * (size_t)(r0 + g + 8)) = make_float4(og8[0], og8[1], og8[2], og8[3]);
    }
  }
}

__global__ void k_mlp_pack(const float* __restrict__ th, const float* __restrict__ norm, float* __restrict__ pk) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= AVBD_MLP_FLOATS) return;
  float v = 0.0f;
  if (k < MLPO_FISTD) {
    v = k < MLP_IN ? norm[k] : 0.0f;
  } else if (k < MLPO_OMEAN) {
    int i = k - MLPO_FISTD;
    v = i < MLP_IN ? 1.0f / norm[MLP_IN + i] : 0.0f;
  } else if (k < MLPO_OSTD) {
    int i = k - MLPO_OMEAN;
    v = i < MLP_OUT ? norm[2 * MLP_IN + i] : (i == MLP_OUT ? norm[2 * MLP_IN + 2 * MLP_OUT] : 0.0f);
  } else if (k < MLPO_B1) {
    int i = k - MLPO_OSTD;
    v = i < MLP_OUT ? norm[2 * MLP_IN + MLP_OUT + i] : 1.0f;
  } else if (k < MLPO_B2) {
    v = th[P_B1 + (k - MLPO_B1)];
  } else if (k < MLPO_B3) {
    v = th[P_B2 + (k - MLPO_B2)];
  } else if (k < MLPO_W1) {
    int i = k - MLPO_B3;
    v = i < MLP_OUT ? th[P_B3 + i] : 0.0f;
  } else {
    // bf16 pairs: row-major [rows][cols], element 2p in the low half.
    float lo = 0.0f, hi = 0.0f;
    if (k < MLPO_W2) {
      int p = k - MLPO_W1, r = p / 16, c = 2 * (p % 16);
      if (c < MLP_IN) lo = th[P_W1 + r * MLP_IN + c];
      if (c + 1 < MLP_IN) hi = th[P_W1 + r * MLP_IN + c + 1];
    } else if (k < MLPO_W3) {
      int p = k - MLPO_W2, r = p / 32, c = 2 * (p % 32);
      lo = th[P_W2 + r * MLP_H + c];
      hi = th[P_W2 + r * MLP_H + c + 1];
    } else {
      int p = k - MLPO_W3, r = p / 32, c = 2 * (p % 32);
      if (r < MLP_OUT) {
        lo = th[P_W3 + r * MLP_H + c];
        hi = th[P_W3 + r * MLP_H + c + 1];
      }
    }
    uint32_t u = 0;
    {
      __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
      u = *reinterpret_cast<uint32_t*>(&h);
    }
    v = __uint_as_float(u);
  }
  pk[k] = v;
}

// ---------------------------------------------------------------------------
// Training (FP32).
// ---------------------------------------------------------------------------
constexpr int TS = 32;          // samples per shared-memory tile
constexpr int TRAIN_THREADS = 256;
constexpr int W1S = 21, W2S = 65, W3S = 65;  // padded shared-memory row strides
constexpr int GRAD_STRIDE = AVBD_MLP_PARAMS + 4;  // partial gradient + loss, per block

struct TrainSmem {
  float w1[MLP_H * W1S], b1[MLP_H], w2[MLP_H * W2S], b2[MLP_H], w3[MLP_OUT * W3S], b3[MLP_OUT];
  float x[TS][MLP_IN], y[TS][MLP_OUT];
  float z1[TS][MLP_H], h1[TS][MLP_H], z2[TS][MLP_H], h2[TS][MLP_H];
  float d3[TS][MLP_OUT], d2[TS][MLP_H], d1[TS][MLP_H];
  float loss[TRAIN_THREADS / 32];
};

__device__ __forceinline__ float dsilu(float z) {
  float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Partial loss and gradient of samples [s0, s1) (pre-scaled by 1/n_total).
__global__ void __launch_bounds__(TRAIN_THREADS) k_mlp_grad(const float* __restrict__ th, const float* __restrict__ X,
                                                            const float* __restrict__ Y, int n, int chunk,
                                                            float* __restrict__ part) {
  extern __shared__ float smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
  const int tid = threadIdx.x;
  for (int k = tid; k < MLP_H * MLP_IN; k += TRAIN_THREADS) S.w1[(k / MLP_IN) * W1S + k % MLP_IN] = th[P_W1 + k];
  for (int k = tid; k < MLP_H * MLP_H; k += TRAIN_THREADS) S.w2[(k / MLP_H) * W2S + k % MLP_H] = th[P_W2 + k];
  for (int k = tid; k < MLP_OUT * MLP_H; k += TRAIN_THREADS) S.w3[(k / MLP_H) * W3S + k % MLP_H] = th[P_W3 + k];
  if (tid < MLP_H) {
    S.b1[tid] = th[P_B1 + tid];
    S.b2[tid] = th[P_B2 + tid];
  }
  if (tid < MLP_OUT) S.b3[tid] = th[P_B3 + tid];
  const float inv_n = 1.0f / (float)n;
  // Register accumulators.  dW2: row j2 = tid >> 2, columns (tid & 3) + 4m.
  float gw2[16], gw1[5], gw3 = 0.0f, gb = 0.0f, lsum = 0.0f;
#pragma unroll
  for (int m = 0; m < 16; ++m) gw2[m] = 0.0f;
#pragma unroll
  for (int m = 0; m < 5; ++m) gw1[m] = 0.0f;
  const int j = tid & 63, sg = tid >> 6;  // hidden unit, sample group (8 samples each)
  const int s_begin = blockIdx.x * chunk, s_end = min(n, s_begin + chunk);
  __syncthreads();
  for (int t0 = s_begin; t0 < s_end; t0 += TS) {
    int ns = min(TS, s_end - t0);
    for (int k = tid; k < TS * MLP_IN; k += TRAIN_THREADS) {
      int s = k / MLP_IN;
      S.x[s][k % MLP_IN] = s < ns ? X[(size_t)(t0 + s) * MLP_IN + k % MLP_IN] : 0.0f;
    }
    for (int k = tid; k < TS * MLP_OUT; k += TRAIN_THREADS) {
      int s = k / MLP_OUT;
      S.y[s][k % MLP_OUT] = s < ns ? Y[(size_t)(t0 + s) * MLP_OUT + k % MLP_OUT] : 0.0f;
    }
    __syncthreads();
    // forward: layer 1
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      int s = sg * 8 + q;
      float z = S.b1[j];
#pragma unroll
      for (int i = 0; i < MLP_IN; ++i) z += S.w1[j * W1S + i] * S.x[s][i];
      S.z1[s][j] = z;
      S.h1[s][j] = z / (1.0f + expf(-z));
    }
    __syncthreads();
    // layer 2
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      int s = sg * 8 + q;
      float z = S.b2[j];
#pragma unroll 16
      for (int k = 0; k < MLP_H; ++k) z += S.w2[j * W2S + k] * S.h1[s][k];
      S.z2[s][j] = z;
      S.h2[s][j] = z / (1.0f + expf(-z));
    }
    __syncthreads();
    // layer 3 + loss gradient (samples beyond ns contribute nothing)
    if (tid < TS * MLP_OUT) {
      int s = tid >> 2, o = tid & 3;
      float z = S.b3[o];
#pragma unroll 16
      for (int k = 0; k < MLP_H; ++k) z += S.w3[o * W3S + k] * S.h2[s][k];
      float e = s < ns ? z - S.y[s][o] : 0.0f;
      lsum += e * e;
      S.d3[s][o] = 2.0f * e * inv_n;
    }
    __syncthreads();
    // dW3, db3 (thread -> (o = tid >> 6, k = tid & 63))
    {
      int o = tid >> 6, k = tid & 63;
      float acc = 0.0f;
#pragma unroll 8
      for (int s = 0; s < TS; ++s) acc += S.d3[s][o] * S.h2[s][k];
      gw3 += acc;
    }
    // backprop into layer 2 pre-activations
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      int s = sg * 8 + q;
      float dh = 0.0f;
#pragma unroll
      for (int o = 0; o < MLP_OUT; ++o) dh += S.w3[o * W3S + j] * S.d3[s][o];
      S.d2[s][j] = dh * dsilu(S.z2[s][j]);
    }
    __syncthreads();
    // dW2 accumulation
    {
      int r = tid >> 2, c0 = tid & 3;
#pragma unroll 4
      for (int s = 0; s < TS; ++s) {
        float dv = S.d2[s][r];
#pragma unroll
        for (int m = 0; m < 16; ++m) gw2[m] += dv * S.h1[s][c0 + 4 * m];
      }
    }
    // backprop into layer 1 pre-activations
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      int s = sg * 8 + q;
      float dh = 0.0f;
#pragma unroll 16
      for (int k = 0; k < MLP_H; ++k) dh += S.w2[k * W2S + j] * S.d2[s][k];
      S.d1[s][j] = dh * dsilu(S.z1[s][j]);
    }
    __syncthreads();
    // dW1: entries tid + 256 m (m < 5) of the 64 x 20 matrix
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      int e = tid + TRAIN_THREADS * m, r = e / MLP_IN, c = e % MLP_IN;
      float acc = 0.0f;
#pragma unroll 8
      for (int s = 0; s < TS; ++s) acc += S.d1[s][r] * S.x[s][c];
      gw1[m] += acc;
    }
    // biases: threads 0..63 b1, 64..127 b2, 128..131 b3
    if (tid < 64) {
      float acc = 0.0f;
      for (int s = 0; s < TS; ++s) acc += S.d1[s][tid];
      gb += acc;
    } else if (tid < 128) {
      float acc = 0.0f;
      for (int s = 0; s < TS; ++s) acc += S.d2[s][tid - 64];
      gb += acc;
    } else if (tid < 132) {
      float acc = 0.0f;
      for (int s = 0; s < TS; ++s) acc += S.d3[s][tid - 128];
      gb += acc;
    }
    __syncthreads();
  }
  float* P = part + (size_t)blockIdx.x * GRAD_STRIDE;
#pragma unroll
  for (int m = 0; m < 16; ++m) P[P_W2 + (tid >> 2) * MLP_H + (tid & 3) + 4 * m] = gw2[m];
#pragma unroll
  for (int m = 0; m < 5; ++m) P[P_W1 + tid + TRAIN_THREADS * m] = gw1[m];
  P[P_W3 + tid] = gw3;
  if (tid < 64) P[P_B1 + tid] = gb;
  else if (tid < 128) P[P_B2 + tid - 64] = gb;
  else if (tid < 132) P[P_B3 + tid - 128] = gb;
  // loss: fixed-order block sum
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((tid & 31) == 0) S.loss[tid >> 5] = lsum;
  __syncthreads();
  if (tid == 0) {
    float l = 0.0f;
    for (int w = 0; w < TRAIN_THREADS / 32; ++w) l += S.loss[w];
    P[AVBD_MLP_PARAMS] = l * inv_n;
  }
}

// grad[p] = sum over blocks b (in order) of part[b][p]; p = AVBD_MLP_PARAMS
// is the loss.
__global__ void k_mlp_reduce(const float* __restrict__ part, int nblk, float* __restrict__ grad,
                             float* __restrict__ loss) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > AVBD_MLP_PARAMS) return;
  float s = 0.0f;
  for (int b = 0; b < nblk; ++b) s += part[(size_t)b * GRAD_STRIDE + p];
  if (p < AVBD_MLP_PARAMS) grad[p] = s;
  else if (loss) *loss = s;
}

__global__ void k_mlp_adam(float* __restrict__ th, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= AVBD_MLP_PARAMS) return;
  float gp = g[p];
  float mp = b1 * m[p] + (1.0f - b1) * gp;
  float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  th[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

int grad_blocks(int n) {
  int nb = (n + 4 * TS - 1) / (4 * TS);  // at least 4 tiles per block
  return nb < 1 ? 1 : (nb > 296 ? 296 : nb);
}

}  // namespace


}  // namespace avbd

using namespace avbd;

namespace avbd {
void set_error_text(const char* what, cudaError_t e);
}

static int mlp_status(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return AVBD_OK;
  avbd::set_error_text(what, e);
  return AVBD_E_CUDA;
}

extern "C" {

int avbd_mlp_pack(const float* theta, const float* norm, float* packed, void* stream) {
  if (!theta || !norm || !packed) {
    avbd::set_error_text("avbd_mlp_pack: null argument", cudaSuccess);
    return AVBD_E_INVALID;
  }
  k_mlp_pack<<<(AVBD_MLP_FLOATS + 255) / 256, 256, 0, (cudaStream_t)stream>>>(theta, norm, packed);
  return mlp_status("avbd_mlp_pack");
}

int avbd_mlp_infer(const float* packed, const float* feat, int n, float* out, void* stream) {
  if (n < 0 || (n > 0 && (!packed || !feat || !out))) {
    avbd::set_error_text("avbd_mlp_infer: bad arguments", cudaSuccess);
    return AVBD_E_INVALID;
  }
  if (n == 0) return AVBD_OK;
  int tiles = (n + 15) / 16;
  int nblk = (tiles + 3) / 4;
  if (nblk > 8 * 148) nblk = 8 * 148;
  k_mlp_infer<<<nblk, 128, 0, (cudaStream_t)stream>>>(packed, feat, n, out);
  return mlp_status("avbd_mlp_infer");
}

size_t avbd_mlp_scratch_bytes(int n) {
  if (n < 1) n = 1;
  return (size_t)grad_blocks(n) * GRAD_STRIDE * sizeof(float);
}

int avbd_mlp_loss_grad(const float* theta, const float* x, const float* y, int n, float* grad, float* loss,
                       void* scratch, size_t scratch_bytes, void* stream) {
  if (n < 1 || !theta || !x || !y || !grad || !scratch) {
    avbd::set_error_text("avbd_mlp_loss_grad: bad arguments", cudaSuccess);
    return AVBD_E_INVALID;
  }
  if (scratch_bytes < avbd_mlp_scratch_bytes(n)) {
    avbd::set_error_text("avbd_mlp_loss_grad: scratch smaller than avbd_mlp_scratch_bytes(n)", cudaSuccess);
    return AVBD_E_INVALID;
  }
  static bool attr_set = false;  // one opt-in per process is enough (same device image)
  size_t smem = sizeof(TrainSmem);
  if (!attr_set) {
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr_set = true;
  }
  int nblk = grad_blocks(n);
  int chunk = (n + nblk - 1) / nblk;
  cudaStream_t st = (cudaStream_t)stream;
  float* part = (float*)scratch;
  k_mlp_grad<<<nblk, TRAIN_THREADS, smem, st>>>(theta, x, y, n, chunk, part);
  k_mlp_reduce<<<(AVBD_MLP_PARAMS + 1 + 255) / 256, 256, 0, st>>>(part, nblk, grad, loss);
  return mlp_status("avbd_mlp_loss_grad");
}

int avbd_mlp_adam(float* theta, const float* grad, float* m, float* v, int t, float lr, float beta1, float beta2,
                  float eps, void* stream) {
  if (!theta || !grad || !m || !v || t < 1) {
    avbd::set_error_text("avbd_mlp_adam: bad arguments", cudaSuccess);
    return AVBD_E_INVALID;
  }
  float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
  k_mlp_adam<<<(AVBD_MLP_PARAMS + 255) / 256, 256, 0, (cudaStream_t)stream>>>(theta, grad, m, v, lr, beta1, beta2,
                                                                             eps, c1, c2);
  return mlp_status("avbd_mlp_adam");
}

}  // extern "C"
