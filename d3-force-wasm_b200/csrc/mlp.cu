// mlp.cu — the learned correction's network (no reference counterpart): a
// per-leaf MLP 12 -> 64 -> 64 -> 2 with GELU, BF16 weights and FP32
// accumulation, and its training (forward, backward and Adam) on the GPU.
//
// Parameters, one float vector (the FP32 master copy; every use rounds the
// weights to bf16, biases stay FP32), weights stored [out][in]:
//   W1 [64][12] | b1 [64] | W2 [64][64] | b2 [64] | W3 [2][64] | b3 [2]
//
// Training kernel (CUDA cores): a CTA of 128 threads takes tiles of 128
// samples, a thread per sample for the forward pass and the input gradients
// (activations in shared memory, unit-major with a padded stride so the
// threads' reads fall in distinct banks), then the weight gradients as
// sums over the tile's samples, a thread per weight row; a CTA keeps its
// gradient sums in shared memory over all its tiles and adds them to the
// global sums once. Loss: mean over samples of sum_o (y_o - t_o)^2.
// Inference (tcgen05, mlp_infer_tc): a CTA per 128 samples, the three layers
// as MMAs of M = 128 with the activations staged as bf16 in shared memory,
// GELU and the biases applied between them from the TMEM accumulators.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "mlp.cuh"
#include "tc.cuh"

namespace d3 {
namespace {

constexpr int TT = 128;       // samples per tile
constexpr int SP = TT + 1;    // padded stride of unit-major activation rows

__device__ __forceinline__ float bf(float w) { return __bfloat162float(__float2bfloat16(w)); }
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678f)) + z * 0.39894228f * expf(-0.5f * z * z);
}

struct TrainSmem {
  float w1[MLP_H][MLP_IN], w2[MLP_H][MLP_H], w3[MLP_OUT][MLP_H];  // bf16-rounded
  float b1[MLP_H], b2[MLP_H], b3[MLP_OUT];
  float x[MLP_IN][SP];
  float a1[MLP_H][SP], g1[MLP_H][SP];  // activation, gelu'(z); g reused for dz
  float a2[MLP_H][SP], g2[MLP_H][SP];
  float dy[MLP_OUT][SP];
  float gsum[MLP_PARAMS];  // this CTA's gradient sums
  float loss;
};

// Gradient of the loss over samples [0, n) (sum over samples of the per-
// sample loss, divided by `norm`), added into grad (zeroed by the caller);
// loss_sum gets the summed loss.
__global__ void __launch_bounds__(TT) k_mlp_grad(const float *x, const float *y, uint32_t n,
                                                 const float *params, float norm, float *grad,
                                                 float *loss_sum) {
  extern __shared__ float mlp_smem[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(mlp_smem);
  const int t = threadIdx.x;
  for (int k = t; k < MLP_H * MLP_IN; k += TT) (&S.w1[0][0])[k] = bf(params[P_W1 + k]);
  for (int k = t; k < MLP_H * MLP_H; k += TT) (&S.w2[0][0])[k] = bf(params[P_W2 + k]);
  for (int k = t; k < MLP_OUT * MLP_H; k += TT) (&S.w3[0][0])[k] = bf(params[P_W3 + k]);
  for (int k = t; k < MLP_H; k += TT) {
    S.b1[k] = params[P_B1 + k];
    S.b2[k] = params[P_B2 + k];
  }
  if (t < MLP_OUT) S.b3[t] = params[P_B3 + t];
  for (int k = t; k < MLP_PARAMS; k += TT) S.gsum[k] = 0;
  if (t == 0) S.loss = 0;
  __syncthreads();
  const float inv = 1.f / norm;
  float my_loss = 0;
  for (uint32_t base = blockIdx.x * TT; base < n; base += gridDim.x * TT) {
    const uint32_t i = base + t;
    const bool act = i < n;
    // forward, a thread per sample
    float xi[MLP_IN];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) {
      xi[k] = act ? x[(size_t)i * MLP_IN + k] : 0.f;
      S.x[k][t] = __bfloat162float(__float2bfloat16(xi[k]));
    }
    for (int j = 0; j < MLP_H; ++j) {
      float z = S.b1[j];
#pragma unroll
      for (int k = 0; k < MLP_IN; ++k) z += S.w1[j][k] * S.x[k][t];
      S.a1[j][t] = bf(gelu(z));
      S.g1[j][t] = gelu_d(z);
    }
    for (int j = 0; j < MLP_H; ++j) {
      float z = S.b2[j];
      for (int k = 0; k < MLP_H; ++k) z += S.w2[j][k] * S.a1[k][t];
      S.a2[j][t] = bf(gelu(z));
      S.g2[j][t] = gelu_d(z);
    }
    for (int o = 0; o < MLP_OUT; ++o) {
      float z = S.b3[o];
      for (int k = 0; k < MLP_H; ++k) z += S.w3[o][k] * S.a2[k][t];
      const float d = act ? z - y[(size_t)i * MLP_OUT + o] : 0.f;
      my_loss += d * d;
      S.dy[o][t] = 2.f * d * inv;
    }
    // input gradients: dz2 = (W3^T dy) gelu'(z2), dz1 = (W2^T dz2) gelu'(z1)
    for (int k = 0; k < MLP_H; ++k) {
      float s = 0;
      for (int o = 0; o < MLP_OUT; ++o) s += S.w3[o][k] * S.dy[o][t];
      S.g2[k][t] *= s;  // g2 now holds dz2
    }
    for (int k = 0; k < MLP_H; ++k) {
      float s = 0;
      for (int j = 0; j < MLP_H; ++j) s += S.w2[j][k] * S.g2[j][t];
      S.g1[k][t] *= s;  // g1 now holds dz1
    }
    __syncthreads();
    // weight gradients: sums over the tile's samples, a thread per row
    if (t < MLP_H) {
      const int j = t;
      float gb1 = 0, gw1[MLP_IN] = {};
      for (int s = 0; s < TT; ++s) {
        const float d = S.g1[j][s];
        gb1 += d;
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) gw1[k] += d * S.x[k][s];
      }
      S.gsum[P_B1 + j] += gb1;
#pragma unroll
      for (int k = 0; k < MLP_IN; ++k) S.gsum[P_W1 + j * MLP_IN + k] += gw1[k];
    } else {
      const int j = t - MLP_H;
      float gb2 = 0;
      for (int s = 0; s < TT; ++s) gb2 += S.g2[j][s];
      S.gsum[P_B2 + j] += gb2;
      for (int k0 = 0; k0 < MLP_H; k0 += 16) {
        float acc[16] = {};
        for (int s = 0; s < TT; ++s) {
          const float d = S.g2[j][s];
#pragma unroll
          for (int k = 0; k < 16; ++k) acc[k] += d * S.a1[k0 + k][s];
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) S.gsum[P_W2 + j * MLP_H + k0 + k] += acc[k];
      }
    }
    if (t < MLP_OUT * MLP_H) {
      const int o = t / MLP_H, k = t % MLP_H;
      float g = 0;
      for (int s = 0; s < TT; ++s) g += S.dy[o][s] * S.a2[k][s];
      S.gsum[P_W3 + o * MLP_H + k] += g;
    }
    if (t < MLP_OUT) {
      float g = 0;
      for (int s = 0; s < TT; ++s) g += S.dy[t][s];
      S.gsum[P_B3 + t] += g;
    }
    __syncthreads();
  }
  atomicAdd(&S.loss, my_loss);
  __syncthreads();
  for (int k = t; k < MLP_PARAMS; k += TT) atomicAdd(&grad[k], S.gsum[k]);
  if (t == 0) atomicAdd(loss_sum, S.loss);
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters.
__global__ void k_mlp_adam(float *params, float *m, float *v, const float *grad, float lr,
                           float b1, float b2, float eps, float c1, float c2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= MLP_PARAMS) return;
  const float g = grad[k];
  const float mk = b1 * m[k] + (1 - b1) * g;
  const float vk = b2 * v[k] + (1 - b2) * g * g;
  m[k] = mk;
  v[k] = vk;
  params[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// The forward pass on CUDA cores (a thread per sample): the check of the
// tensor-core inference.
__global__ void k_mlp_infer_cc(const float *x, uint32_t n, const float *params, float *y) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float xi[MLP_IN], h1[MLP_H], h2[MLP_H];
  for (int k = 0; k < MLP_IN; ++k) xi[k] = bf(x[(size_t)i * MLP_IN + k]);
  for (int j = 0; j < MLP_H; ++j) {
    float z = params[P_B1 + j];
    for (int k = 0; k < MLP_IN; ++k) z += bf(params[P_W1 + j * MLP_IN + k]) * xi[k];
    h1[j] = bf(gelu(z));
  }
  for (int j = 0; j < MLP_H; ++j) {
    float z = params[P_B2 + j];
    for (int k = 0; k < MLP_H; ++k) z += bf(params[P_W2 + j * MLP_H + k]) * h1[k];
    h2[j] = bf(gelu(z));
  }
  for (int o = 0; o < MLP_OUT; ++o) {
    float z = params[P_B3 + o];
    for (int k = 0; k < MLP_H; ++k) z += bf(params[P_W3 + o * MLP_H + k]) * h2[k];
    y[(size_t)i * MLP_OUT + o] = z;
  }
}

}  // namespace

// ---- inference on the tensor cores ---------------------------------------------------------

// Shared memory of k_mlp_infer_tc: the operand tiles (bf16, K-major, the
// tile layout of tc.cuh) and the barriers.
struct InferSmem {
  unsigned char x[TT * 16 * 2];          // A1: 128 x 16 (12 inputs, zero padded)
  unsigned char h[TT * MLP_H * 2];       // A2 / A3: 128 x 64
  unsigned char w1[MLP_H * 16 * 2];      // B1: 64 (out) x 16 (in)
  unsigned char w2[MLP_H * MLP_H * 2];   // B2: 64 x 64
  unsigned char w3[16 * MLP_H * 2];      // B3: 16 (2 outputs, zero padded) x 64
  float b1[MLP_H], b2[MLP_H], b3[MLP_OUT];
  uint64_t bar;
  uint32_t tmem, err;
};

__device__ __forceinline__ void put_bf16(unsigned char *tile, uint32_t rows, uint32_t r, uint32_t k,
                                         float v) {
  *reinterpret_cast<__nv_bfloat16 *>(tile + tc::tile_offset(r, k / 8, rows) + (k % 8) * 2) =
      __float2bfloat16(v);
}

// y[i] = MLP(x[i]) for the 128 samples of this CTA's tile. x: n x 12 FP32;
// per-sample hook: rows with row_ok false produce nothing.
__global__ void __launch_bounds__(TT) k_mlp_infer_tc(const float *x, uint32_t n,
                                                     const float *params, float *y,
                                                     uint32_t *err_flag) {
  extern __shared__ __align__(1024) unsigned char mlp_tc_smem[];
  InferSmem &S = *reinterpret_cast<InferSmem *>(mlp_tc_smem);
  const uint32_t t = threadIdx.x, warp = t >> 5;
  const uint32_t i = blockIdx.x * TT + t;
  // operands: this thread's input row, and a share of the weight tiles
  for (uint32_t k = 0; k < 16; ++k)
    put_bf16(S.x, TT, t, k, (i < n && k < (uint32_t)MLP_IN) ? x[(size_t)i * MLP_IN + k] : 0.f);
  for (uint32_t e = t; e < MLP_H * 16; e += TT) {
    const uint32_t o = e / 16, k = e % 16;
    put_bf16(S.w1, MLP_H, o, k, k < (uint32_t)MLP_IN ? params[P_W1 + o * MLP_IN + k] : 0.f);
  }
  for (uint32_t e = t; e < MLP_H * MLP_H; e += TT)
    put_bf16(S.w2, MLP_H, e / MLP_H, e % MLP_H, params[P_W2 + e]);
  for (uint32_t e = t; e < 16 * MLP_H; e += TT) {
    const uint32_t o = e / MLP_H, k = e % MLP_H;
    put_bf16(S.w3, 16, o, k, o < (uint32_t)MLP_OUT ? params[P_W3 + o * MLP_H + k] : 0.f);
  }
  if (t < (uint32_t)MLP_H) {
    S.b1[t] = params[P_B1 + t];
    S.b2[t] = params[P_B2 + t];
  }
  if (t < (uint32_t)MLP_OUT) S.b3[t] = params[P_B3 + t];
  if (t == 0) {
    tc::mbar_init(&S.bar, 1);
    S.err = 0;
    tc::mbar_init_fence();
  }
  __syncwarp();
  if (warp == 0) {
    tc::tmem_alloc(&S.tmem, 128);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = S.tmem;
  const uint32_t lane_base = (warp * 32u) << 16;
  volatile uint32_t *abort = &S.err;
  constexpr uint64_t BUDGET = 50ull * 1000 * 1000;
  const uint32_t hl = (TT / 8) * 128;  // LBO of the 128-row activation tiles
  bool ok = true;
  uint32_t phase = 0;
  // one layer: D (cols col0..) = A (rows TT, K = kdim) x B (rows nrows, K = kdim)
  auto layer = [&](const unsigned char *A, const unsigned char *B, uint32_t nrows, uint32_t kdim,
                   uint32_t col0) {
    if (t == 0) {
      tc::fence_after_sync();
      const uint32_t a0 = tc::smem_addr(A), b0 = tc::smem_addr(B), bl = (nrows / 8) * 128;
      const uint32_t idesc = tc::idesc_bf16_f32(TT, nrows);
      for (uint32_t ks = 0; ks < kdim / 16; ++ks)
        tc::mma_bf16(tmem + col0, tc::smem_desc(a0 + ks * 2 * hl, hl, 128),
                     tc::smem_desc(b0 + ks * 2 * bl, bl, 128), idesc, ks ? 1u : 0u);
      tc::commit(&S.bar);
    }
    if (!tc::mbar_wait(&S.bar, phase & 1, abort, BUDGET)) ok = false;
    ++phase;
    tc::fence_after_sync();
    ok = __syncthreads_and(ok);  // every thread of a warp takes the same path into tcgen05.ld
  };
  float v[32];
  // layer 1: x W1^T -> TMEM cols 0..63
  layer(S.x, S.w1, MLP_H, 16, 0);
  if (ok) {
    for (uint32_t c0 = 0; c0 < (uint32_t)MLP_H; c0 += 32) {
      tc::tmem_ld32(tmem + lane_base + c0, v);
      for (uint32_t k = 0; k < 32; ++k) put_bf16(S.h, TT, t, c0 + k, gelu(v[k] + S.b1[c0 + k]));
    }
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  // layer 2: h1 W2^T -> cols 64..127
  if (ok) layer(S.h, S.w2, MLP_H, MLP_H, 64);
  if (ok) {
    // the MMA has read h1 (its completion was waited on): h2 overwrites it
    for (uint32_t c0 = 0; c0 < (uint32_t)MLP_H; c0 += 32) {
      tc::tmem_ld32(tmem + lane_base + 64 + c0, v);
      for (uint32_t k = 0; k < 32; ++k) put_bf16(S.h, TT, t, c0 + k, gelu(v[k] + S.b2[c0 + k]));
    }
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  // layer 3: h2 W3^T -> cols 0..15
  if (ok) layer(S.h, S.w3, 16, MLP_H, 0);
  if (ok) {
    tc::tmem_ld32(tmem + lane_base, v);
    if (i < n)
      for (uint32_t o = 0; o < (uint32_t)MLP_OUT; ++o) y[(size_t)i * MLP_OUT + o] = v[o] + S.b3[o];
  }
  tc::fence_before_sync();
  const bool all_ok = __syncthreads_and(ok);
  if (warp == 0 && all_ok) tc::tmem_dealloc(tmem, 128);
  if (t == 0 && !all_ok && err_flag) atomicOr(err_flag, ST_WAIT_TIMEOUT);
}

int mlp_infer_tc(const float *x, uint32_t n, const float *params, float *y, uint32_t *err_flag,
                 cudaStream_t st) {
  if (n == 0) return 0;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(InferSmem));
    attr = true;
  }
  D3_LAUNCH(k_mlp_infer_tc, blocks_for(n, TT), TT, sizeof(InferSmem), st)(x, n, params, y,
                                                                         err_flag);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace d3

using namespace d3;

namespace {

int grad_launch(const float *x, const float *y, uint32_t n, const float *params, float *grad,
                float *loss, cudaStream_t st) {
  static int blocks = 0;
  if (!blocks) {
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(TrainSmem));
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    blocks = sms;
  }
  unsigned b = blocks_for(n, TT);
  if (b > (unsigned)blocks) b = blocks;
  if (cudaMemsetAsync(grad, 0, MLP_PARAMS * 4, st) != cudaSuccess ||
      cudaMemsetAsync(loss, 0, 4, st) != cudaSuccess)
    return -1;
  D3_LAUNCH(k_mlp_grad, b, TT, sizeof(TrainSmem), st)(x, y, n, params, (float)n, grad, loss);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

extern "C" int32_t d3_mlp_grad(const float *x, const float *y, uint32_t n, const float *params,
                               float *grad, float *loss) {
  if (!x || !y || !params || !grad || !loss || n == 0) return D3_BAD_ARGUMENT;
  float *d = nullptr;
  if (cudaMalloc(&d, (2 * MLP_PARAMS + 1) * 4) != cudaSuccess) return D3_OUT_OF_MEMORY;
  float *dp = d, *dg = d + MLP_PARAMS, *dl = d + 2 * MLP_PARAMS;
  int32_t rc = D3_OK;
  if (cudaMemcpy(dp, params, MLP_PARAMS * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      grad_launch(x, y, n, dp, dg, dl, 0) ||
      cudaMemcpy(grad, dg, MLP_PARAMS * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(loss, dl, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = D3_WORKER_FAILED;
  *loss /= (float)n;
  cudaFree(d);
  return rc;
}

extern "C" int32_t d3_mlp_train(const float *x, const float *y, uint32_t n, uint32_t batch,
                                uint32_t steps, float lr, float *params, float *losses) {
  if (!x || !y || !params || n == 0 || batch == 0) return D3_BAD_ARGUMENT;
  float *d = nullptr;
  if (cudaMalloc(&d, (4 * MLP_PARAMS + 1) * 4) != cudaSuccess) return D3_OUT_OF_MEMORY;
  float *dp = d, *dm = d + MLP_PARAMS, *dv = d + 2 * MLP_PARAMS, *dg = d + 3 * MLP_PARAMS,
        *dl = d + 4 * MLP_PARAMS;
  int32_t rc = D3_OK;
  cudaStream_t st = 0;
  if (cudaMemcpy(dp, params, MLP_PARAMS * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(dm, 0, 2 * MLP_PARAMS * 4) != cudaSuccess)
    rc = D3_WORKER_FAILED;
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1, c2 = 1;
  uint32_t off = 0;
  for (uint32_t s = 0; s < steps && rc == D3_OK; ++s) {
    const uint32_t nb = batch < n ? batch : n;
    if (off + nb > n) off = 0;  // batches walk the (pre-shuffled) samples in order
    if (grad_launch(x + (size_t)off * MLP_IN, y + (size_t)off * MLP_OUT, nb, dp, dg, dl, st)) {
      rc = D3_WORKER_FAILED;
      break;
    }
    off += nb;
    c1 *= b1;
    c2 *= b2;
    D3_LAUNCH(k_mlp_adam, blocks_for(MLP_PARAMS, 256), 256, 0, st)(dp, dm, dv, dg, lr, b1, b2,
                                                                    1e-8f, 1 - c1, 1 - c2);
    if (losses) {
      float l = 0;
      if (cudaMemcpyAsync(&l, dl, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        rc = D3_WORKER_FAILED;
      losses[s] = l / (float)nb;
    }
  }
  if (rc == D3_OK && (cudaMemcpy(params, dp, MLP_PARAMS * 4, cudaMemcpyDeviceToHost) != cudaSuccess))
    rc = D3_WORKER_FAILED;
  cudaFree(d);
  return rc;
}

extern "C" int32_t d3_mlp_infer(const float *x, uint32_t n, const float *params, float *y,
                                uint32_t tensor_cores) {
  if (!x || !params || !y) return D3_BAD_ARGUMENT;
  float *dp = nullptr;
  uint32_t *flag = nullptr;
  if (cudaMalloc(&dp, MLP_PARAMS * 4) != cudaSuccess || cudaMalloc(&flag, 4) != cudaSuccess) {
    cudaFree(dp);
    return D3_OUT_OF_MEMORY;
  }
  int32_t rc = D3_OK;
  uint32_t h_flag = 0;
  if (cudaMemcpy(dp, params, MLP_PARAMS * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(flag, 0, 4) != cudaSuccess)
    rc = D3_WORKER_FAILED;
  if (rc == D3_OK) {
    if (tensor_cores) {
      if (mlp_infer_tc(x, n, dp, y, flag, 0)) rc = D3_WORKER_FAILED;
    } else {
      D3_LAUNCH(k_mlp_infer_cc, blocks_for(n, 128), 128, 0, 0)(x, n, dp, y);
    }
  }
  if (cudaMemcpy(&h_flag, flag, 4, cudaMemcpyDeviceToHost) != cudaSuccess || h_flag)
    rc = D3_WORKER_FAILED;
  cudaFree(dp);
  cudaFree(flag);
  return rc;
}
