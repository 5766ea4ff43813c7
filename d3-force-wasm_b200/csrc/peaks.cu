// peaks.cu — device rates the exact tick's roofline is measured against.
//
// The driver's measured peaks give HBM bandwidth and BF16 tensor throughput;
// the exact kernels run on the FP64 pipe without FMA contraction (strict
// IEEE f64, no fused multiply-add, as the reference's @setFloatMode(.strict)
// wasm code) and wait on one another through L2. d3_device_peaks times, with
// CUDA events on one stream:
//   out[0] DADD per second over the whole GPU (independent chains)
//   out[1] DMUL per second
//   out[2] DFMA per second (x2 for flop/s)
//   out[3] IEEE f64 divisions per second (correctly rounded, -prec-div=true)
//   out[4] IEEE f64 square roots per second
//   out[5] the one-way handoff latency between two SMs in microseconds: a
//          release store of a flag in global memory seen by an acquire load
//          spinning on another SM (half of a measured ping-pong round trip)
//   out[6] SMs, out[7] SM clock (kHz, the device attribute)
//   out[8] (len >= 9) FP32 FMA per second
// Every spin is bounded; a wait that runs out makes the call fail.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "common.cuh"

namespace d3 {
namespace {

constexpr int PK_THREADS = 256;
constexpr int PK_CHAINS = 8;  // independent dependency chains per thread

template <int OP>
__global__ void __launch_bounds__(PK_THREADS) k_peak_fp64(double *out, int iters, double a,
                                                           double b) {
  double v[PK_CHAINS];
  const double seed = 1.0 + 1e-9 * (blockIdx.x * blockDim.x + threadIdx.x);
#pragma unroll
  for (int c = 0; c < PK_CHAINS; ++c) v[c] = seed + c;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) {
      if (OP == 0) v[c] = __dadd_rn(v[c], a);
      else if (OP == 1) v[c] = __dmul_rn(v[c], a);
      else if (OP == 2) v[c] = __fma_rn(v[c], a, b);
      else if (OP == 3) v[c] = b / v[c] + a;  // the add keeps the value in range
      else v[c] = sqrt(v[c]) + a;
    }
  }
  double s = 0;
#pragma unroll
  for (int c = 0; c < PK_CHAINS; ++c) s += v[c];
  if (s == 12345.678) out[0] = s;  // keeps the chains alive
}

__global__ void __launch_bounds__(PK_THREADS) k_peak_ffma(double *out, int iters, float a, float b) {
  float v[PK_CHAINS];
  const float seed = 1.0f + 1e-6f * (threadIdx.x & 63);
#pragma unroll
  for (int c = 0; c < PK_CHAINS; ++c) v[c] = seed + c;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) v[c] = __fmaf_rn(v[c], a, b);
  }
  float s = 0;
#pragma unroll
  for (int c = 0; c < PK_CHAINS; ++c) s += v[c];
  if (s == 12345.678f) out[0] = s;
}

// Ping-pong between block 0 and block 1 of a cooperative launch (so both are
// resident at once): block 0 writes k + 1 when it sees k (even), block 1
// when it sees k (odd). Each wait gives up after `limit` polls.
__global__ void k_pingpong(unsigned *flag, int rounds, unsigned long long limit,
                           unsigned long long *result) {
  if (threadIdx.x != 0 || blockIdx.x > 1) return;
  const unsigned me = blockIdx.x;
  unsigned long long t0 = 0;
  if (me == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (int r = 0; r < rounds; ++r) {
    const unsigned want = 2u * r + me;
    unsigned long long polls = 0;
    unsigned v;
    for (;;) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
      if (v == want) break;
      if (++polls > limit) {
        atomicAdd(&result[1], 1ull);  // gave up
        return;
      }
    }
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(flag), "r"(want + 1) : "memory");
  }
  if (me == 0) {
    unsigned long long t1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
    result[0] = t1 - t0;  // nanoseconds
  }
}

float time_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

}  // namespace
}  // namespace d3

using namespace d3;

extern "C" int32_t d3_device_peaks(double *out, uint32_t len) {
  if (!out || len < 8) return D3_BAD_ARGUMENT;
  int dev = 0, sms = 0, clk_khz = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return D3_WORKER_FAILED;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, dev);
  double *sink = nullptr;
  unsigned *flag = nullptr;
  unsigned long long *res = nullptr;
  if (cudaMalloc(&sink, 64) != cudaSuccess || cudaMalloc(&flag, 64) != cudaSuccess ||
      cudaMalloc(&res, 64) != cudaSuccess) {
    cudaFree(sink);
    cudaFree(flag);
    return D3_OUT_OF_MEMORY;
  }
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_peak_fp64<0>, PK_THREADS, 0);
  const int blocks = sms * (per > 0 ? per : 1);
  const double ops_per_iter = (double)blocks * PK_THREADS * PK_CHAINS;
  int32_t rc = D3_OK;
  auto run = [&](auto kernel, int iters) {
    kernel<<<blocks, PK_THREADS, 0, st>>>(sink, 4, 1.0000001, 0.5);  // warm-up
    cudaEventRecord(e0, st);
    kernel<<<blocks, PK_THREADS, 0, st>>>(sink, iters, 1.0000001, 0.5);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = D3_WORKER_FAILED;
    return ops_per_iter * iters / (time_ms(e0, e1) * 1e-3);
  };
  out[0] = run(k_peak_fp64<0>, 1024);
  out[1] = run(k_peak_fp64<1>, 1024);
  out[2] = run(k_peak_fp64<2>, 1024);
  out[3] = run(k_peak_fp64<3>, 128);
  out[4] = run(k_peak_fp64<4>, 128);
  // handoff latency: 2000 rounds, each wait at most 2^20 polls (well under a
  // second)
  const int rounds = 2000;
  cudaMemsetAsync(flag, 0, 64, st);
  cudaMemsetAsync(res, 0, 64, st);
  {
    int r = rounds;
    unsigned long long limit = 1ull << 20;
    void *args[] = {&flag, &r, &limit, &res};
    if (cudaLaunchCooperativeKernel((const void *)k_pingpong, 2, 32, args, 0, st) != cudaSuccess)
      rc = D3_WORKER_FAILED;
  }
  unsigned long long h[2] = {0, 0};
  if (cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess || h[1] != 0)
    rc = D3_WORKER_FAILED;
  // nanoseconds per round trip (two handoffs) -> microseconds per handoff
  out[5] = (double)h[0] / rounds / 2.0 * 1e-3;
  out[6] = sms;
  out[7] = clk_khz;
  if (len >= 9) {
    // FP32 FMA per second (x2 for flop/s): the fast forms' near field
    k_peak_ffma<<<blocks, PK_THREADS, 0, st>>>(sink, 4, 0.9999999f, 0.5f);
    cudaEventRecord(e0, st);
    k_peak_ffma<<<blocks, PK_THREADS, 0, st>>>(sink, 4096, 0.9999999f, 0.5f);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = D3_WORKER_FAILED;
    out[8] = ops_per_iter * 4096 / (time_ms(e0, e1) * 1e-3);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(sink);
  cudaFree(flag);
  cudaFree(res);
  return rc;
}
