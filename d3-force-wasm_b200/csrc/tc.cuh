// tc.cuh — the sm_100a tensor-core path: tcgen05 MMA with operands in shared
// memory and the accumulator in tensor memory (TMEM), as inline PTX.
//
// Operand layout (both operands K-major, no swizzle): a tile of R rows x K
// bf16 values is stored as "core matrices" of 8 rows x 16 bytes (8 values);
// the core matrix of row group g (rows 8g .. 8g+7) and 16-byte column chunk c
// sits at byte  c * (R / 8) * 128 + g * 128, its rows 16 bytes apart. So one
// MMA of K = 16 reads chunks c, c + 1: leading byte offset (between the two
// chunks) = (R / 8) * 128, stride byte offset (between row groups) = 128.
// tc_tile_offset() gives the byte offset of (row, chunk).
//
// Every wait on an mbarrier is bounded: after its time budget it gives up,
// sets the CTA's abort flag and returns false; the other threads' waits see
// the flag and give up at once (no spin can outlive its budget).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace d3 {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of (row, 16-byte chunk) in a K-major, unswizzled tile of `rows` rows.
__host__ __device__ __forceinline__ uint32_t tile_offset(uint32_t row, uint32_t chunk,
                                                         uint32_t rows) {
  return chunk * (rows / 8) * 128 + (row / 8) * 128 + (row % 8) * 16;
}

// Shared-memory matrix descriptor (tcgen05 format, version 1): start address,
// leading and stride byte offsets (all >> 4), base offset 0, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // layout type 0 (no swizzle) in bits 61-63
}

// Instruction descriptor, kind::f16: BF16 A and B (K-major), F32 accumulator,
// M x N.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t m, uint32_t n) {
  return (1u << 4)            // D format F32
         | (1u << 7)          // A format BF16
         | (1u << 10)         // B format BF16
         | ((n >> 3) << 17)   // N / 8
         | ((m >> 4) << 24);  // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
        "r"(0u), "r"(0u));
}

// The mbarrier at `bar` gets one arrival when every tcgen05 operation this
// thread issued before has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_addr(bar))
      : "memory");
}

// TMEM allocation by one whole warp; the base address is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(dst)),
               "r"(cols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
               : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy writes to shared memory become visible to the tensor core.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 32 consecutive 32-bit TMEM columns of this thread's lane (warp w of a
// warpgroup reads lanes 32 (w % 4) .. 32 (w % 4) + 31).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                   smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase with parity `parity` to complete. Gives up when
// *abort is set (another thread of the CTA gave up) or after budget_ns of
// global time, setting *abort; returns whether the phase completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile uint32_t *abort,
                                          uint64_t budget_ns) {
  const uint32_t a = smem_addr(bar);
  uint64_t t0 = 0;
  for (uint32_t i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (*abort) return false;
    if ((i & 63) == 0) {
      const uint64_t t = now_ns();
      if (i == 0) t0 = t;
      else if (t - t0 > budget_ns) {
        *abort = 1;
        return false;
      }
    }
  }
}

// 16 bytes from global memory to shared memory without a register (the L2
// path); `bytes` < 16 reads that many and fills the rest with zeros (0: no
// read at all).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// Waits until at most N of this thread's committed groups are still in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Round to bf16 and the bf16 remainder (x ~ hi + lo to about 2^-17 relative).
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __double2bfloat16(x);
  lo = __double2bfloat16(x - (double)__bfloat162float(hi));
}

}  // namespace tc
}  // namespace d3
