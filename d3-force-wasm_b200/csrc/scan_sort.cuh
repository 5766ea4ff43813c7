// scan_sort.cuh — device-wide exclusive scan and stable LSD radix sort.
//
// The sort is the reference's algorithm (sort.zig:55-91: stable LSD radix,
// 8-bit digits, per-chunk histograms turned into offsets that keep equal
// digits in input order) laid out for the GPU: one tile of TILE keys per CTA,
// a digit-major histogram (digit * tiles + tile) so one exclusive scan yields
// every tile's base per digit, and a stable in-tile ranking with warp match.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace d3 {

// ---- scans inside a cooperative launch -------------------------------------

// Block-wide sum of one value per thread (every thread gets it); `sw` is
// shared scratch of 32 words.
__device__ inline uint32_t block_sum(uint32_t v, uint32_t *sw) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sw[warp] = v;
  __syncthreads();
  uint32_t t = 0;
  for (unsigned w = 0; w < blockDim.x / 32; ++w) t += sw[w];
  return t;
}

// Block-wide exclusive scan of one value per thread; the total to *tot.
__device__ inline uint32_t block_excl(uint32_t v, uint32_t *sw, uint32_t &tot) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  __syncthreads();
  if (lane == 31) sw[warp] = incl;
  __syncthreads();
  uint32_t pre = 0;
  tot = 0;
  for (unsigned w = 0; w < nw; ++w) {
    if (w < warp) pre += sw[w];
    tot += sw[w];
  }
  return pre + incl - v;
}

// out[0..len) = exclusive scan of in[0..len) over the whole grid; returns the
// total. One grid barrier inside; the caller syncs before reading out.
__device__ inline uint32_t grid_excl_scan(cooperative_groups::grid_group &g, const uint32_t *in, uint32_t *out,
                                   uint32_t len, uint32_t *bsum) {
  __shared__ uint32_t sw[32];
  const uint32_t nb = gridDim.x, b = blockIdx.x, t = threadIdx.x;
  const uint32_t seg = (len + nb - 1) / nb;
  const uint32_t s0 = min(len, b * seg), s1 = min(len, s0 + seg);
  uint32_t acc = 0;
  for (uint32_t i = s0 + t; i < s1; i += blockDim.x) acc += __ldcg(&in[i]);
  acc = block_sum(acc, sw);
  if (t == 0) bsum[b] = acc;
  g.sync();
  uint32_t off = 0, tot = 0;
  for (uint32_t k = t; k < nb; k += blockDim.x) {
    const uint32_t x = __ldcg(&bsum[k]);
    if (k < b) off += x;
    tot += x;
  }
  off = block_sum(off, sw);
  tot = block_sum(tot, sw);
  uint32_t run = off;
  for (uint32_t base = s0; base < s1; base += blockDim.x) {
    const uint32_t i = base + t;
    const uint32_t x = i < s1 ? __ldcg(&in[i]) : 0;
    uint32_t tile;
    const uint32_t ex = block_excl(x, sw, tile);
    if (i < s1) out[i] = run + ex;
    run += tile;
  }
  return tot;
}



constexpr unsigned SCAN_BLOCK = 1024;

// Exclusive scan of n u32 into out (may alias in); total to *total if given.
// Scratch: `partials` of at least blocks_for(n, SCAN_BLOCK * 4) + 1 words.
void scan_u32(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *partials,
              uint32_t *total, cudaStream_t st);

constexpr unsigned SORT_TILE = 2048;
constexpr unsigned SORT_THREADS = 256;

// Stable sort of (keys, vals)[0..n) by key bytes [byte_lo, byte_hi), then (if
// `partition_hi_bit`) a stable partition on bit 31 of the value, zeros first
// (folded into the last byte pass as a 9-bit digit). Results end in
// keys/vals. Scratch: keys_tmp, vals_tmp (n each) and hist of at least
// 512 * tiles + 1 words plus scan partials.
struct SortScratch {
  uint64_t *keys_tmp;
  uint32_t *vals_tmp;
  uint32_t *hist;      // 512 * tiles
  uint32_t *partials;  // scan partials
};
void radix_sort_u64(uint64_t *keys, uint32_t *vals, uint32_t n, int byte_lo, int byte_hi,
                    bool partition_hi_bit, const SortScratch &s, cudaStream_t st);

inline size_t sort_hist_words(uint32_t n) {
  size_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
  if (!tiles) tiles = 1;
  return 512 * tiles + 1;
}
inline size_t scan_partial_words(size_t n) { return blocks_for(n, SCAN_BLOCK * 4) + 2; }

}  // namespace d3
