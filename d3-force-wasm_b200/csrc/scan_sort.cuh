// scan_sort.cuh — device-wide exclusive scan and stable LSD radix sort.
//
// The sort is the reference's algorithm (sort.zig:55-91: stable LSD radix,
// 8-bit digits, per-chunk histograms turned into offsets that keep equal
// digits in input order) laid out for the GPU: one tile of TILE keys per CTA,
// a digit-major histogram (digit * tiles + tile) so one exclusive scan yields
// every tile's base per digit, and a stable in-tile ranking with warp match.
#pragma once

#include "common.cuh"

namespace d3 {

constexpr unsigned SCAN_BLOCK = 1024;

// Exclusive scan of n u32 into out (may alias in); total to *total if given.
// Scratch: `partials` of at least blocks_for(n, SCAN_BLOCK * 4) + 1 words.
void scan_u32(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *partials,
              uint32_t *total, cudaStream_t st);

constexpr unsigned SORT_TILE = 2048;
constexpr unsigned SORT_THREADS = 256;

// Stable sort of (keys, vals)[0..n) by key bytes [byte_lo, byte_hi), then (if
// `partition_hi_bit`) a stable partition on bit 31 of the value, zeros first.
// Results end in keys/vals. Scratch: keys_tmp, vals_tmp (n each) and hist of
// at least 256 * tiles + 1 words plus scan partials.
struct SortScratch {
  uint64_t *keys_tmp;
  uint32_t *vals_tmp;
  uint32_t *hist;      // 256 * tiles
  uint32_t *partials;  // scan partials
};
void radix_sort_u64(uint64_t *keys, uint32_t *vals, uint32_t n, int byte_lo, int byte_hi,
                    bool partition_hi_bit, const SortScratch &s, cudaStream_t st);

inline size_t sort_hist_words(uint32_t n) {
  size_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
  if (!tiles) tiles = 1;
  return 256 * tiles + 1;
}
inline size_t scan_partial_words(size_t n) { return blocks_for(n, SCAN_BLOCK * 4) + 2; }

}  // namespace d3
