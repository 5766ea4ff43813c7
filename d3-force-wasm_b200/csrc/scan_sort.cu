// scan_sort.cu — device-wide exclusive scan and stable LSD radix sort.
#include "scan_sort.cuh"

namespace d3 {

// ---- exclusive scan --------------------------------------------------------

// Block-wide exclusive scan of one value per thread (blockDim a multiple of
// 32, at most 1024); the block total goes to *total.
__device__ inline uint32_t block_exclusive_scan(uint32_t v, uint32_t *sw, uint32_t *total) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  if (lane == 31) sw[warp] = x;
  __syncthreads();
  const unsigned nw = blockDim.x >> 5;
  if (warp == 0) {
    uint32_t w = lane < nw ? sw[lane] : 0;
    uint32_t t = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= (unsigned)o) t += y;
    }
    if (lane < nw) sw[lane] = t - w;
    if (lane == nw - 1) sw[32] = t;
  }
  __syncthreads();
  uint32_t r = sw[warp] + x - v;
  *total = sw[32];
  __syncthreads();
  return r;
}

// Each block scans 4 * blockDim values (4 consecutive per thread).
__global__ void k_scan_local(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *partials) {
  __shared__ uint32_t sw[33];
  const size_t base = (size_t)blockIdx.x * blockDim.x * 4 + threadIdx.x * 4;
  uint32_t v[4];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  uint32_t tot;
  uint32_t ex = block_exclusive_scan(s, sw, &tot);
  uint32_t run = ex;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// Scans the block partials in place (one block; loops if many).
__global__ void k_scan_partials(uint32_t *partials, uint32_t nb, uint32_t *total) {
  __shared__ uint32_t sw[33];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t off = 0; off < nb; off += blockDim.x) {
    uint32_t i = off + threadIdx.x;
    uint32_t v = i < nb ? partials[i] : 0;
    uint32_t tot;
    uint32_t ex = block_exclusive_scan(v, sw, &tot);
    if (i < nb) partials[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_add(uint32_t *out, uint32_t n, const uint32_t *partials) {
  const size_t base = (size_t)blockIdx.x * blockDim.x * 4 + threadIdx.x * 4;
  uint32_t p = partials[blockIdx.x];
  if (p == 0) return;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (base + k < n) out[base + k] += p;
}

void scan_u32(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *partials, uint32_t *total,
              cudaStream_t st) {
  unsigned nb = blocks_for(n, SCAN_BLOCK * 4);
  D3_LAUNCH(k_scan_local, nb, SCAN_BLOCK, 0, st)(in, out, n, partials);
  D3_LAUNCH(k_scan_partials, 1, SCAN_BLOCK, 0, st)(partials, nb, total);
  if (nb > 1) D3_LAUNCH(k_scan_add, nb, SCAN_BLOCK, 0, st)(out, n, partials);
}

// ---- radix sort -------------------------------------------------------------

// Digit modes: BYTE, the key's byte at `shift` (256 buckets); PART_BYTE, the
// value's bit 31 above the key's byte at `shift` (512 buckets: the partition
// on bit 31 folded into the last byte pass, the same stable order as a byte
// pass followed by a partition pass).
enum : int { BYTE = 0, PART_BYTE = 1 };

template <int MODE>
__host__ __device__ constexpr unsigned buckets() {
  return MODE == PART_BYTE ? 512u : 256u;
}

template <int MODE>
__device__ inline uint32_t digit_of(uint64_t k, uint32_t v, int shift) {
  const uint32_t b = (uint32_t)(k >> shift) & 255u;
  return MODE == PART_BYTE ? ((v >> 31) << 8) | b : b;
}

template <int MODE>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist(const uint64_t *keys, const uint32_t *vals,
                                                            uint32_t n, int shift, uint32_t *hist,
                                                            uint32_t tiles) {
  constexpr unsigned NB = buckets<MODE>();
  __shared__ uint32_t h[NB];
  for (unsigned d = threadIdx.x; d < NB; d += blockDim.x) h[d] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * SORT_TILE;
  for (unsigned k = threadIdx.x; k < SORT_TILE; k += blockDim.x) {
    size_t i = base + k;
    if (i < n) atomicAdd(&h[digit_of<MODE>(keys[i], vals[i], shift)], 1u);
  }
  __syncthreads();
  for (unsigned d = threadIdx.x; d < NB; d += blockDim.x) hist[(size_t)d * tiles + blockIdx.x] = h[d];
}

// Stable scatter of one tile of SORT_TILE keys: warp w takes the tile's
// w-th run of 32 x PER keys, in PER rounds of 32. In a round a key's rank
// among equal digits is the warp's count of that digit so far plus the lanes
// below it with the same digit (warp match). The warps' counts then give
// each key its place in the tile sorted by digit (stable); the tile is
// reordered in shared memory and written in that order, so consecutive
// threads write consecutive places of one digit's run (tile offset from the
// scanned histograms).
template <int MODE>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_scatter(const uint64_t *keys, const uint32_t *vals,
                                                               uint64_t *okeys, uint32_t *ovals,
                                                               uint32_t n, int shift,
                                                               const uint32_t *offsets,
                                                               uint32_t tiles) {
  constexpr unsigned NB = buckets<MODE>();
  constexpr unsigned WARPS = SORT_THREADS / 32, PER = SORT_TILE / SORT_THREADS;
  __shared__ uint32_t wh[WARPS][NB];
  __shared__ uint32_t lstart[NB], gbase[NB];
  __shared__ uint64_t skey[SORT_TILE];
  __shared__ uint32_t sval[SORT_TILE];
  __shared__ uint32_t wsum[WARPS];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1;
  for (unsigned d = threadIdx.x; d < WARPS * NB; d += blockDim.x) (&wh[0][0])[d] = 0;
  const size_t tbase = (size_t)blockIdx.x * SORT_TILE;
  const size_t wbase = tbase + (size_t)warp * 32 * PER;
  const uint32_t tn = n - tbase < SORT_TILE ? (uint32_t)(n - tbase) : SORT_TILE;
  uint64_t k[PER];
  uint32_t v[PER], dg[PER], rk[PER];
#pragma unroll
  for (unsigned r = 0; r < PER; ++r) {
    const size_t i = wbase + r * 32 + lane;
    k[r] = i < n ? keys[i] : 0;
    v[r] = i < n ? vals[i] : 0;
  }
  __syncthreads();
#pragma unroll
  for (unsigned r = 0; r < PER; ++r) {
    const bool valid = wbase + r * 32 + lane < n;
    const uint32_t d = valid ? digit_of<MODE>(k[r], v[r], shift) : NB + lane;  // never matches
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned below = __popc(peers & lt);
    const uint32_t cnt = valid ? wh[warp][d] : 0;
    __syncwarp();
    if (valid && below == 0) wh[warp][d] = cnt + __popc(peers);
    __syncwarp();
    dg[r] = d;
    rk[r] = cnt + below;
  }
  __syncthreads();
  // per digit: the earlier warps' counts (in place) and the tile's count;
  // the tile's digit starts by a block scan of the counts
  uint32_t tot[NB / SORT_THREADS];
#pragma unroll
  for (unsigned j = 0; j < NB / SORT_THREADS; ++j) {
    const unsigned d = j * SORT_THREADS + threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (unsigned w = 0; w < WARPS; ++w) {
      const uint32_t t = wh[w][d];
      wh[w][d] = run;
      run += t;
    }
    tot[j] = run;
    gbase[d] = offsets[(size_t)d * tiles + blockIdx.x];
  }
  // exclusive scan of the NB tile counts, a chunk of SORT_THREADS digits at a
  // time (thread t holds digit j * SORT_THREADS + t of chunk j)
  {
    uint32_t chunk_base = 0;
#pragma unroll
    for (unsigned j = 0; j < NB / SORT_THREADS; ++j) {
      uint32_t x = tot[j], in = x;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, in, o);
        if (lane >= (unsigned)o) in += y;
      }
      __syncthreads();
      if (lane == 31) wsum[warp] = in;
      __syncthreads();
      uint32_t pre = 0, all = 0;
      for (unsigned w = 0; w < WARPS; ++w) {
        if (w < warp) pre += wsum[w];
        all += wsum[w];
      }
      lstart[j * SORT_THREADS + threadIdx.x] = chunk_base + pre + in - x;
      chunk_base += all;
    }
  }
  __syncthreads();
  // each key into its place in the tile's digit order
#pragma unroll
  for (unsigned r = 0; r < PER; ++r)
    if (wbase + r * 32 + lane < n) {
      const uint32_t at = lstart[dg[r]] + wh[warp][dg[r]] + rk[r];
      skey[at] = k[r];
      sval[at] = v[r];
    }
  __syncthreads();
  // write in tile order: place i of digit d goes to gbase[d] + i - lstart[d]
  for (uint32_t i = threadIdx.x; i < tn; i += blockDim.x) {
    const uint64_t kk = skey[i];
    const uint32_t vv = sval[i];
    const uint32_t d = digit_of<MODE>(kk, vv, shift);
    const uint32_t pos = gbase[d] + (i - lstart[d]);
    okeys[pos] = kk;
    ovals[pos] = vv;
  }
}

template <int MODE>
static void sort_pass(const uint64_t *ik, const uint32_t *iv, uint64_t *ok, uint32_t *ov, uint32_t n,
                      int shift, const SortScratch &s, cudaStream_t st) {
  uint32_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
  D3_LAUNCH(k_sort_hist<MODE>, tiles, SORT_THREADS, 0, st)(ik, iv, n, shift, s.hist, tiles);
  scan_u32(s.hist, s.hist, buckets<MODE>() * tiles, s.partials, nullptr, st);
  D3_LAUNCH(k_sort_scatter<MODE>, tiles, SORT_THREADS, 0, st)(ik, iv, ok, ov, n, shift, s.hist,
                                                             tiles);
}

void radix_sort_u64(uint64_t *keys, uint32_t *vals, uint32_t n, int byte_lo, int byte_hi,
                    bool partition_hi_bit, const SortScratch &s, cudaStream_t st) {
  if (n == 0) return;
  uint64_t *ak = keys, *bk = s.keys_tmp;
  uint32_t *av = vals, *bv = s.vals_tmp;
  for (int b = byte_lo; b < byte_hi; ++b) {
    // the partition on bit 31 rides on the last byte pass
    if (partition_hi_bit && b + 1 == byte_hi) sort_pass<PART_BYTE>(ak, av, bk, bv, n, 8 * b, s, st);
    else sort_pass<BYTE>(ak, av, bk, bv, n, 8 * b, s, st);
    uint64_t *tk = ak; ak = bk; bk = tk;
    uint32_t *tv = av; av = bv; bv = tv;
  }
  if (ak != keys) {
    cudaMemcpyAsync(keys, ak, (size_t)n * 8, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(vals, av, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
  }
}

}  // namespace d3
