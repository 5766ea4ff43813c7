// fmm.cu — fast many-body: the 2-D FMM of fmm.zig on the device, bit-identical
// to its serial recursion (fmm.zig:247-354).
//
// The reference computes, per target, sums whose order is fixed by a serial
// dual-tree recursion from (root, root). Every accumulation here runs in that
// order, so the device result equals the reference's bit for bit:
//
//  keys     square extent, 16-bit quantised Morton keys, stable 4-pass sort
//           (tree.zig:287-309, 346-364).
//  cells    level-order cells over the sorted keys, leaf at <= 32 points or
//           depth 16, children contiguous (fmm.zig:685-717); all levels at
//           once from each point's shared digits (four launches, no level
//           barriers).
//  upward   per level from the deepest: bounding box, centre and radius
//           (fmm.zig:721-754), P2M at leaves and M2M from the children
//           (fmm.zig:757-806), then M_k /= k! (fmm.zig:629-642).
//  lists    the recursion's calls, expanded level by level. A call (A, B)
//           either ends (M2L of B into A, P2P of B into A's points, or nothing
//           past distanceMax), or splits B (the calls (A, B_j) follow at once,
//           in order), or splits A (the call goes to every child of A). So
//           every child of A receives the same ordered list of B's — the
//           "forward" list of A — and each cell's M2L and P2P lists come out
//           in the order the serial recursion meets them.
//  m2l      per cell, its M2L sources in list order: one lane per (source,
//           l) computes the two-lane correlation of fmm.zig:561-610, then one
//           lane per coefficient adds the sources in order; L_l is unscaled by
//           (-1)^l / l! (fmm.zig:645-657).
//  p2p      per leaf, one lane per target point runs fmm.zig:477-553 against
//           each source leaf of its list in order.
//  downward per level from the root: L2L into the children
//           (fmm.zig:823-849), L2P at leaves (fmm.zig:853-886).
#include <cooperative_groups.h>

#include "fast.cuh"
#include "scan_sort.cuh"

namespace cg = cooperative_groups;

namespace d3 {

constexpr uint32_t FMM_MAX_ORDER = 24;
constexpr uint32_t FMM_DEFAULT_ORDER = 8;
constexpr double FMM_DEFAULT_OPENING = 1.4;
constexpr uint32_t FMM_LEAF = 32;
constexpr uint32_t FMM_LEVELS = 16;
constexpr double FMM_MIN_SEP2 = 1e-28;
constexpr uint32_t FMM_TAB = 2 * FMM_MAX_ORDER + 2;  // rows of the binomial table
constexpr unsigned FMM_THREADS = 256;
constexpr unsigned FMM_WARPS = FMM_THREADS / 32;
constexpr uint32_t FMM_STACK = 64;


struct FmmTables {
  double fact[FMM_TAB];
  double binom[FMM_TAB * FMM_TAB];  // binom[n * FMM_TAB + k]
};

// info words (device, mirrored to the host after the cell build)
// (FI_LIST_OVERFLOW + level parity: a level's overflow is read at the start of
// the next level, while that level writes the other word.)
enum : uint32_t { FI_CELLS = 0, FI_OVERFLOW, FI_LEVELS, FI_POOL_M2L, FI_POOL_P2P, FI_POOL_FWD,
                  FI_LIST_OVERFLOW, FI_LVL = 8,  // FI_LVL + d: first cell of level d
                  FI_M = 40,                     // points to act on (0 when the extent is bad)
                  FI_BAD = 41 };                 // 1: the extent is not finite and positive

struct FmmDev {
  uint32_t pcap = 0, ccap = 0;
  size_t coef_cap = 0, cap_m2l = 0, cap_p2p = 0, cap_fwd = 0;
  double *px = nullptr, *py = nullptr, *ps = nullptr, *ux = nullptr, *uy = nullptr;
  FCell *cells = nullptr;
  double *bx0 = nullptr, *by0 = nullptr, *bx1 = nullptr, *by1 = nullptr;
  uint32_t *m2l_off = nullptr, *m2l_cnt = nullptr, *p2p_off = nullptr, *p2p_cnt = nullptr;
  uint32_t *fwd_off = nullptr, *fwd_cnt = nullptr;
  uint32_t *m2l = nullptr, *p2p = nullptr, *fwd = nullptr;
  double *mco = nullptr, *lco = nullptr;
  FmmTables *tab = nullptr;
  uint32_t tab_p = 0;
  uint32_t *info = nullptr, *bsum = nullptr;
  double *square = nullptr;      // box x0, y0, side
  uint32_t *h_info = nullptr;    // pinned mirror of info
  double *h_geom = nullptr;      // pinned: the geometry read back (w, 1 / w, ox, oy)
  double *geom = nullptr;        // device: w, 1 / w, ox, oy (k_fmm_geom)
  int coop_blocks = 0;
  size_t last_m2l = 0, last_p2p = 0, last_fwd = 0;  // list sizes of the previous run
  // the cell build: per-block counts per level, each cell's start and level
  uint32_t *cb_count = nullptr, *start_of = nullptr;
  uint16_t *pt_levels = nullptr;  // per point: the levels it starts cells at, d0 << 8 | d1
  uint8_t *level_of = nullptr;
  size_t cb_count_cap = 0, start_cap = 0, level_cap = 0;
};

struct FmmArgs {
  const uint64_t *keys;
  const uint32_t *perm;
  const double *px, *py, *ps, *ux, *uy;
  FCell *cells;
  double *bx0, *by0, *bx1, *by1;
  double *mco, *lco;
  const FmmTables *tab;
  double *vx, *vy;
  uint32_t *m2l, *p2p, *fwd;
  uint32_t *m2l_off, *m2l_cnt, *p2p_off, *p2p_cnt, *fwd_off, *fwd_cnt;
  uint32_t *info;
  size_t cap_m2l, cap_p2p, cap_fwd;
  uint32_t ncells, nlev, p, q, stride;
  double mac_far, dmax_scaled, dmin_scaled, dmin2, dmax2, inv_w;
  int ring, has_dmax;
  const double *seed;
};

__device__ inline double ldg_cg(const double *p) { return __ldcg(p); }
__device__ inline uint32_t ldg_cg(const uint32_t *p) { return __ldcg(p); }

// zig @min / @max on finite operands
__device__ inline double zmin(double a, double b) { return b < a ? b : a; }
__device__ inline double zmax(double a, double b) { return b > a ? b : a; }

// ---- keys and gather --------------------------------------------------------

// tree.zig:346-364, 688-695
__device__ inline uint64_t spread16(uint32_t v) {
  uint64_t x = v & 0xFFFF;
  x = (x | (x << 8)) & 0x00FF00FF;
  x = (x | (x << 4)) & 0x0F0F0F0F;
  x = (x | (x << 2)) & 0x33333333;
  x = (x | (x << 1)) & 0x55555555;
  return x;
}

// Sort value: the node, with bit 31 for a NaN coordinate (partitioned last).
__global__ void k_fmm_keys(const double *xs, const double *ys, uint32_t n, const double *square,
                           uint64_t *keys, uint32_t *sv) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = xs[i], y = ys[i];
  if (x != x || y != y) {
    keys[i] = 0;
    sv[i] = i | 0x80000000u;
    return;
  }
  const double b0 = square[0], b1 = square[1], scale = 65536.0 / square[2];
  const double fx = floor((x - b0) * scale), fy = floor((y - b1) * scale);
  const uint32_t qx = (uint32_t)(fx < 65535 ? fx : 65535);
  const uint32_t qy = (uint32_t)(fy < 65535 ? fy : 65535);
  keys[i] = spread16(qx) | (spread16(qy) << 1);
  sv[i] = i;
}

// fmm.zig:668-682
// The run's geometry from the square's extent (tree.zig:287-309): geom =
// {w, 1 / w, ox, oy}; FI_M = the finite points, or 0 with FI_BAD = 1 when
// there are some but the extent is not finite and positive (the exact kernel
// runs instead). The
// same IEEE f64 operations the host would do, so the values are the same.
__global__ void k_fmm_geom(const double *extent, const uint32_t *tinfo, double *geom,
                           uint32_t *info) {
  const double e0 = extent[0], e1 = extent[1], e2 = extent[2], e3 = extent[3];
  const double w = e2 - e0;
  const bool ok = w > 0 && w < INFINITY;
  geom[0] = w;
  geom[1] = 1 / w;
  geom[2] = (e0 + e2) / 2;
  geom[3] = (e1 + e3) / 2;
  const uint32_t m = tinfo[0];
  info[FI_M] = ok ? m : 0;
  info[FI_BAD] = m > 0 && !ok ? 1 : 0;
}

__global__ void k_fmm_gather(const uint32_t *perm, const double *xs, const double *ys,
                             const double *strength, const uint32_t *info, double alpha,
                             const double *geom, double *px, double *py, double *ps, double *ux,
                             double *uy) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= info[FI_M]) return;
  const double inv_w = geom[1], ox = geom[2], oy = geom[3];
  const uint32_t i = perm[j];
  const double x = xs[i], y = ys[i];
  px[j] = x;
  py[j] = y;
  const double st = strength[i] * alpha;
  ps[j] = st != st ? 0 : st;
  ux[j] = (x - ox) * inv_w;
  uy[j] = (y - oy) * inv_w;
}

// ---- grid-wide helpers --------------------------------------------------------

// ---- cells (fmm.zig:685-717) ---------------------------------------------------

// The child ranges of a cell at depth d: bnd[q] .. bnd[q + 1] holds digit q.
// Returns the number of non-empty children (0 for a leaf).
__device__ uint32_t child_ranges(const uint64_t *keys, uint32_t first, uint32_t count, uint32_t d,
                                 uint32_t *bnd) {
  if (count <= FMM_LEAF || d >= FMM_LEVELS) return 0;
  const unsigned shift = 2 * (FMM_LEVELS - 1 - d);
  const uint32_t end = first + count;
  bnd[0] = first;
  bnd[4] = end;
  for (uint32_t q = 1; q < 4; ++q) {
    uint32_t lo = bnd[q - 1], hi = end;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if (((keys[mid] >> shift) & 3) < q) lo = mid + 1;
      else hi = mid;
    }
    bnd[q] = lo;
  }
  uint32_t nc = 0;
  for (uint32_t q = 0; q < 4; ++q) nc += bnd[q + 1] > bnd[q];
  return nc;
}

// ---- cells, all levels at once -------------------------------------------------------
//
// The same cells as fmm.zig:685-717 (level order, each level in key order,
// children contiguous in digit order), built without a pass per level. A
// level-d cell is a maximal run of sorted keys sharing d digits whose
// enclosing level-(d-1) run holds more than FMM_LEAF points (d <= 16). So a
// point k starts cells at the levels d in (lcp(k), top(k)], where lcp(k) is
// the digits it shares with point k - 1, provided the level-lcp(k) run around
// it holds more than FMM_LEAF points, and top(k) = min(16, max(lcp + 1,
// A(k) + 1)) with A(k) the digits keys k and k + FMM_LEAF share (a run that
// starts at k holds more than FMM_LEAF points exactly at the levels <= A(k)).
// Passes: per point the flags and per-block counts per level; a scan of the
// counts; per point the cells' places (level start + block offset + rank in
// the block); per cell its range, children and parent by binary searches.

constexpr uint32_t CB_THREADS = 256;
constexpr uint32_t CB_LEVELS = FMM_LEVELS + 1;  // levels 0 .. 16

__device__ inline int shared_digits(uint32_t a, uint32_t b) {
  return a == b ? 16 : __clz(a ^ b) >> 1;
}

// First index in [lo, hi) whose key >= t (keys sorted; low 32 bits).
__device__ inline uint32_t key_lower(const uint64_t *keys, uint32_t lo, uint32_t hi, uint64_t t) {
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if ((uint64_t)(uint32_t)keys[mid] < t) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// The same first index for a run known to hold k - 1 (keys[k - 1] >= t):
// galloping back from k - 1, then a binary search of the last stride, so a
// short run costs a few loads.
__device__ inline uint32_t key_lower_back(const uint64_t *keys, uint32_t k, uint64_t t) {
  uint32_t hi = k - 1;  // keys[hi] >= t
  uint32_t lo = 0;
  for (uint32_t step = 1; step <= hi; step <<= 1) {
    const uint32_t probe = hi - step;
    if ((uint64_t)(uint32_t)keys[probe] < t) {
      lo = probe + 1;
      break;
    }
    hi = probe;
  }
  return key_lower(keys, lo, hi, t);
}

// First index in [k, m) whose key >= t, for keys[k] < t: galloping forward
// from k, then a binary search of the last stride (a short run costs a few
// loads).
__device__ inline uint32_t key_lower_fwd(const uint64_t *keys, uint32_t k, uint32_t m, uint64_t t) {
  uint32_t lo = k + 1, hi = m;  // the answer is in [lo, hi]
  for (uint32_t step = 1; lo < m; step <<= 1) {
    const uint32_t probe = step < m - lo ? lo + step - 1 : m - 1;
    if ((uint64_t)(uint32_t)keys[probe] >= t) {
      hi = probe;
      break;
    }
    lo = probe + 1;
  }
  return key_lower(keys, lo, hi, t);
}

// The levels at which point k starts cells: [d0, d1] (empty when d1 < d0).
__device__ void cell_levels(const uint64_t *keys, uint32_t m, uint32_t k, int &d0, int &d1) {
  const uint32_t key = (uint32_t)keys[k];
  const int lcp = k == 0 ? -1 : shared_digits((uint32_t)keys[k - 1], key);
  d0 = lcp + 1;
  d1 = -1;
  if (lcp >= (int)FMM_LEVELS) return;
  if (k > 0) {
    // the level-lcp run around k must hold more than FMM_LEAF points
    const uint64_t t = lcp ? (uint64_t)(key >> (32 - 2 * lcp)) << (32 - 2 * lcp) : 0;
    const uint32_t s0 = key_lower_back(keys, k, t);
    if (s0 + FMM_LEAF >= m) return;
    if (shared_digits((uint32_t)keys[s0], (uint32_t)keys[s0 + FMM_LEAF]) < lcp) return;
  }
  const int A = k + FMM_LEAF < m ? shared_digits(key, (uint32_t)keys[k + FMM_LEAF]) : -1;
  int top = A + 1 > d0 ? A + 1 : d0;
  d1 = top < (int)FMM_LEVELS ? top : (int)FMM_LEVELS;
}

__global__ void __launch_bounds__(CB_THREADS) k_cells_count(const uint64_t *keys,
                                                            const uint32_t *info, uint32_t *bcount,
                                                            uint16_t *levels) {
  const uint32_t m = info[FI_M];
  __shared__ uint32_t wc[CB_LEVELS][CB_THREADS / 32];
  const uint32_t k = blockIdx.x * CB_THREADS + threadIdx.x;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int d0 = 0, d1 = -1;
  if (k < m) {
    cell_levels(keys, m, k, d0, d1);
    levels[k] = (uint16_t)(((uint32_t)d0 << 8) | ((uint32_t)d1 & 0xFFu));  // for k_cells_place
  }
  for (int d = 0; d < (int)CB_LEVELS; ++d) {
    const unsigned b = __ballot_sync(0xffffffffu, d >= d0 && d <= d1);
    if (lane == 0) wc[d][warp] = __popc(b);
  }
  __syncthreads();
  if (threadIdx.x < CB_LEVELS) {
    uint32_t t = 0;
    for (uint32_t w = 0; w < CB_THREADS / 32; ++w) t += wc[threadIdx.x][w];
    bcount[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
  }
}

// One block per level: the exclusive scan of that level's block counts; the
// level's cell count goes to info FI_LVL + d (k_cells_starts turns the counts
// into starts).
__global__ void __launch_bounds__(1024) k_cells_scan(uint32_t *bcount, uint32_t nb,
                                                     uint32_t *info) {
  __shared__ uint32_t sw[32];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t d = blockIdx.x;
  uint32_t *v = bcount + (size_t)d * nb;
  uint32_t run = 0;
  for (uint32_t base = 0; base < nb; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t x = i < nb ? v[i] : 0;
    uint32_t incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (unsigned)o) incl += y;
    }
    if (lane == 31) sw[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0, tile = 0;
    for (unsigned w = 0; w < nw; ++w) {
      if (w < warp) wpre += sw[w];
      tile += sw[w];
    }
    if (i < nb) v[i] = run + wpre + incl - x;
    run += tile;
    __syncthreads();
  }
  if (threadIdx.x == 0) info[FI_LVL + d] = run;
}

// One warp: the level starts (info FI_LVL + d) from the per-level counts, the
// cell total, the level count, and the overflow word when the cells do not
// fit `ccap`.
__global__ void __launch_bounds__(32) k_cells_starts(uint32_t ccap, uint32_t *info) {
  static_assert(CB_LEVELS <= 32, "one lane per level");
  const unsigned lane = threadIdx.x;
  const uint32_t x = lane < CB_LEVELS ? info[FI_LVL + lane] : 0;
  uint32_t incl = x;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  const uint32_t at = __shfl_sync(0xffffffffu, incl, 31);
  const unsigned used = __ballot_sync(0xffffffffu, x != 0);
  if (lane < CB_LEVELS) info[FI_LVL + lane] = incl - x;
  if (lane == 0) {
    info[FI_LVL + CB_LEVELS] = at;
    info[FI_CELLS] = at;
    info[FI_LEVELS] = used ? 32 - __clz(used) : 0;
    info[FI_OVERFLOW] = at > ccap ? at : 0;
  }
}

// start_of[cell] = the point that starts it; level_of[cell] = its level.
// (the point's levels as k_cells_count found them)
__global__ void __launch_bounds__(CB_THREADS) k_cells_place(const uint16_t *levels,
                                                            const uint32_t *bcount,
                                                            const uint32_t *info,
                                                            uint32_t *start_of,
                                                            uint8_t *level_of) {
  __shared__ uint32_t wc[CB_LEVELS][CB_THREADS / 32];
  if (__ldcg(&info[FI_OVERFLOW])) return;
  const uint32_t m = info[FI_M];
  const uint32_t k = blockIdx.x * CB_THREADS + threadIdx.x;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int d0 = 0, d1 = -1;
  if (k < m) {
    const uint32_t v = levels[k];
    d0 = (int)(v >> 8);
    d1 = (int)(int8_t)(v & 0xFFu);
  }
  uint32_t rank[CB_LEVELS];
  for (int d = 0; d < (int)CB_LEVELS; ++d) {
    const unsigned b = __ballot_sync(0xffffffffu, d >= d0 && d <= d1);
    rank[d] = __popc(b & ((1u << lane) - 1));
    if (lane == 0) wc[d][warp] = __popc(b);
  }
  __syncthreads();
  if (k >= m) return;
  for (int d = d0; d <= d1; ++d) {
    uint32_t pre = 0;
    for (uint32_t w = 0; w < warp; ++w) pre += wc[d][w];
    const uint32_t c = __ldcg(&info[FI_LVL + d]) + bcount[(size_t)d * gridDim.x + blockIdx.x] +
                       pre + rank[d];
    start_of[c] = k;
    level_of[c] = (uint8_t)d;
  }
}

__global__ void __launch_bounds__(CB_THREADS) k_cells_fill(const uint64_t *keys,
                                                           const uint32_t *start_of,
                                                           const uint8_t *level_of,
                                                           const uint32_t *info, FCell *cells) {
  const uint32_t m = info[FI_M];
  const uint32_t total = __ldcg(&info[FI_CELLS]);
  if (__ldcg(&info[FI_OVERFLOW])) return;
  const uint32_t c = blockIdx.x * CB_THREADS + threadIdx.x;
  if (c >= total) return;
  const uint32_t k = start_of[c];
  const int d = level_of[c];
  const uint32_t key = (uint32_t)keys[k];
  // the run: the points sharing d digits with k
  uint32_t end = m;
  if (d > 0) {
    const uint64_t pre = key >> (32 - 2 * d);
    end = key_lower_fwd(keys, k, m, (pre + 1) << (32 - 2 * d));
  }
  FCell f;
  f.cx = f.cy = f.r = 0;
  f.first = k;
  f.count = end - k;
  f.depth = (uint32_t)d;
  f.child0 = 0;
  f.nchild = 0;
  if (f.count > FMM_LEAF && d < (int)FMM_LEVELS) {
    uint32_t bnd[5];
    f.nchild = child_ranges(keys, k, f.count, (uint32_t)d, bnd);
    // the first child starts at k: its place among level d + 1's starts
    const uint32_t lo = __ldcg(&info[FI_LVL + d + 1]), hi = __ldcg(&info[FI_LVL + d + 2]);
    uint32_t a = lo, b = hi;
    while (a < b) {
      const uint32_t mid = a + (b - a) / 2;
      if (start_of[mid] < k) a = mid + 1;
      else b = mid;
    }
    f.child0 = a;
  }
  f.parent = NONE;
  if (d > 0) {
    // the level d - 1 cell holding k: the last start <= k among that level's
    const uint32_t lo = __ldcg(&info[FI_LVL + d - 1]), hi = __ldcg(&info[FI_LVL + d]);
    uint32_t a = lo, b = hi;
    while (a < b) {
      const uint32_t mid = a + (b - a) / 2;
      if (start_of[mid] <= k) a = mid + 1;
      else b = mid;
    }
    f.parent = a - 1;
  }
  cells[c] = f;
}

// ---- upward: geometry, P2M, M2M, scale ------------------------------------------

// fmm.zig:614-623: powers of d = (dre, dim) into pw[0..p] (re) and pw[q..] (im).
__device__ inline void shift_powers(double dre, double dim, uint32_t p, double *pw) {
  const uint32_t q = p + 1;
  double re = 1, im = 0;
  pw[0] = 1;
  pw[q] = 0;
  for (uint32_t k = 1; k <= p; ++k) {
    const double nre = re * dre - im * dim;
    const double nim = re * dim + im * dre;
    re = nre;
    im = nim;
    pw[k] = re;
    pw[q + k] = im;
  }
}

// Minimum / maximum as the serial scan's strict comparisons: the first
// occurrence in point order wins a tie.
__device__ inline void minmax_merge(double &mn, uint32_t &imn, double &mx, uint32_t &imx,
                                    double omn, uint32_t oimn, double omx, uint32_t oimx) {
  if (omn < mn || (omn == mn && oimn < imn)) { mn = omn; imn = oimn; }
  if (omx > mx || (omx == mx && oimx < imx)) { mx = omx; imx = oimx; }
}

// One cell, by one warp. ws: this warp's shared scratch (32 * stride doubles).
__device__ void upward_cell(const FmmArgs &a, uint32_t c, double *ws) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t p = a.p, q = a.q, stride = a.stride;
  const uint32_t first = a.cells[c].first, count = a.cells[c].count;
  const uint32_t nchild = ldg_cg(&a.cells[c].nchild), child0 = ldg_cg(&a.cells[c].child0);
  double x0, y0, x1, y1;
  if (nchild == 0) {
    double mnx = INFINITY, mxx = -INFINITY, mny = INFINITY, mxy = -INFINITY;
    uint32_t imnx = NONE, imxx = NONE, imny = NONE, imxy = NONE;
    for (uint32_t k = first + lane; k < first + count; k += 32) {
      const double x = a.ux[k], y = a.uy[k];
      if (x < mnx) { mnx = x; imnx = k; }
      if (x > mxx) { mxx = x; imxx = k; }
      if (y < mny) { mny = y; imny = k; }
      if (y > mxy) { mxy = y; imxy = k; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double a0 = __shfl_xor_sync(0xffffffffu, mnx, o), a1 = __shfl_xor_sync(0xffffffffu, mxx, o);
      const uint32_t i0 = __shfl_xor_sync(0xffffffffu, imnx, o), i1 = __shfl_xor_sync(0xffffffffu, imxx, o);
      const double b0 = __shfl_xor_sync(0xffffffffu, mny, o), b1 = __shfl_xor_sync(0xffffffffu, mxy, o);
      const uint32_t j0 = __shfl_xor_sync(0xffffffffu, imny, o), j1 = __shfl_xor_sync(0xffffffffu, imxy, o);
      minmax_merge(mnx, imnx, mxx, imxx, a0, i0, a1, i1);
      minmax_merge(mny, imny, mxy, imxy, b0, j0, b1, j1);
    }
    x0 = mnx; x1 = mxx; y0 = mny; y1 = mxy;
  } else {
    x0 = INFINITY; y0 = INFINITY; x1 = -INFINITY; y1 = -INFINITY;
    for (uint32_t ch = child0; ch < child0 + nchild; ++ch) {
      x0 = zmin(x0, ldg_cg(&a.bx0[ch]));
      x1 = zmax(x1, ldg_cg(&a.bx1[ch]));
      y0 = zmin(y0, ldg_cg(&a.by0[ch]));
      y1 = zmax(y1, ldg_cg(&a.by1[ch]));
    }
  }
  const double cx = (x0 + x1) / 2, cy = (y0 + y1) / 2;
  if (lane == 0) {
    a.bx0[c] = x0; a.by0[c] = y0; a.bx1[c] = x1; a.by1[c] = y1;
    const double dx = x1 - x0, dy = y1 - y0;
    a.cells[c].cx = cx;
    a.cells[c].cy = cy;
    a.cells[c].r = 0.5 * sqrt(dx * dx + dy * dy);
  }
  double *mco = a.mco + (size_t)c * stride;
  if (nchild == 0) {
    // P2M (fmm.zig:757-780): lane t holds point t's terms; then lane r adds
    // real r (re 0..q-1, im q..2q-1) over the points in order.
    double acc0 = 0, acc1 = 0;
    const uint32_t r0 = lane, r1 = lane + 32;
    for (uint32_t base = first; base < first + count; base += 32) {
      const uint32_t k = base + lane;
      const uint32_t np = min(32u, first + count - base);
      double *row = ws + lane * stride;
      if (k < first + count) {
        const double sv = a.ps[k];
        if (sv != sv) {
          row[0] = NAN;  // skipped point
        } else {
          const double zre = a.ux[k] - cx, zim = a.uy[k] - cy;
          double pre = 1, pim = 0;
          row[0] = sv;
          row[q] = 0;
          for (uint32_t o = 1; o < q; ++o) {
            const double nre = pre * zre - pim * zim;
            const double nim = pre * zim + pim * zre;
            pre = nre;
            pim = nim;
            row[o] = sv * pre;
            row[q + o] = sv * pim;
          }
        }
      }
      __syncwarp();
      for (uint32_t t = 0; t < np; ++t) {
        const double *rt = ws + t * stride;
        const double sv = rt[0];
        if (sv != sv) continue;
        if (r0 < stride && r0 != q) acc0 += rt[r0];
        if (r1 < stride && r1 != q) acc1 += rt[r1];
      }
      __syncwarp();
    }
    if (r0 < stride) mco[r0] = acc0;
    if (r1 < stride) mco[r1] = acc1;
  } else {
    // M2M (fmm.zig:782-806): lane nn sums the children in order.
    double sre_acc = 0, sim_acc = 0;
    const uint32_t nn = lane;
    for (uint32_t ch = child0; ch < child0 + nchild; ++ch) {
      if (lane == 0) shift_powers(ldg_cg(&a.cells[ch].cx) - cx, ldg_cg(&a.cells[ch].cy) - cy, p, ws);
      __syncwarp();
      if (nn < q) {
        const double *cre = a.mco + (size_t)ch * stride, *cim = cre + q;
        double sre = 0, sim = 0;
        for (uint32_t k = 0; k <= nn; ++k) {
          const double b = a.tab->binom[nn * FMM_TAB + k];
          const double xre = ldg_cg(&cre[k]) * b, xim = ldg_cg(&cim[k]) * b;
          sre += xre * ws[nn - k] - xim * ws[q + nn - k];
          sim += xre * ws[q + nn - k] + xim * ws[nn - k];
        }
        sre_acc += sre;
        sim_acc += sim;
      }
      __syncwarp();
    }
    if (nn < q) {
      mco[nn] = sre_acc;
      mco[q + nn] = sim_acc;
    }
  }
}

__global__ void __launch_bounds__(FMM_THREADS) k_fmm_upward(FmmArgs a) {
  extern __shared__ double fmm_smem[];
  cg::grid_group g = cg::this_grid();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  double *ws = fmm_smem + (threadIdx.x >> 5) * 32 * a.stride;
  const uint32_t *lvl = a.info + FI_LVL;
  for (int lev = (int)a.nlev - 1; lev >= 0; --lev) {
    for (uint32_t c = lvl[lev] + gw; c < lvl[lev + 1]; c += nwarps) upward_cell(a, c, ws);
    g.sync();
  }
  // fmm.zig:629-642: M_k /= k! for k >= 2
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const size_t total = (size_t)a.ncells * a.q;
  for (size_t idx = tid; idx < total; idx += nth) {
    const uint32_t c = (uint32_t)(idx / a.q), o = (uint32_t)(idx % a.q);
    if (o < 2) continue;
    double *m = a.mco + (size_t)c * a.stride;
    const double inv = 1 / a.tab->fact[o];
    m[o] = ldg_cg(&m[o]) * inv;
    m[a.q + o] = ldg_cg(&m[a.q + o]) * inv;
  }
}

// ---- interaction lists (fmm.zig:400-453) -------------------------------------------

// Expands one call (A, b) of cell c = A with the recursion's order: splits of
// B are followed at once, depth first. WRITE false: counts only (nm, np, nf
// are added to); WRITE true: the events are written from om / op / of on.
// Returns false if the local stack overflowed.
template <bool WRITE>
__device__ bool expand_call(const FmmArgs &a, uint32_t c, const FCell &A, uint32_t b, uint32_t &nm,
                            uint32_t &np, uint32_t &nf, uint32_t om, uint32_t op, uint32_t of) {
  uint32_t stack[FMM_STACK];
  const bool la = A.nchild == 0;
  uint32_t sp = 0;
  stack[sp++] = b;
  while (sp) {
    const uint32_t B = stack[--sp];
    if (B == c) {
      if (la) {
        if (WRITE) a.p2p[op + np] = c;
        ++np;
      } else {
        for (uint32_t j = 0; j < A.nchild; ++j) {
          if (WRITE) a.fwd[of + nf] = A.child0 + j;
          ++nf;
        }
      }
      continue;
    }
    const FCell Bc = a.cells[B];
    const double ra = A.r, rb = Bc.r;
    const double dx = A.cx - Bc.cx, dy = A.cy - Bc.cy;
    const double d2 = dx * dx + dy * dy;
    const double rmax = zmax(ra, rb), rmin = zmin(ra, rb);
    const double thr = a.mac_far * rmax + rmin;
    if (d2 > FMM_MIN_SEP2 && d2 >= thr * thr) {
      bool separated = true;
      if (a.ring) {
        const double gap = sqrt(d2) - ra - rb;
        if (gap >= a.dmax_scaled) continue;
        if (gap + 2 * (ra + rb) > a.dmax_scaled || gap < a.dmin_scaled) separated = false;
      }
      if (separated) {
        if (WRITE) a.m2l[om + nm] = B;
        ++nm;
        continue;
      }
    }
    const bool lb = Bc.nchild == 0;
    if (la && lb) {
      if (WRITE) a.p2p[op + np] = B;
      ++np;
    } else if (la || (!lb && rb > ra)) {
      if (sp + Bc.nchild > FMM_STACK) return false;
      for (uint32_t j = Bc.nchild; j-- > 0;) stack[sp++] = Bc.child0 + j;
    } else {
      if (WRITE) a.fwd[of + nf] = B;
      ++nf;
    }
  }
  return true;
}

__device__ inline uint32_t warp_excl(uint32_t v, uint32_t &total) {
  const unsigned lane = threadIdx.x & 31;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  total = __shfl_sync(0xffffffffu, incl, 31);
  return incl - v;
}

// The calls of cell c (its parent's forward list in order, or (root, root)),
// by one warp: lane k expands calls k, k + 32, ...; each call's events are
// placed after those of the calls before it (a warp scan of the counts).
// Counts, then a reservation in the pools, then counts again and the writes.
__device__ void warp_expand_cell(const FmmArgs &a, uint32_t c, uint32_t *ovf) {
  const unsigned lane = threadIdx.x & 31;
  const FCell A = a.cells[c];
  const uint32_t *in = nullptr;
  uint32_t nin = 1;
  if (c != 0) {
    in = a.fwd + ldg_cg(&a.fwd_off[A.parent]);
    nin = ldg_cg(&a.fwd_cnt[A.parent]);
  }
  uint32_t tm = 0, tp = 0, tf = 0;
  bool ok = true;
  for (uint32_t u0 = 0; u0 < nin; u0 += 32) {
    const uint32_t u = u0 + lane;
    uint32_t nm = 0, np = 0, nf = 0;
    if (u < nin && !expand_call<false>(a, c, A, c == 0 ? 0 : ldg_cg(&in[u]), nm, np, nf, 0, 0, 0))
      ok = false;
    uint32_t t;
    warp_excl(nm, t); tm += t;
    warp_excl(np, t); tp += t;
    warp_excl(nf, t); tf += t;
  }
  ok = __all_sync(0xffffffffu, ok);
  if (!ok) {
    tm = tp = tf = 0;
    if (lane == 0) atomicOr(ovf, 2u);
  }
  uint32_t om = 0, op = 0, of = 0;
  if (lane == 0) {
    om = atomicAdd(&a.info[FI_POOL_M2L], tm);
    op = atomicAdd(&a.info[FI_POOL_P2P], tp);
    of = atomicAdd(&a.info[FI_POOL_FWD], tf);
    a.m2l_off[c] = om; a.m2l_cnt[c] = tm;
    a.p2p_off[c] = op; a.p2p_cnt[c] = tp;
    a.fwd_off[c] = of; a.fwd_cnt[c] = tf;
  }
  om = __shfl_sync(0xffffffffu, om, 0);
  op = __shfl_sync(0xffffffffu, op, 0);
  of = __shfl_sync(0xffffffffu, of, 0);
  if (!ok) return;
  if ((size_t)om + tm > a.cap_m2l || (size_t)op + tp > a.cap_p2p || (size_t)of + tf > a.cap_fwd) {
    if (lane == 0) atomicOr(ovf, 1u);
    return;
  }
  for (uint32_t u0 = 0; u0 < nin; u0 += 32) {
    const uint32_t u = u0 + lane;
    const uint32_t b = u < nin ? (c == 0 ? 0 : ldg_cg(&in[u])) : 0;
    uint32_t nm = 0, np = 0, nf = 0;
    if (u < nin) expand_call<false>(a, c, A, b, nm, np, nf, 0, 0, 0);
    uint32_t t0, t1, t2;
    const uint32_t xm = warp_excl(nm, t0), xp = warp_excl(np, t1), xf = warp_excl(nf, t2);
    if (u < nin) {
      uint32_t wm = 0, wp = 0, wf = 0;
      expand_call<true>(a, c, A, b, wm, wp, wf, om + xm, op + xp, of + xf);
    }
    om += t0;
    op += t1;
    of += t2;
  }
}

// Level by level from the root, a warp per cell; a grid barrier between
// levels (a cell's calls are its parent's forward list).
__global__ void __launch_bounds__(FMM_THREADS) k_fmm_lists(FmmArgs a) {
  cg::grid_group g = cg::this_grid();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t gw = tid >> 5, nwarps = nth >> 5;
  const uint32_t *lvl = a.info + FI_LVL;
  for (uint32_t lev = 0; lev < a.nlev; ++lev) {
    // the previous level's word: nobody writes it during this level, so every
    // thread takes the same branch
    if (lev && ldg_cg(&a.info[FI_LIST_OVERFLOW + ((lev - 1) & 1)])) break;
    uint32_t *ovf = &a.info[FI_LIST_OVERFLOW + (lev & 1)];
    for (uint32_t c = lvl[lev] + gw; c < lvl[lev + 1]; c += nwarps) warp_expand_cell(a, c, ovf);
    g.sync();
  }
}

// ---- M2L (fmm.zig:561-610) and the unscale of L (fmm.zig:645-657) --------------------

__global__ void __launch_bounds__(FMM_THREADS) k_fmm_m2l(FmmArgs a) {
  extern __shared__ double fmm_smem[];
  const unsigned lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t p = a.p, q = a.q, stride = a.stride, nt = 2 * p + 1;
  const uint32_t S = 32 / q;  // sources per step
  // per warp: T [S][2 nt], M [S][stride], C [S][stride]
  double *ws = fmm_smem + wl * (size_t)S * (2 * nt + 2 * stride);
  double *Ts = ws, *Ms = ws + S * 2 * nt, *Cs = Ms + S * stride;
  const uint32_t s = lane / q, l = lane % q;
  for (uint32_t c = gw; c < a.ncells; c += nwarps) {
    const double acx = a.cells[c].cx, acy = a.cells[c].cy;
    const uint32_t cnt = a.m2l_cnt[c], off = a.m2l_off[c];
    double acc_re = 0, acc_im = 0;
    for (uint32_t base = 0; base < cnt; base += S) {
      const uint32_t ns = min(S, cnt - base);
      if (lane < ns) {
        const uint32_t B = a.m2l[off + base + lane];
        const double dx = acx - a.cells[B].cx, dy = acy - a.cells[B].cy;
        const double d2 = dx * dx + dy * dy;
        const double ire = dx / d2, iim = -dy / d2;
        double are = ire, aim = iim;
        double *tr = Ts + lane * 2 * nt, *ti = tr + nt;
        tr[0] = are;
        ti[0] = aim;
        for (uint32_t mm = 1; mm < nt; ++mm) {
          const double nre = are * ire - aim * iim;
          const double nim = are * iim + aim * ire;
          are = nre;
          aim = nim;
          tr[mm] = are * a.tab->fact[mm];
          ti[mm] = aim * a.tab->fact[mm];
        }
      }
      for (uint32_t idx = lane; idx < ns * stride; idx += 32) {
        const uint32_t ss = idx / stride, r = idx % stride;
        const uint32_t B = a.m2l[off + base + ss];
        Ms[ss * stride + r] = a.mco[(size_t)B * stride + r];
      }
      __syncwarp();
      if (s < ns) {
        const double *tr = Ts + s * 2 * nt, *ti = tr + nt;
        const double *mre = Ms + s * stride, *mim = mre + q;
        double v0re = 0, v1re = 0, v0im = 0, v1im = 0;
        uint32_t k = 0;
        for (; k + 2 <= q; k += 2) {
          v0re += mre[k] * tr[l + k] - mim[k] * ti[l + k];
          v1re += mre[k + 1] * tr[l + k + 1] - mim[k + 1] * ti[l + k + 1];
          v0im += mre[k] * ti[l + k] + mim[k] * tr[l + k];
          v1im += mre[k + 1] * ti[l + k + 1] + mim[k + 1] * tr[l + k + 1];
        }
        double sre = v0re + v1re, sim = v0im + v1im;
        if (k < q) {
          sre += mre[k] * tr[l + k] - mim[k] * ti[l + k];
          sim += mre[k] * ti[l + k] + mim[k] * tr[l + k];
        }
        Cs[s * stride + l] = sre;
        Cs[s * stride + q + l] = sim;
      }
      __syncwarp();
      if (lane < q) {
        for (uint32_t t = 0; t < ns; ++t) {
          acc_re += Cs[t * stride + lane];
          acc_im += Cs[t * stride + q + lane];
        }
      }
      __syncwarp();
    }
    if (lane < q) {
      const double inv = ((lane & 1) ? -1.0 : 1.0) / a.tab->fact[lane];
      double *L = a.lco + (size_t)c * stride;
      L[lane] = acc_re * inv;
      L[q + lane] = acc_im * inv;
    }
  }
}

// ---- P2P (fmm.zig:477-553) ------------------------------------------------------------

__device__ inline void fmm_pair(const FmmArgs &a, uint64_t seed, uint32_t ti, uint32_t tj, double xi,
                                double yi, double &vx, double &vy) {
  if (tj == ti) return;
  const double sj = a.ps[tj];
  double x = a.px[tj] - xi, y = a.py[tj] - yi;
  double l = x * x + y * y;
  if (l >= a.dmax2) return;
  if (x == 0 || y == 0) {
    const uint32_t i = a.perm[ti], j = a.perm[tj];
    if (x == 0) { x = hash_jiggle(seed, i, j, 0); l += x * x; }
    if (y == 0) { y = hash_jiggle(seed, i, j, 1); l += y * y; }
  }
  if (l < a.dmin2) l = sqrt(a.dmin2 * l);
  const double wj = sj / l;
  vx += x * wj;
  vy += y * wj;
}

// One target against sources [b0, b1), four pairs per division on two lanes
// (lane 0: k, k + 2; lane 1: k + 1, k + 3).
__device__ void fmm_target(const FmmArgs &a, uint64_t seed, uint32_t ti, uint32_t b0, uint32_t b1,
                           double xi, double yi, double &vxr, double &vyr) {
  double vx = vxr, vy = vyr;
  double ax0 = 0, ax1 = 0, ay0 = 0, ay1 = 0;
  uint32_t k = b0;
  for (; k + 4 <= b1; k += 4) {
    const double sa0 = a.ps[k], sa1 = a.ps[k + 1], sb0 = a.ps[k + 2], sb1 = a.ps[k + 3];
    const double xa0 = a.px[k] - xi, xa1 = a.px[k + 1] - xi;
    const double ya0 = a.py[k] - yi, ya1 = a.py[k + 1] - yi;
    const double xb0 = a.px[k + 2] - xi, xb1 = a.px[k + 3] - xi;
    const double yb0 = a.py[k + 2] - yi, yb1 = a.py[k + 3] - yi;
    const double la0 = xa0 * xa0 + ya0 * ya0, la1 = xa1 * xa1 + ya1 * ya1;
    const double lb0 = xb0 * xb0 + yb0 * yb0, lb1 = xb1 * xb1 + yb1 * yb1;
    const double z0 = xa0 * ya0 * xb0 * yb0, z1 = xa1 * ya1 * xb1 * yb1;
    const double mn = zmin(zmin(la0, lb0), zmin(la1, lb1));
    if (z0 == 0 || z1 == 0 || !(mn >= a.dmin2) || (ti >= k && ti < k + 4)) {
      for (uint32_t u = 0; u < 4; ++u) fmm_pair(a, seed, ti, k + u, xi, yi, vx, vy);
      continue;
    }
    const double pa0 = la0 * la1, pa1 = la1 * la0;
    const double pb0 = lb0 * lb1, pb1 = lb1 * lb0;
    const double inv0 = 1 / (pa0 * pb0), inv1 = 1 / (pa1 * pb1);
    double wa0 = sa0 * la1 * pb0 * inv0, wa1 = sa1 * la0 * pb1 * inv1;
    double wb0 = sb0 * lb1 * pa0 * inv0, wb1 = sb1 * lb0 * pa1 * inv1;
    if (a.has_dmax) {
      if (!(la0 < a.dmax2)) wa0 = 0;
      if (!(la1 < a.dmax2)) wa1 = 0;
      if (!(lb0 < a.dmax2)) wb0 = 0;
      if (!(lb1 < a.dmax2)) wb1 = 0;
    }
    ax0 += xa0 * wa0 + xb0 * wb0;
    ax1 += xa1 * wa1 + xb1 * wb1;
    ay0 += ya0 * wa0 + yb0 * wb0;
    ay1 += ya1 * wa1 + yb1 * wb1;
  }
  for (; k < b1; ++k) fmm_pair(a, seed, ti, k, xi, yi, vx, vy);
  vxr = vx + (ax0 + ax1);
  vyr = vy + (ay0 + ay1);
}

__global__ void __launch_bounds__(FMM_THREADS, 4) k_fmm_p2p(FmmArgs a) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint64_t seed = (uint64_t)__double_as_longlong(*a.seed);
  for (uint32_t c = gw; c < a.ncells; c += nwarps) {
    const uint32_t cnt = a.p2p_cnt[c];
    if (!cnt) continue;
    const uint32_t off = a.p2p_off[c], first = a.cells[c].first, count = a.cells[c].count;
    for (uint32_t base = first; base < first + count; base += 32) {
      const uint32_t ti = base + lane;
      if (ti >= first + count) continue;
      const uint32_t i = a.perm[ti];
      const double xi = a.px[ti], yi = a.py[ti];
      double vx = a.vx[i], vy = a.vy[i];
      for (uint32_t e = 0; e < cnt; ++e) {
        const uint32_t B = a.p2p[off + e];
        const uint32_t b0 = a.cells[B].first, b1 = b0 + a.cells[B].count;
        fmm_target(a, seed, ti, b0, b1, xi, yi, vx, vy);
      }
      a.vx[i] = vx;
      a.vy[i] = vy;
    }
  }
}

// ---- downward: L2L (fmm.zig:823-849), L2P (fmm.zig:853-886) ---------------------------

__global__ void __launch_bounds__(FMM_THREADS) k_fmm_down(FmmArgs a) {
  extern __shared__ double fmm_smem[];
  cg::grid_group g = cg::this_grid();
  const unsigned lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t p = a.p, q = a.q, stride = a.stride;
  double *ws = fmm_smem + (threadIdx.x >> 5) * 2 * (size_t)stride;  // L of the cell, then powers
  double *Lw = ws, *pw = ws + stride;
  const uint32_t *lvl = a.info + FI_LVL;
  for (uint32_t lev = 0; lev < a.nlev; ++lev) {
    for (uint32_t c = lvl[lev] + gw; c < lvl[lev + 1]; c += nwarps) {
      const double cx = a.cells[c].cx, cy = a.cells[c].cy;
      const uint32_t nchild = a.cells[c].nchild, child0 = a.cells[c].child0;
      for (uint32_t r = lane; r < stride; r += 32) Lw[r] = ldg_cg(&a.lco[(size_t)c * stride + r]);
      __syncwarp();
      if (nchild == 0) {
        const uint32_t first = a.cells[c].first, count = a.cells[c].count;
        for (uint32_t k = first + lane; k < first + count; k += 32) {
          const uint32_t j = a.perm[k];
          const double wre = a.ux[k] - cx, wim = a.uy[k] - cy;
          double are = Lw[p], aim = Lw[q + p];
          for (uint32_t l = p; l > 0;) {
            --l;
            const double nre = are * wre - aim * wim + Lw[l];
            const double nim = are * wim + aim * wre + Lw[q + l];
            are = nre;
            aim = nim;
          }
          a.vx[j] = a.vx[j] - are * a.inv_w;
          a.vy[j] = a.vy[j] + aim * a.inv_w;
        }
      } else {
        for (uint32_t ch = child0; ch < child0 + nchild; ++ch) {
          if (lane == 0) shift_powers(a.cells[ch].cx - cx, a.cells[ch].cy - cy, p, pw);
          __syncwarp();
          const uint32_t mm = lane;
          if (mm < q) {
            double sre = 0, sim = 0;
            for (uint32_t l = mm; l < q; ++l) {
              const double b = a.tab->binom[l * FMM_TAB + mm];
              const double xre = Lw[l] * b, xim = Lw[q + l] * b;
              sre += xre * pw[l - mm] - xim * pw[q + l - mm];
              sim += xre * pw[q + l - mm] + xim * pw[l - mm];
            }
            double *C = a.lco + (size_t)ch * stride;
            C[mm] = C[mm] + sre;
            C[q + mm] = C[q + mm] + sim;
          }
          __syncwarp();
        }
      }
      __syncwarp();
    }
    g.sync();
  }
}

// ---- host ------------------------------------------------------------------------------

// Makes p hold at least `need` elements, with headroom so a slowly growing
// need does not reallocate every run.
template <typename T>
int grow(T *&p, size_t &cap, size_t need) {
  if (need <= cap && p) return 0;
  cudaFree(p);
  p = nullptr;
  cap = need + need / 2;
  D3_CUDA_OK(cudaMalloc(&p, cap * sizeof(T)));
  return 0;
}

int fmm_reserve_points(FmmDev &f, uint32_t n) {
  if (n <= f.pcap && f.pcap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  cudaFree(f.px); cudaFree(f.py); cudaFree(f.ps); cudaFree(f.ux); cudaFree(f.uy);
  D3_CUDA_OK(cudaMalloc(&f.px, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.py, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.ps, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.ux, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.uy, cap * 8ull));
  cudaFree(f.pt_levels);
  D3_CUDA_OK(cudaMalloc(&f.pt_levels, cap * 2ull));
  f.pcap = cap;
  return 0;
}

int fmm_reserve_cells(FmmDev &f, uint32_t ccap) {
  if (ccap <= f.ccap && f.ccap) return 0;
  cudaFree(f.cells); cudaFree(f.bx0); cudaFree(f.by0); cudaFree(f.bx1); cudaFree(f.by1);
  cudaFree(f.m2l_off); cudaFree(f.m2l_cnt); cudaFree(f.p2p_off);
  cudaFree(f.p2p_cnt); cudaFree(f.fwd_off); cudaFree(f.fwd_cnt);
  D3_CUDA_OK(cudaMalloc(&f.cells, ccap * sizeof(FCell)));
  D3_CUDA_OK(cudaMalloc(&f.bx0, ccap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.by0, ccap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.bx1, ccap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.by1, ccap * 8ull));
  D3_CUDA_OK(cudaMalloc(&f.m2l_off, ccap * 4ull));
  D3_CUDA_OK(cudaMalloc(&f.m2l_cnt, ccap * 4ull));
  D3_CUDA_OK(cudaMalloc(&f.p2p_off, ccap * 4ull));
  D3_CUDA_OK(cudaMalloc(&f.p2p_cnt, ccap * 4ull));
  D3_CUDA_OK(cudaMalloc(&f.fwd_off, ccap * 4ull));
  D3_CUDA_OK(cudaMalloc(&f.fwd_cnt, ccap * 4ull));
  f.ccap = ccap;
  return 0;
}

void fmm_free(FastScratch &s) {
  FmmDev *f = static_cast<FmmDev *>(s.fmm);
  if (!f) return;
  cudaFree(f->px); cudaFree(f->py); cudaFree(f->ps); cudaFree(f->ux); cudaFree(f->uy);
  cudaFree(f->pt_levels);
  cudaFree(f->cells); cudaFree(f->bx0); cudaFree(f->by0); cudaFree(f->bx1); cudaFree(f->by1);
  cudaFree(f->m2l_off); cudaFree(f->m2l_cnt); cudaFree(f->p2p_off);
  cudaFree(f->p2p_cnt); cudaFree(f->fwd_off); cudaFree(f->fwd_cnt); cudaFree(f->m2l);
  cudaFree(f->p2p); cudaFree(f->fwd); cudaFree(f->mco); cudaFree(f->lco); cudaFree(f->tab);
  cudaFree(f->info); cudaFree(f->bsum); cudaFree(f->square); cudaFree(f->geom);
  cudaFree(f->cb_count); cudaFree(f->start_of); cudaFree(f->level_of);
  cudaFreeHost(f->h_info); cudaFreeHost(f->h_geom);
  delete f;
  s.fmm = nullptr;
}

static int coop_launch(const void *fn, int blocks, size_t smem, FmmArgs &args, cudaStream_t st) {
  void *params[] = {&args};
  ++g_launches;
  return cudaLaunchCooperativeKernel(fn, blocks, FMM_THREADS, params, smem, st) == cudaSuccess ? 0
                                                                                                  : -1;
}

static int sync_read(FmmDev &f, cudaStream_t st) {
  if (cudaMemcpyAsync(f.h_info, f.info, 64 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -1;
  return 0;
}

int fmm_prepare(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
                double alpha, FmmPrep &out, cudaStream_t st) {
  const uint32_t n = a.n;
  if (!s.fmm) {
    FmmDev *f = new FmmDev();
    s.fmm = f;
    D3_CUDA_OK(cudaMalloc(&f->info, 64 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(f->info, 0, 64 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMalloc(&f->square, 4 * sizeof(double)));
    D3_CUDA_OK(cudaMalloc(&f->tab, sizeof(FmmTables)));
    D3_CUDA_OK(cudaMalloc(&f->geom, 4 * sizeof(double)));
    D3_CUDA_OK(cudaHostAlloc(&f->h_info, 64 * sizeof(uint32_t), cudaHostAllocDefault));
    D3_CUDA_OK(cudaHostAlloc(&f->h_geom, 8 * sizeof(double), cudaHostAllocDefault));
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // the largest dynamic shared memory any of the kernels asks for (order 24)
    const size_t smax = FMM_WARPS * 32 * (size_t)(2 * (FMM_MAX_ORDER + 1)) * 8;
    cudaFuncSetAttribute(k_fmm_upward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
    cudaFuncSetAttribute(k_fmm_m2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
    int per_up = 0, per_lists = 0, per_down = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_up, k_fmm_upward, FMM_THREADS, smax);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_lists, k_fmm_lists, FMM_THREADS, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_down, k_fmm_down, FMM_THREADS,
                                                  FMM_WARPS * 2 * (size_t)(2 * (FMM_MAX_ORDER + 1)) * 8);
    per = per_up;
    if (per_lists < per) per = per_lists;
    if (per_down < per) per = per_down;
    if (per > 2) per = 2;
    if (per < 1) per = 1;
    f->coop_blocks = sms * per;
    D3_CUDA_OK(cudaMalloc(&f->bsum, (size_t)f->coop_blocks * 4));
  }
  FmmDev &f = *static_cast<FmmDev *>(s.fmm);
  if (fmm_reserve_points(f, n)) return -1;
  // keys: square extent, quantised Morton keys, stable sort (NaN nodes last)
  fast_box(t, a.x, a.y, n, f.square, st);
  D3_LAUNCH(k_fmm_keys, blocks_for(n, 256), 256, 0, st)(a.x, a.y, n, f.square, t.keys, t.sv);
  SortScratch ss{t.keys_tmp, t.sv_tmp, t.hist, t.scan_part};
  radix_sort_u64(t.keys, t.sv, n, 0, 4, true, ss, st);
  // the geometry, the point count and the gather stay on the device: the
  // host reads them with the cell counts, in one synchronisation
  D3_LAUNCH(k_fmm_geom, 1, 1, 0, st)(t.extent, t.info, f.geom, f.info);
  D3_LAUNCH(k_fmm_gather, blocks_for(n, 256), 256, 0, st)(t.sv, a.x, a.y, strengths, f.info, alpha,
                                                          f.geom, f.px, f.py, f.ps, f.ux, f.uy);
  // cells (level order); grow and rebuild if they do not fit
  uint32_t want = 2 * (n / FMM_LEAF + 1) + 64;
  for (int attempt = 0;; ++attempt) {
    if (fmm_reserve_cells(f, want > f.ccap ? want : f.ccap)) return -1;
    {
      const uint32_t nb = (n + CB_THREADS - 1) / CB_THREADS;
      if (grow(f.cb_count, f.cb_count_cap, (size_t)nb * CB_LEVELS) ||
          grow(f.start_of, f.start_cap, (size_t)f.ccap) || grow(f.level_of, f.level_cap, (size_t)f.ccap))
        return -1;
      D3_LAUNCH(k_cells_count, nb, CB_THREADS, 0, st)(t.keys, f.info, f.cb_count, f.pt_levels);
      D3_LAUNCH(k_cells_scan, CB_LEVELS, 1024, 0, st)(f.cb_count, nb, f.info);
      D3_LAUNCH(k_cells_starts, 1, 32, 0, st)(f.ccap, f.info);
      D3_LAUNCH(k_cells_place, nb, CB_THREADS, 0, st)(f.pt_levels, f.cb_count, f.info, f.start_of,
                                                    f.level_of);
      D3_LAUNCH(k_cells_fill, blocks_for(f.ccap, CB_THREADS), CB_THREADS, 0, st)(
          t.keys, f.start_of, f.level_of, f.info, f.cells);
    }
    if (cudaMemcpyAsync(f.h_geom, f.geom, 4 * sizeof(double), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        sync_read(f, st))
      return -1;
    if (f.h_info[FI_BAD]) return 0;  // the exact kernel runs instead
    if (!f.h_info[FI_M]) return 2;   // nothing to do (tree.zig:287-309 with an empty box)
    if (!f.h_info[FI_OVERFLOW]) break;
    if (attempt > 8) return -1;
    want = 2 * f.h_info[FI_OVERFLOW] + 64;
  }
  const uint32_t m = f.h_info[FI_M];
  const double w = f.h_geom[0], inv_w = f.h_geom[1], ox = f.h_geom[2], oy = f.h_geom[3];
  out.m = m;
  out.ncells = f.h_info[FI_CELLS];
  out.nlev = f.h_info[FI_LEVELS];
  for (uint32_t d = 0; d <= out.nlev && d < FMM_LEVELS + 2; ++d) out.lvl[d] = f.h_info[FI_LVL + d];
  out.w = w;
  out.inv_w = inv_w;
  out.ox = ox;
  out.oy = oy;
  out.keys = t.keys;
  out.perm = t.sv;
  out.px = f.px; out.py = f.py; out.ps = f.ps; out.ux = f.ux; out.uy = f.uy;
  out.cells = f.cells;
  out.info = f.info;
  out.coop_blocks = f.coop_blocks;
  return 1;
}

int fmm_run(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
            const FmmParams &prm, const double *seed, uint32_t *status, cudaStream_t st) {
  (void)status;
  FmmPrep pr;
  const int pre = fmm_prepare(s, t, a, strengths, prm.alpha, pr, st);
  if (pre == 2) return 1;
  if (pre <= 0) return pre;
  FmmDev &f = *static_cast<FmmDev *>(s.fmm);
  const uint32_t m = pr.m;
  (void)m;
  const double w = pr.w;
  uint32_t p = FMM_DEFAULT_ORDER;
  if (prm.order >= 1 && prm.order <= (double)FMM_MAX_ORDER) p = (uint32_t)prm.order;
  double kappa = prm.opening;
  if (!(kappa > 1)) kappa = FMM_DEFAULT_OPENING;
  if (f.tab_p != p) {
    // fmm.zig:223-238
    FmmTables h;
    memset(&h, 0, sizeof h);
    const size_t nmax = 2 * p + 2;
    for (size_t nn = 0; nn < nmax; ++nn) {
      h.binom[nn * FMM_TAB] = 1;
      for (size_t k = 1; k <= nn; ++k)
        h.binom[nn * FMM_TAB + k] =
            h.binom[(nn - 1) * FMM_TAB + k - 1] + (k < nn ? h.binom[(nn - 1) * FMM_TAB + k] : 0);
    }
    h.fact[0] = 1;
    for (size_t k = 1; k < nmax; ++k) h.fact[k] = h.fact[k - 1] * (double)k;
    if (cudaMemcpyAsync(f.tab, &h, sizeof h, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return -1;
    f.tab_p = p;
  }
  const uint32_t q = p + 1, stride = 2 * q;
  FmmArgs args;
  memset(&args, 0, sizeof args);
  args.keys = t.keys;
  args.perm = t.sv;
  args.px = f.px; args.py = f.py; args.ps = f.ps; args.ux = f.ux; args.uy = f.uy;
  args.tab = f.tab;
  args.vx = a.vx; args.vy = a.vy;
  args.info = f.info;
  args.p = p; args.q = q; args.stride = stride;
  args.inv_w = pr.inv_w;
  args.mac_far = 2 * kappa - 1;
  double dmax_scaled = INFINITY;
  if (prm.dmax2 < INFINITY) dmax_scaled = sqrt(prm.dmax2) / w;
  const double dmin_scaled = prm.dmin2 > 0 ? sqrt(prm.dmin2) / w : 0;
  args.dmax_scaled = dmax_scaled;
  args.dmin_scaled = dmin_scaled;
  args.ring = dmin_scaled > 0 || dmax_scaled < INFINITY;
  args.has_dmax = dmax_scaled < INFINITY;
  args.dmin2 = prm.dmin2;
  args.dmax2 = prm.dmax2;
  args.seed = seed;
  const uint32_t ncells = pr.ncells, nlev = pr.nlev;
  args.cells = f.cells;
  args.bx0 = f.bx0; args.by0 = f.by0; args.bx1 = f.bx1; args.by1 = f.by1;
  args.ncells = ncells;
  args.nlev = nlev;
  if ((size_t)ncells * stride > f.coef_cap || !f.mco) {
    cudaFree(f.mco);
    cudaFree(f.lco);
    f.mco = f.lco = nullptr;
    f.coef_cap = (size_t)ncells * stride + (size_t)ncells * stride / 4;
    D3_CUDA_OK(cudaMalloc(&f.mco, f.coef_cap * 8));
    D3_CUDA_OK(cudaMalloc(&f.lco, f.coef_cap * 8));
  }
  args.mco = f.mco;
  args.lco = f.lco;
  args.m2l_off = f.m2l_off; args.m2l_cnt = f.m2l_cnt;
  args.p2p_off = f.p2p_off; args.p2p_cnt = f.p2p_cnt;
  args.fwd_off = f.fwd_off; args.fwd_cnt = f.fwd_cnt;
  const size_t smem_up = FMM_WARPS * 32 * (size_t)stride * 8;
  if (coop_launch((const void *)k_fmm_upward, f.coop_blocks, smem_up, args, st)) return -1;
  // interaction lists; grow the pools and redo on overflow
  // first guesses from the cell count, then what the previous run needed
  size_t need_m2l = (size_t)ncells * 48 + 1024, need_p2p = (size_t)ncells * 16 + 1024,
         need_fwd = (size_t)ncells * 16 + 1024;
  if (f.last_m2l) {
    need_m2l = f.last_m2l + f.last_m2l / 4 + 1024;
    need_p2p = f.last_p2p + f.last_p2p / 4 + 1024;
    need_fwd = f.last_fwd + f.last_fwd / 4 + 1024;
  }
  for (int attempt = 0;; ++attempt) {
    if (grow(f.m2l, f.cap_m2l, need_m2l) || grow(f.p2p, f.cap_p2p, need_p2p) ||
        grow(f.fwd, f.cap_fwd, need_fwd))
      return -1;
    args.m2l = f.m2l; args.p2p = f.p2p; args.fwd = f.fwd;
    args.cap_m2l = f.cap_m2l; args.cap_p2p = f.cap_p2p; args.cap_fwd = f.cap_fwd;
    if (cudaMemsetAsync(f.info + FI_POOL_M2L, 0, 5 * sizeof(uint32_t), st) != cudaSuccess) return -1;
    if (coop_launch((const void *)k_fmm_lists, f.coop_blocks, 0, args, st)) return -1;
    if (sync_read(f, st)) return -1;
    const uint32_t ovf = f.h_info[FI_LIST_OVERFLOW] | f.h_info[FI_LIST_OVERFLOW + 1];
    if (!ovf) {
      f.last_m2l = f.h_info[FI_POOL_M2L];
      f.last_p2p = f.h_info[FI_POOL_P2P];
      f.last_fwd = f.h_info[FI_POOL_FWD];
      break;
    }
    if ((ovf & 2) || attempt > 8) return -1;  // a call stack overflowed
    need_m2l = 2 * (size_t)(f.h_info[FI_POOL_M2L] > need_m2l ? f.h_info[FI_POOL_M2L] : need_m2l);
    need_p2p = 2 * (size_t)(f.h_info[FI_POOL_P2P] > need_p2p ? f.h_info[FI_POOL_P2P] : need_p2p);
    need_fwd = 2 * (size_t)(f.h_info[FI_POOL_FWD] > need_fwd ? f.h_info[FI_POOL_FWD] : need_fwd);
  }
  const uint32_t S = 32 / q;
  const size_t smem_m2l = FMM_WARPS * (size_t)S * (2 * (2 * p + 1) + 2 * stride) * 8;
  const unsigned wblocks = blocks_for((size_t)ncells * 32, FMM_THREADS);
  D3_LAUNCH(k_fmm_m2l, wblocks, FMM_THREADS, smem_m2l, st)(args);
  D3_LAUNCH(k_fmm_p2p, wblocks, FMM_THREADS, 0, st)(args);
  const size_t smem_down = FMM_WARPS * 2 * (size_t)stride * 8;
  if (coop_launch((const void *)k_fmm_down, f.coop_blocks, smem_down, args, st)) return -1;
  return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

}  // namespace d3
