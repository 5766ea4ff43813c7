// tree.cu — d3-quadtree-identical tree build on the device.
//
// d3's tree is a function of the extent and the point set: a quadrant is a
// leaf exactly when all its points coincide (tree.zig:1-22). The build:
//   1. bounding box with addAll's first-wins comparisons, then d3's `cover`
//      (tree.zig:148-187, 230-248, 316-340);
//   2. 32-level Morton keys by d3's own midpoint test (tree.zig:252-284);
//   3. stable sort of the keys (three LSD radix passes on the top 24 bits, then
//      a rank within each run of equal top bits), then a stable partition that
//      moves points with a NaN coordinate last (they are left out of the tree);
//   4. cells in closed form: every cell is identified by (first sorted point,
//      depth); cells starting at point k have consecutive depths d0..leaf, so
//      cell index = base[k] + depth - d0 with base the exclusive scan of the
//      per-point cell counts. This is d3's `visit` preorder (children 0..3).
//   5. below the 32 key levels (distinct points in one key) the reference's
//      stable midpoint partition runs serially per group (tree.zig:449-479).
#include <cooperative_groups.h>

#include <cstdlib>

#include "tree.cuh"

namespace cg = cooperative_groups;

namespace d3 {

// Loads of data that other blocks of the same launch wrote (through L2: L1 is
// not coherent across SMs).
__device__ inline uint64_t ldc(const uint64_t *p) { return __ldcg((const unsigned long long *)p); }
__device__ inline uint32_t ldc(const uint32_t *p) { return __ldcg(p); }
__device__ inline int8_t ldc(const int8_t *p) { return (int8_t)__ldcg((const signed char *)p); }
__device__ inline uint8_t ldc(const uint8_t *p) { return (uint8_t)__ldcg((const unsigned char *)p); }

struct BoxPart {
  double v[4];   // min x, min y, max x, max y
  uint32_t i[4]; // index of the point that set each
  uint32_t m;    // points without a NaN coordinate
  uint32_t pad;
};

static_assert(sizeof(BoxPart) <= 64, "box partials are reserved at 64 bytes each");

static constexpr unsigned BOX_THREADS = 256;
static constexpr unsigned BOX_BLOCKS_MAX = 592;  // 4 per SM

// Minimum / maximum with the serial scan's rule: strict comparison, so on a
// tie (+0 / -0) the lower index wins.
__device__ inline bool better_min(double a, uint32_t ia, double b, uint32_t ib) {
  return a < b || (a == b && ia < ib);
}
__device__ inline bool better_max(double a, uint32_t ia, double b, uint32_t ib) {
  return a > b || (a == b && ia < ib);
}

__device__ inline void box_merge(double *v, uint32_t *ix, uint32_t &m, const double *v2,
                                 const uint32_t *i2, uint32_t m2) {
  if (better_min(v2[0], i2[0], v[0], ix[0])) { v[0] = v2[0]; ix[0] = i2[0]; }
  if (better_min(v2[1], i2[1], v[1], ix[1])) { v[1] = v2[1]; ix[1] = i2[1]; }
  if (better_max(v2[2], i2[2], v[2], ix[2])) { v[2] = v2[2]; ix[2] = i2[2]; }
  if (better_max(v2[3], i2[3], v[3], ix[3])) { v[3] = v2[3]; ix[3] = i2[3]; }
  m += m2;
}

// The block's merged box (every thread gets it): warp shuffles, then the
// warps' results by warp 0 (the merge is commutative and associative).
__device__ void block_box_reduce(double *v, uint32_t *ix, uint32_t &m) {
  __shared__ double sv[BOX_THREADS / 32][4];
  __shared__ uint32_t si[BOX_THREADS / 32][4];
  __shared__ uint32_t sm[BOX_THREADS / 32];
  const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  auto warp_reduce = [&]() {
    for (int o = 16; o > 0; o >>= 1) {
      double v2[4];
      uint32_t i2[4];
      for (int q = 0; q < 4; ++q) {
        v2[q] = __shfl_down_sync(0xffffffffu, v[q], o);
        i2[q] = __shfl_down_sync(0xffffffffu, ix[q], o);
      }
      const uint32_t m2 = __shfl_down_sync(0xffffffffu, m, o);
      if (lane + o < 32) box_merge(v, ix, m, v2, i2, m2);
    }
  };
  warp_reduce();
  if (lane == 0) {
    for (int q = 0; q < 4; ++q) {
      sv[w][q] = v[q];
      si[w][q] = ix[q];
    }
    sm[w] = m;
  }
  __syncthreads();
  if (w == 0) {
    if (lane < nw) {
      for (int q = 0; q < 4; ++q) {
        v[q] = sv[lane][q];
        ix[q] = si[lane][q];
      }
      m = sm[lane];
    } else {
      v[0] = v[1] = INFINITY;
      v[2] = v[3] = -INFINITY;
      for (int q = 0; q < 4; ++q) ix[q] = NONE;
      m = 0;
    }
    warp_reduce();
    if (lane == 0) {
      for (int q = 0; q < 4; ++q) {
        sv[0][q] = v[q];
        si[0][q] = ix[q];
      }
      sm[0] = m;
    }
  }
  __syncthreads();
  for (int q = 0; q < 4; ++q) {
    v[q] = sv[0][q];
    ix[q] = si[0][q];
  }
  m = sm[0];
  __syncthreads();
}

// d3-quadtree's cover (tree.zig:148-187).
__device__ void cover(double *e, double x, double y) {
  if (isnan(x) || isnan(y)) return;
  double x0 = e[0], y0 = e[1], x1 = e[2], y1 = e[3];
  if (isnan(x0)) {
    x0 = floor(x);
    x1 = x0 + 1;
    y0 = floor(y);
    y1 = y0 + 1;
  } else {
    double z = x1 - x0;
    if (z == 0 || z != z) z = 1;
    uint32_t guard = 0;
    while ((x0 > x || x >= x1 || y0 > y || y >= y1) && guard < MAX_DEPTH) {
      int i = ((y < y0) << 1) | (x < x0);
      z *= 2;
      switch (i) {
        case 0: x1 = x0 + z; y1 = y0 + z; break;
        case 1: x0 = x1 - z; y1 = y0 + z; break;
        case 2: x1 = x0 + z; y0 = y1 - z; break;
        default: x0 = x1 - z; y0 = y1 - z; break;
      }
      ++guard;
    }
  }
  e[0] = x0; e[1] = y0; e[2] = x1; e[3] = y1;
}

// The bounding box of the points without a NaN coordinate. Exact mode
// (square == nullptr): d3's cover of the box into `extent`. Fast mode: the
// square of tree.zig:287-309 (side = the larger of width and height, 1 when
// that is not positive) into `extent`, and box x0, y0 and side into square[].
__global__ void __launch_bounds__(BOX_THREADS) k_box(const double *xs, const double *ys, uint32_t n,
                                                     BoxPart *parts, double *extent, uint32_t *info,
                                                     double *square) {
  double v[4] = {INFINITY, INFINITY, -INFINITY, -INFINITY};
  uint32_t ix[4] = {NONE, NONE, NONE, NONE};
  uint32_t m = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x = xs[i], y = ys[i];
    if (x != x || y != y) continue;
    double pv[4] = {x, y, x, y};
    uint32_t pi[4] = {i, i, i, i};
    box_merge(v, ix, m, pv, pi, 1);
  }
  block_box_reduce(v, ix, m);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    BoxPart p;
    for (int q = 0; q < 4; ++q) { p.v[q] = v[q]; p.i[q] = ix[q]; }
    p.m = m;
    parts[blockIdx.x] = p;
    __threadfence();
    last = atomicAdd(&info[4], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a[4] = {INFINITY, INFINITY, -INFINITY, -INFINITY};
  uint32_t ai[4] = {NONE, NONE, NONE, NONE};
  uint32_t am = 0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    const volatile BoxPart *p = &parts[b];
    double pv[4];
    uint32_t pi[4];
    for (int q = 0; q < 4; ++q) { pv[q] = p->v[q]; pi[q] = p->i[q]; }
    box_merge(a, ai, am, pv, pi, p->m);
  }
  block_box_reduce(a, ai, am);
  if (threadIdx.x == 0) {
    info[4] = 0;
    double e[4] = {NAN, NAN, NAN, NAN};
    info[0] = am;
    if (!(a[0] > a[2] || a[1] > a[3])) {
      if (square) {
        const double w = a[2] - a[0], h = a[3] - a[1];
        double side = w > h ? w : h;
        if (!(side > 0)) side = 1;
        e[0] = a[0]; e[1] = a[1]; e[2] = a[0] + side; e[3] = a[1] + side;
        square[0] = a[0]; square[1] = a[1]; square[2] = side;
      } else {
        cover(e, a[0], a[1]);
        cover(e, a[2], a[3]);
      }
    }
    for (int q = 0; q < 4; ++q) extent[q] = e[q];
    info[1] = 0;
    info[2] = 0;
    info[3] = am ? 0 : NONE;
    info[5] = 0;
  }
}

// tree.zig:252-284: 32-level key by d3's midpoint test; the sort value carries
// bit 31 for points with a NaN coordinate (partitioned last).
__device__ void keys_at(uint32_t i, const double *xs, const double *ys, const double *extent,
                        uint64_t *keys, uint32_t *sv) {
  double x = xs[i], y = ys[i];
  if (x != x || y != y) {
    keys[i] = 0;
    sv[i] = i | 0x80000000u;
    return;
  }
  double x0 = extent[0], y0 = extent[1], x1 = extent[2], y1 = extent[3];
  uint64_t key = 0;
#pragma unroll 4
  for (int lv = 0; lv < KEY_LEVELS; ++lv) {
    double xm = (x0 + x1) / 2;
    double ym = (y0 + y1) / 2;
    bool right = x >= xm;
    if (right) x0 = xm; else x1 = xm;
    bool bottom = y >= ym;
    if (bottom) y0 = ym; else y1 = ym;
    key = (key << 2) | ((uint64_t)bottom << 1) | (uint64_t)right;
  }
  keys[i] = key;
  sv[i] = i;
}

// perm (sorted node indices, then the NaN nodes in index order), and per
// sorted point the levels its key shares with the previous one: -1 for the
// first, 64 for the same position (no boundary), else min(32, clz / 2).
__device__ void runs_at(uint32_t k, uint32_t m, const double *xs, const double *ys,
                        const uint64_t *keys, const uint32_t *sv, uint32_t *perm, int8_t *lcpx,
                        uint32_t *leaf_of) {
  uint32_t p = ldc(&sv[k]) & 0x7fffffffu;
  perm[k] = p;
  if (k >= m) {
    leaf_of[p] = NONE;
    return;
  }
  if (k == 0) {
    lcpx[0] = -1;
    return;
  }
  uint32_t q = ldc(&sv[k - 1]) & 0x7fffffffu;
  if (xs[p] == xs[q] && ys[p] == ys[q]) {
    lcpx[k] = 64;
    return;
  }
  uint64_t d = ldc(&keys[k]) ^ ldc(&keys[k - 1]);
  int l = d ? (__clzll(d) >> 1) : 32;
  lcpx[k] = (int8_t)(l < 32 ? l : 32);
}

__device__ inline bool is_start(const int8_t *lcpx, uint32_t k) {
  int l = ldc(&lcpx[k]);
  return k == 0 || l < 32;  // -1 only at k = 0; 32 and 64 are not starts
}

// Bounds of the cell at depth d on key's path (tree.zig:482-499 applied d times).
__device__ inline void path_bounds(const double *extent, uint64_t key, int d, double &x0, double &y0,
                                   double &x1, double &y1) {
  x0 = extent[0]; y0 = extent[1]; x1 = extent[2]; y1 = extent[3];
  for (int lv = 0; lv < d; ++lv) {
    uint32_t dg = (uint32_t)(key >> (62 - 2 * lv)) & 3u;
    double xm = (x0 + x1) / 2;
    double ym = (y0 + y1) / 2;
    if (dg & 1) x0 = xm; else x1 = xm;
    if (dg & 2) y0 = ym; else y1 = ym;
  }
}

__device__ inline int quadrant(double x, double y, double xm, double ym) {
  return ((y >= ym) << 1) | (x >= xm);
}

// The reference's serial build below the key resolution, on one group of
// equal keys [lo, hi) whose depth-32 cell is `c32` (tree.zig:449-479, 505-549).
// count mode (write = false) returns the number of cells below depth 32;
// write mode emits them from c32 + 1 in preorder and sets their skip indices.
// Frames live in frames[4 lo, 4 hi): at most one frame per point is pending.
__device__ uint32_t deep_group(bool write, uint32_t lo, uint32_t hi, uint32_t c32, uint64_t key,
                               const double *extent, const double *xs, const double *ys,
                               uint32_t *perm, uint32_t *perm_tmp, Frame *frames, Cell *cells,
                               uint32_t *parent, uint8_t *pnch, uint32_t *skip, uint32_t skip_after,
                               uint32_t *depth_out, uint32_t *leaf_of) {
  Frame *stack = frames + 4 * (size_t)lo;
  const uint32_t cap = 4 * (hi - lo);
  uint32_t sp = 0, emitted = 0, maxd = 32;
  Frame f32;
  f32.lo = lo; f32.hi = hi; f32.depth = 32; f32.parent = c32; f32.slot = 0;
  path_bounds(extent, key, 32, f32.x0, f32.y0, f32.x1, f32.y1);
  uint32_t next = c32 + 1;
  bool first = true;
  Frame f = f32;
  for (;;) {
    if (!first) {
      if (sp == 0) break;
      f = stack[--sp];
      uint32_t me = next++;
      ++emitted;
      if (f.depth > maxd) maxd = f.depth;
      if (write) {
        Cell c;
        c.child[0] = c.child[1] = c.child[2] = c.child[3] = NONE;
        c.first = f.lo; c.count = f.hi - f.lo;
        c.x0 = f.x0; c.y0 = f.y0; c.x1 = f.x1; c.y1 = f.y1;
        c.x = c.y = c.value = c.r = 0;
        cells[me] = c;
        cells[f.parent].child[f.slot] = me;
        parent[me] = f.parent;
        pnch[me] = (uint8_t)f.pad;
      }
      f.parent = me;
      // allSame by position (tree.zig:437-444); the depth guard of tree.zig:33
      bool same = true;
      uint32_t p0 = ldc(&perm[f.lo]);
      for (uint32_t k = f.lo + 1; k < f.hi; ++k) {
        uint32_t p = ldc(&perm[k]);
        if (xs[p] != xs[p0] || ys[p] != ys[p0]) { same = false; break; }
      }
      if (f.depth >= MAX_DEPTH || same) {
        if (write)
          for (uint32_t k = f.lo; k < f.hi; ++k) leaf_of[ldc(&perm[k])] = me;
        continue;
      }
    }
    first = false;
    // split: stable partition of perm[lo, hi) by the midpoint quadrant
    double xm = (f.x0 + f.x1) / 2, ym = (f.y0 + f.y1) / 2;
    uint32_t counts[4] = {0, 0, 0, 0}, off[4], b[5];
    for (uint32_t k = f.lo; k < f.hi; ++k) {
      uint32_t p = ldc(&perm[k]);
      counts[quadrant(xs[p], ys[p], xm, ym)]++;
    }
    uint32_t sum = f.lo;
    for (int q = 0; q < 4; ++q) { off[q] = sum; b[q] = sum; sum += counts[q]; }
    b[4] = f.hi;
    for (uint32_t k = f.lo; k < f.hi; ++k) {
      uint32_t p = ldc(&perm[k]);
      perm_tmp[off[quadrant(xs[p], ys[p], xm, ym)]++] = p;
    }
    for (uint32_t k = f.lo; k < f.hi; ++k) perm[k] = ldc(&perm_tmp[k]);
    uint32_t nq = 0;
    for (int q = 0; q < 4; ++q) nq += b[q] != b[q + 1];
    for (int q = 3; q >= 0; --q) {
      if (b[q] == b[q + 1]) continue;
      if (sp >= cap) return emitted;  // cannot happen: pending frames hold disjoint points
      Frame c;
      c.lo = b[q]; c.hi = b[q + 1]; c.depth = f.depth + 1; c.parent = f.parent; c.slot = q;
      c.pad = nq;  // the parent's child count
      bool right = q & 1, bottom = q & 2;
      c.x0 = right ? xm : f.x0; c.y0 = bottom ? ym : f.y0;
      c.x1 = right ? f.x1 : xm; c.y1 = bottom ? f.y1 : ym;
      stack[sp++] = c;
    }
  }
  if (write) {
    // skip: the first later cell of the group starting at or past the end
    uint32_t end_idx = c32 + 1 + emitted;
    for (uint32_t c = c32 + 1; c < end_idx; ++c) {
      uint32_t e = cells[c].first + cells[c].count, j = c + 1;
      while (j < end_idx && cells[j].first < e) ++j;
      skip[c] = j < end_idx ? j : skip_after;
    }
  }
  if (depth_out) atomicMax(depth_out, maxd);
  return emitted;
}

// Cells starting at each sorted point: per start k, depths d0..leaf, plus the
// cells below depth 32 of a deep group.
__device__ void count_at(uint32_t k, uint32_t m, const double *xs, const double *ys,
                         const uint64_t *keys, const int8_t *lcpx, const double *extent,
                         uint32_t *perm, uint32_t *perm_tmp, Frame *frames, uint32_t *cnt,
                         uint32_t *run_end, uint8_t *leafd) {
  if (k >= m) {
    cnt[k] = 0;  // points with a NaN coordinate start no cell
    return;
  }
  if (!is_start(lcpx, k)) {
    cnt[k] = 0;
    return;
  }
  int d0 = k == 0 ? 0 : ldc(&lcpx[k]) + 1;
  uint32_t j = k + 1;
  while (j < m && ldc(&lcpx[j]) == 64) ++j;
  int lr = j < m ? ldc(&lcpx[j]) : -1;
  if (lr < 32) {
    int ld = lr + 1 > d0 ? lr + 1 : d0;
    leafd[k] = (uint8_t)ld;
    run_end[k] = j;
    cnt[k] = (uint32_t)(ld - d0 + 1);
    return;
  }
  uint32_t g1 = j;
  while (g1 < m && ldc(&lcpx[g1]) >= 32) ++g1;
  leafd[k] = 33;
  run_end[k] = g1;
  uint32_t deep = deep_group(false, k, g1, 0, ldc(&keys[k]), extent, xs, ys, perm, perm_tmp, frames,
                             nullptr, nullptr, nullptr, nullptr, 0, nullptr, nullptr);
  cnt[k] = (uint32_t)(32 - d0 + 1) + deep;
}

// First index in [lo, hi) with keys[j] >= t (keys sorted). Plain loads: the
// keys are final by the cells phase, and the grid barrier before it orders
// their writes before these reads (these searches hit L1 on their upper steps).
__device__ inline uint32_t lower_bound(const uint64_t *keys, uint32_t lo, uint32_t hi, uint64_t t) {
  while (lo < hi) {
    uint32_t mid = lo + ((hi - lo) >> 1);
    if (keys[mid] < t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// First index in [lo, hi) whose key's top 2d bits differ from pk (d >= 1),
// given that keys[lo] has them: doubling steps from lo, then bisection (the
// cost grows with the log of the cell's size, not of the array's).
__device__ inline uint32_t prefix_end(const uint64_t *keys, uint32_t lo, uint32_t hi, uint64_t pk,
                                      int d) {
  const int sh = 64 - 2 * d;
  uint32_t ok = lo, step = 1;
  for (;;) {
    const uint32_t probe = ok + step;
    if (probe >= hi || (keys[probe] >> sh) != pk) {
      hi = probe < hi ? probe : hi;
      break;
    }
    ok = probe;
    step <<= 1;
  }
  uint32_t l = ok + 1;
  while (l < hi) {
    uint32_t mid = l + ((hi - l) >> 1);
    if ((keys[mid] >> sh) == pk) l = mid + 1; else hi = mid;
  }
  return l;
}

// lower_bound by a whole warp (all lanes, same arguments): 32 probes a round.
__device__ uint32_t warp_lower_bound(const uint64_t *keys, uint32_t lo, uint32_t hi, uint64_t t) {
  const unsigned lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const uint32_t step = (hi - lo + 31) / 32;
    const uint32_t pos = lo + lane * step;
    const unsigned ge = __ballot_sync(0xffffffffu, pos >= hi || keys[pos] >= t);
    if (ge & 1u) return lo;
    const uint32_t f = ge ? (uint32_t)__ffs(ge) - 1 : 32;  // the first probe with keys >= t
    const uint32_t nhi = f == 32 ? hi : min(hi, lo + f * step);
    lo = lo + (f - 1) * step + 1;
    hi = nhi;
  }
  const uint32_t pos = lo + lane;
  const unsigned ge = __ballot_sync(0xffffffffu, pos >= hi || keys[pos] >= t);
  return ge ? min(hi, lo + (uint32_t)__ffs(ge) - 1) : hi;
}

// Cells at depths below TB_TOP_D (at most 85) search the whole point range:
// whole warps emit them.
constexpr int TB_TOP_D = 4;

// Cell emission, one thread per cell. A start k owns cells base[k] +
// (0 .. dlast - d0) (depths d0 .. dlast); `owner[c]` = k | OWN_TAG for those
// (below-resolution cells of a deep group stay NONE: the thread of the group's
// depth-32 cell emits them after it).
constexpr uint32_t OWN_TAG = 0x80000000u;

__device__ void own_at(uint32_t k, uint32_t m, const int8_t *lcpx, const uint32_t *base,
                       const uint32_t *cnt, const uint8_t *leafd, uint32_t *owner, uint32_t *info,
                       uint32_t *top) {
  if (!is_start(lcpx, k)) return;
  const int d0 = k == 0 ? 0 : ldc(&lcpx[k]) + 1;
  const int ld = ldc(&leafd[k]);
  const int dlast = ld == 33 ? 32 : ld;
  const uint32_t c0 = ldc(&base[k]);
  for (int d = d0; d <= dlast; ++d) owner[c0 + (d - d0)] = k | OWN_TAG;
  for (int d = d0; d <= dlast && d < TB_TOP_D; ++d) top[atomicAdd(&info[8], 1u)] = c0 + (d - d0);
  const uint32_t chain = (uint32_t)(dlast - d0 + 1), all = ldc(&cnt[k]);
  for (uint32_t c = c0 + chain; c < c0 + all; ++c) owner[c] = NONE;
  atomicMax(&info[2], (uint32_t)dlast);
}

template <bool WARP>
__device__ void emit_cell(uint32_t c, uint32_t m, uint32_t total, const double *xs, const double *ys,
                          const uint64_t *keys, const int8_t *lcpx, const double *extent,
                          uint32_t *perm, uint32_t *perm_tmp, Frame *frames, const uint32_t *base,
                          const uint32_t *run_end, const uint8_t *leafd, Cell *cells, uint32_t *skip,
                          uint32_t *parent, uint8_t *pnch, uint32_t *counter, uint32_t *info,
                          uint32_t *leaf_of) {
  const uint32_t own = ldc(&counter[c]);
  if (own == NONE || !(own & OWN_TAG)) return;
  const uint32_t k = own & ~OWN_TAG;
  const uint64_t key = ldc(&keys[k]);
  const int d0 = k == 0 ? 0 : ldc(&lcpx[k]) + 1;
  const int ld = ldc(&leafd[k]);
  const bool deep = ld == 33;
  const uint32_t c0 = ldc(&base[k]);
  const int d = d0 + (int)(c - c0);
  if (!WARP && d < TB_TOP_D) return;  // a top cell: emitted by a warp
  const bool writer = !WARP || (threadIdx.x & 31) == 0;
  const uint32_t rend = ldc(&run_end[k]);
  double x0, y0, x1, y1;
  path_bounds(extent, key, d, x0, y0, x1, y1);
  if (c == 0 && writer) {
    parent[0] = NONE;
    pnch[0] = 0;  // the root has no parent
  }
  const bool leaf = !deep && d == ld;
  uint32_t end;
  if (leaf || (deep && d == 32)) {
    end = rend;
  } else if (d == 0) {
    end = m;
  } else if (WARP) {
    const uint64_t pk = key >> (64 - 2 * d);
    end = pk + 1 < (1ull << (2 * d)) ? warp_lower_bound(keys, k, m, (pk + 1) << (64 - 2 * d)) : m;
  } else {
    end = prefix_end(keys, k, m, key >> (64 - 2 * d), d);
  }
  Cell cell;
  cell.child[0] = cell.child[1] = cell.child[2] = cell.child[3] = NONE;
  cell.first = k;
  cell.count = end - k;
  cell.x0 = x0; cell.y0 = y0; cell.x1 = x1; cell.y1 = y1;
  cell.x = cell.y = cell.value = cell.r = 0;
  const uint32_t sk = end < m ? ldc(&base[end]) : total;
  if (writer) skip[c] = sk;
  if (!leaf && d < 32) {
    const uint64_t top = d == 0 ? 0 : (key >> (64 - 2 * d)) << (64 - 2 * d);
    uint32_t b[5];
    b[0] = k;
    b[4] = end;
    for (uint32_t q = 1; q < 4; ++q) {
      const uint64_t t = top | ((uint64_t)q << (62 - 2 * d));
      b[q] = WARP ? warp_lower_bound(keys, b[q - 1], end, t) : lower_bound(keys, b[q - 1], end, t);
    }
    if (!writer) return;
    uint8_t nch = 0;
    for (int q = 0; q < 4; ++q) nch += b[q] != b[q + 1];
    for (int q = 0; q < 4; ++q) {
      if (b[q] == b[q + 1]) continue;
      uint32_t a = b[q];
      int cd0 = a == k ? d0 : ldc(&lcpx[a]) + 1;
      uint32_t ch = ldc(&base[a]) + (uint32_t)(d + 1 - cd0);
      cell.child[q] = ch;
      parent[ch] = c;
      pnch[ch] = nch;
    }
  }
  if (!writer) return;
  cells[c] = cell;
  counter[c] = 0;
  if (leaf)
    for (uint32_t p = k; p < rend; ++p) leaf_of[ldc(&perm[p])] = c;
  if (deep && d == 32) {
    const uint32_t after = rend < m ? ldc(&base[rend]) : total;
    const uint32_t emitted = deep_group(true, k, rend, c, key, extent, xs, ys, perm, perm_tmp,
                                        frames, cells, parent, pnch, skip, after, &info[2], leaf_of);
    for (uint32_t q = c + 1; q <= c + emitted; ++q) counter[q] = 0;
  }
}

// ---- the build as one cooperative launch --------------------------------------

constexpr unsigned TB_THREADS = 256;
constexpr unsigned TB_TILE = 256;  // keys per sort tile (one per thread)

struct TreeBuildArgs {
  const double *xs, *ys;
  const double *vxs, *vys;  // if set, the points are (xs + vxs, ys + vys), written to pxs, pys
  double *pxs, *pys;
  uint32_t n, tiles, cells_cap;
  uint64_t *keys, *keys_tmp;
  uint32_t *sv, *sv_tmp, *perm, *perm_tmp;
  int8_t *lcpx;
  uint32_t *cnt, *base, *run_end;
  uint8_t *leafd;
  Frame *frames;
  Cell *cells;
  uint32_t *skip, *parent, *counter, *leaf_of;
  uint8_t *pnch;
  BoxPart *parts;
  uint32_t *hist, *hist2;  // tiles * 256 per-tile digit counts, two passes' worth
  uint32_t *dtot, *bsum;   // 256 digit totals, grid partials
  double *extent;
  uint32_t *info, *status;
  unsigned long long *stamps;  // globaltimer at the phase ends (block 0)
};

__device__ inline void tb_stamp(const TreeBuildArgs &a, int k) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    a.stamps[k] = t;
  }
}

template <bool PART>
__device__ inline uint32_t tb_digit(uint64_t k, uint32_t v, int shift) {
  if (PART) return v >> 31;
  return (uint32_t)(k >> shift) & 255u;
}

// The digit of the pass after `shift` (next < 0: the NaN partition).
__device__ inline uint32_t tb_next_digit(uint64_t k, uint32_t v, int next) {
  return next < 0 ? v >> 31 : (uint32_t)(k >> next) & 255u;
}

// One stable LSD pass from (ik, iv) to (ok, ov), given `cur`: per tile
// (TB_TILE keys) the counts of each digit, tile-major. Phase 1: per digit (a
// block each) the exclusive prefix of its counts over the tiles, and the
// digit totals; the other blocks clear `nxt` (if clear). Phase 2: the
// scatter, in which a key's rank among equal digits of its tile = earlier
// warps' counts + lanes below it in its warp with the same digit (warp
// match); each key also counts its digit of the next pass (`next`, if
// has_next) into `nxt` at its new tile. Two grid barriers.
template <bool PART>
__device__ void tb_sort_pass(cg::grid_group &g, const TreeBuildArgs &a, const uint64_t *ik,
                             const uint32_t *iv, uint64_t *ok, uint32_t *ov, int shift,
                             uint32_t *cur, uint32_t *nxt, bool has_next, int next, bool clear) {
  __shared__ uint32_t h[256];
  __shared__ uint32_t wcnt[TB_THREADS / 32][256];
  __shared__ uint32_t sw[32];
  const unsigned t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t n = a.n, tiles = a.tiles;
  const uint32_t tid = blockIdx.x * blockDim.x + t, nth = gridDim.x * blockDim.x;
  for (uint32_t d = blockIdx.x; d < 256; d += gridDim.x) {
    uint32_t run = 0;
    for (uint32_t t0 = 0; t0 < tiles; t0 += TB_THREADS) {
      const uint32_t tt = t0 + t;
      const uint32_t x = tt < tiles ? ldc(&cur[(size_t)tt * 256 + d]) : 0;
      uint32_t tot;
      const uint32_t ex = block_excl(x, sw, tot);
      if (tt < tiles) cur[(size_t)tt * 256 + d] = run + ex;
      run += tot;
    }
    if (t == 0) a.dtot[d] = run;
  }
  if (clear)
    for (uint32_t i = tid; i < tiles * 256; i += nth) nxt[i] = 0;
  g.sync();
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    uint32_t tot;
    const uint32_t dbase = block_excl(ldc(&a.dtot[t]), sw, tot);
    h[t] = dbase + ldc(&cur[(size_t)tile * 256 + t]);
    for (int k = t; k < 256 * (TB_THREADS / 32); k += blockDim.x) (&wcnt[0][0])[k] = 0;
    __syncthreads();
    const uint32_t i = tile * TB_TILE + t;
    const bool valid = i < n;
    const uint64_t k = valid ? ldc(&ik[i]) : 0;
    const uint32_t v = valid ? ldc(&iv[i]) : 0;
    const uint32_t d = valid ? tb_digit<PART>(k, v, shift) : 256u + lane;  // never matches
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned below = __popc(peers & ((1u << lane) - 1));
    if (valid && below == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t before = 0;
      for (unsigned w = 0; w < warp; ++w) before += wcnt[w][d];
      const uint32_t pos = h[d] + before + below;
      ok[pos] = k;
      ov[pos] = v;
      if (has_next) atomicAdd(&nxt[(size_t)(pos / TB_TILE) * 256 + tb_next_digit(k, v, next)], 1u);
    }
    __syncthreads();
  }
  g.sync();
}

constexpr uint32_t TB_RUN_MAX = 256;

// The sorted place of point k (of keys, vals sorted by the top 24 key bits)
// within its run of equal top bits, by the rest of the key and then the
// point index: written to (ok, ov); returns it. A run longer than TB_RUN_MAX
// sets *flag instead (and returns NONE).
__device__ uint32_t tb_run_rank(const uint64_t *keys, const uint32_t *vals, uint32_t n, uint32_t k,
                                uint64_t *ok, uint32_t *ov, uint32_t *flag) {
  constexpr uint64_t LOW = (1ull << 40) - 1;
  const uint64_t key = ldc(&keys[k]);
  const uint32_t v = ldc(&vals[k]);
  const uint64_t top = key >> 40, low = key & LOW;
  const uint32_t idx = v & 0x7fffffffu;
  uint32_t s = k, e = k + 1;
  while (s > 0 && k - s < TB_RUN_MAX && (ldc(&keys[s - 1]) >> 40) == top) --s;
  while (e < n && e - s <= TB_RUN_MAX && (ldc(&keys[e]) >> 40) == top) ++e;
  if (e - s > TB_RUN_MAX) {
    atomicOr(flag, 1u);
    return NONE;
  }
  uint32_t rank = 0;
  for (uint32_t j = s; j < e; ++j) {
    const uint64_t lj = ldc(&keys[j]) & LOW;
    const uint32_t ij = ldc(&vals[j]) & 0x7fffffffu;
    rank += lj < low || (lj == low && ij < idx);
  }
  const uint32_t pos = s + rank;
  ok[pos] = key;
  ov[pos] = v;
  return pos;
}

// The tree build's cooperative launch did not happen.
__global__ void k_tree_failed(uint32_t *info, uint32_t *status) {
  info[1] = 0;
  info[5] = 0xffffffffu;
  if (status) atomicOr(status, ST_LAUNCH_FAILED);
}

__global__ void __launch_bounds__(TB_THREADS) k_tree_build(TreeBuildArgs a) {
  cg::grid_group g = cg::this_grid();
  __shared__ double se[4];
  __shared__ uint32_t sm_m;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t n = a.n;
  tb_stamp(a, 0);
  // 1. the box: block partials, then every block merges all of them (the
  //    first-wins merge is order independent, so every block gets the same)
  {
    double v[4] = {INFINITY, INFINITY, -INFINITY, -INFINITY};
    uint32_t ix[4] = {NONE, NONE, NONE, NONE};
    uint32_t m = 0;
    for (uint32_t i = tid; i < n; i += nth) {
      double x = a.xs[i], y = a.ys[i];
      if (a.vxs) {
        x += a.vxs[i];
        y += a.vys[i];
        a.pxs[i] = x;
        a.pys[i] = y;
      }
      if (x != x || y != y) continue;
      double pv[4] = {x, y, x, y};
      uint32_t pi[4] = {i, i, i, i};
      box_merge(v, ix, m, pv, pi, 1);
    }
    block_box_reduce(v, ix, m);
    if (threadIdx.x == 0) {
      BoxPart p;
      for (int q = 0; q < 4; ++q) { p.v[q] = v[q]; p.i[q] = ix[q]; }
      p.m = m;
      a.parts[blockIdx.x] = p;
    }
    for (uint32_t i = tid; i < a.tiles * 256; i += nth) a.hist[i] = 0;
  }
  g.sync();
  {
    double v[4] = {INFINITY, INFINITY, -INFINITY, -INFINITY};
    uint32_t ix[4] = {NONE, NONE, NONE, NONE};
    uint32_t m = 0;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
      const BoxPart *p = &a.parts[b];
      double pv[4];
      uint32_t pi[4];
      for (int q = 0; q < 4; ++q) {
        pv[q] = __ldcg(&p->v[q]);
        pi[q] = __ldcg(&p->i[q]);
      }
      box_merge(v, ix, m, pv, pi, __ldcg(&p->m));
    }
    block_box_reduce(v, ix, m);
    if (threadIdx.x == 0) {
      double e[4] = {NAN, NAN, NAN, NAN};
      if (!(v[0] > v[2] || v[1] > v[3])) {
        cover(e, v[0], v[1]);
        cover(e, v[2], v[3]);
      }
      for (int q = 0; q < 4; ++q) se[q] = e[q];
      sm_m = m;
      if (blockIdx.x == 0) {
        for (int q = 0; q < 4; ++q) a.extent[q] = e[q];
        a.info[0] = m;
        a.info[1] = 0;
        a.info[2] = 0;
        a.info[3] = m ? 0 : NONE;
        a.info[4] = 0;
        a.info[5] = 0;
        a.info[7] = 0;
        a.info[8] = 0;
      }
    }
    __syncthreads();
  }
  const uint32_t m = sm_m;
  if (n == 0) return;
  // the points: as given, or shifted by the velocities in the box phase
  const double *X = a.vxs ? a.pxs : a.xs, *Y = a.vxs ? a.pys : a.ys;
  // 2. keys, and the first sort pass's digit counts (cleared above)
  tb_stamp(a, 1);
  for (uint32_t i = tid; i < n; i += nth) {
    keys_at(i, X, Y, se, a.keys, a.sv);
    atomicAdd(&a.hist[(size_t)(i / TB_TILE) * 256 + (uint32_t)((a.keys[i] >> 40) & 255u)], 1u);
  }
  g.sync();
  tb_stamp(a, 2);
  // 3. the stable sort by key, then the NaN partition if any point has one:
  //    three LSD passes on the top 24 key bits; then each run of equal top
  //    bits (normally one to three points) is ordered by the rest of the key
  //    and the point index, each point placed by its rank in its run. If a run
  //    is longer than TB_RUN_MAX, the 8 full LSD passes run on the top-sorted
  //    order instead (still stable: equal keys keep index order in a run).
  const bool part = m < n;
  tb_sort_pass<false>(g, a, a.keys, a.sv, a.keys_tmp, a.sv_tmp, 40, a.hist, a.hist2, true, 48, true);
  tb_sort_pass<false>(g, a, a.keys_tmp, a.sv_tmp, a.keys, a.sv, 48, a.hist2, a.hist, true, 56, true);
  tb_sort_pass<false>(g, a, a.keys, a.sv, a.keys_tmp, a.sv_tmp, 56, a.hist, a.hist2, false, 0, true);
  for (uint32_t k = tid; k < n; k += nth) {
    const uint32_t pos = tb_run_rank(a.keys_tmp, a.sv_tmp, n, k, a.keys, a.sv, &a.info[7]);
    if (part && pos != NONE)
      atomicAdd(&a.hist2[(size_t)(pos / TB_TILE) * 256 + (ldc(&a.sv_tmp[k]) >> 31)], 1u);
  }
  for (uint32_t i = tid; i < a.tiles * 256; i += nth) a.hist[i] = 0;
  g.sync();
  uint64_t *fk = a.keys;  // the sorted keys and values
  uint32_t *fv = a.sv, *fh = a.hist2;
  if (ldc(&a.info[7])) {
    for (uint32_t k = tid; k < n; k += nth)
      atomicAdd(&a.hist[(size_t)(k / TB_TILE) * 256 + (uint32_t)(ldc(&a.keys_tmp[k]) & 255u)], 1u);
    g.sync();
    uint64_t *ak = a.keys_tmp, *bk = a.keys;
    uint32_t *av = a.sv_tmp, *bv = a.sv;
    uint32_t *hc = a.hist, *hn = a.hist2;
    for (int b = 0; b < 8; ++b) {
      const bool has_next = b < 7 || part;
      tb_sort_pass<false>(g, a, ak, av, bk, bv, 8 * b, hc, hn, has_next, b < 7 ? 8 * (b + 1) : -1,
                          has_next);
      uint64_t *tk = ak; ak = bk; bk = tk;
      uint32_t *tv = av; av = bv; bv = tv;
      uint32_t *th = hc; hc = hn; hn = th;
    }
    fk = ak;
    fv = av;
    fh = hc;
  }
  if (part) {
    uint64_t *ok = fk == a.keys ? a.keys_tmp : a.keys;
    uint32_t *ov = fv == a.sv ? a.sv_tmp : a.sv;
    tb_sort_pass<true>(g, a, fk, fv, ok, ov, 0, fh, nullptr, false, 0, false);
    fk = ok;
    fv = ov;
  }
  tb_stamp(a, 3);
  // 4. perm and the shared levels; 5. cells per start
  for (uint32_t k = tid; k < n; k += nth)
    runs_at(k, m, X, Y, fk, fv, a.perm, a.lcpx, a.leaf_of);
  g.sync();
  tb_stamp(a, 4);
  for (uint32_t k = tid; k < n; k += nth)
    count_at(k, m, X, Y, fk, a.lcpx, se, a.perm, a.perm_tmp, a.frames, a.cnt, a.run_end,
             a.leafd);
  g.sync();
  tb_stamp(a, 5);
  // 6. cell indices: the exclusive scan of the counts
  const uint32_t total = grid_excl_scan(g, a.cnt, a.base, n, a.bsum);
  // info[1] is the cell count every later pass walks: on overflow it stays 0
  // (an empty tree), so no pass reads or writes past the cell buffers;
  // info[6] keeps the count the tree needed.
  if (tid == 0) {
    a.info[1] = total <= a.cells_cap ? total : 0;
    a.info[6] = total;
  }
  g.sync();
  tb_stamp(a, 6);
  // 7. the cells
  if (total > a.cells_cap) {
    if (tid == 0) {
      a.info[5] = 1;
      atomicOr(a.status, ST_DEEP_STACK);
    }
    return;
  }
  uint32_t *top = reinterpret_cast<uint32_t *>(a.parts);  // the box partials are done with
  for (uint32_t k = tid; k < m; k += nth)
    own_at(k, m, a.lcpx, a.base, a.cnt, a.leafd, a.counter, a.info, top);
  g.sync();
  tb_stamp(a, 7);
  for (uint32_t c = tid; c < total; c += nth)
    emit_cell<false>(c, m, total, X, Y, fk, a.lcpx, se, a.perm, a.perm_tmp, a.frames, a.base,
                     a.run_end, a.leafd, a.cells, a.skip, a.parent, a.pnch, a.counter, a.info,
                     a.leaf_of);
  {
    const uint32_t ntop = ldc(&a.info[8]), gw = tid >> 5, nw = nth >> 5;
    for (uint32_t k = gw; k < ntop; k += nw)
      emit_cell<true>(ldc(&top[k]), m, total, X, Y, fk, a.lcpx, se, a.perm, a.perm_tmp,
                      a.frames, a.base, a.run_end, a.leafd, a.cells, a.skip, a.parent, a.pnch,
                      a.counter, a.info, a.leaf_of);
  }
  __syncthreads();
  tb_stamp(a, 8);  // block 0's cells only
}

int tree_reserve(TreeDev &t, uint32_t n) {
  if (!t.info) {
    D3_CUDA_OK(cudaMalloc(&t.info, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(t.info, 0, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMalloc(&t.extent, 4 * sizeof(double)));
    D3_CUDA_OK(cudaMalloc(&t.box_part, BOX_BLOCKS_MAX * sizeof(BoxPart)));
    D3_CUDA_OK(cudaMalloc(&t.stamps, 16 * sizeof(unsigned long long)));
    D3_CUDA_OK(cudaMemset(t.stamps, 0, 16 * sizeof(unsigned long long)));
  }
  if (n <= t.cap && t.cap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  cudaFree(t.keys); cudaFree(t.keys_tmp); cudaFree(t.sv); cudaFree(t.sv_tmp); cudaFree(t.perm);
  cudaFree(t.perm_tmp); cudaFree(t.lcpx); cudaFree(t.cnt); cudaFree(t.base); cudaFree(t.run_end);
  cudaFree(t.leafd); cudaFree(t.frames); cudaFree(t.cells); cudaFree(t.skip); cudaFree(t.parent);
  cudaFree(t.counter); cudaFree(t.scan_part); cudaFree(t.hist); cudaFree(t.leaf_of);
  cudaFree(t.pnch); cudaFree(t.rec);
  size_t cells = 4 * (size_t)cap + 1024;
  D3_CUDA_OK(cudaMalloc(&t.keys, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&t.keys_tmp, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&t.sv, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&t.sv_tmp, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&t.perm, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&t.perm_tmp, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&t.lcpx, cap));
  D3_CUDA_OK(cudaMalloc(&t.cnt, (cap + 1) * 4ull));
  D3_CUDA_OK(cudaMalloc(&t.base, (cap + 1) * 4ull));
  D3_CUDA_OK(cudaMalloc(&t.run_end, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&t.leafd, cap));
  D3_CUDA_OK(cudaMalloc(&t.frames, 4 * (size_t)cap * sizeof(Frame)));
  D3_CUDA_OK(cudaMalloc(&t.cells, cells * sizeof(Cell)));
  D3_CUDA_OK(cudaMalloc(&t.skip, cells * 4));
  D3_CUDA_OK(cudaMalloc(&t.parent, cells * 4));
  D3_CUDA_OK(cudaMalloc(&t.counter, cells * 4));
  D3_CUDA_OK(cudaMalloc(&t.pnch, cells));
  D3_CUDA_OK(cudaMalloc(&t.rec, cells * 64));
  D3_CUDA_OK(cudaMalloc(&t.leaf_of, cap * 4ull));
  size_t sp = scan_partial_words(sort_hist_words(cap) > cap + 1 ? sort_hist_words(cap) : cap + 1);
  D3_CUDA_OK(cudaMalloc(&t.scan_part, sp * 4));
  D3_CUDA_OK(cudaMalloc(&t.hist, tree_hist_words(cap) * 4));
  t.cap = cap;
  t.cells_cap = (uint32_t)cells;
  return 0;
}

void tree_free(TreeDev &t) {
  cudaFree(t.keys); cudaFree(t.keys_tmp); cudaFree(t.sv); cudaFree(t.sv_tmp); cudaFree(t.perm);
  cudaFree(t.perm_tmp); cudaFree(t.lcpx); cudaFree(t.cnt); cudaFree(t.base); cudaFree(t.run_end);
  cudaFree(t.leafd); cudaFree(t.frames); cudaFree(t.cells); cudaFree(t.skip); cudaFree(t.parent);
  cudaFree(t.counter); cudaFree(t.scan_part); cudaFree(t.hist); cudaFree(t.info);
  cudaFree(t.leaf_of); cudaFree(t.pnch); cudaFree(t.rec);
  cudaFree(t.extent); cudaFree(t.box_part); cudaFree(t.stamps);
  t = TreeDev();
}

void fast_box(TreeDev &t, const double *xs, const double *ys, uint32_t n, double *square,
              cudaStream_t st) {
  unsigned bb = blocks_for(n, BOX_THREADS * 4);
  if (bb > BOX_BLOCKS_MAX) bb = BOX_BLOCKS_MAX;
  D3_LAUNCH(k_box, bb, BOX_THREADS, 0, st)(xs, ys, n, (BoxPart *)t.box_part, t.extent, t.info,
                                           square);
}

static int g_tree_blocks = 0;

void tree_build(TreeDev &t, const double *xs, const double *ys, uint32_t n, uint32_t *status,
                cudaStream_t st) {
  tree_build_shifted(t, xs, ys, nullptr, nullptr, nullptr, nullptr, n, status, st);
}

void tree_build_shifted(TreeDev &t, const double *xs, const double *ys, const double *vxs,
                        const double *vys, double *pxs, double *pys, uint32_t n, uint32_t *status,
                        cudaStream_t st) {
  if (!g_tree_blocks) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tree_build, TB_THREADS, 0);
    // blocks per SM: at most 2, or D3_TREE_BLOCKS_PER_SM (1 .. occupancy)
    int want = per > 2 ? 2 : per;
    if (const char *e = getenv("D3_TREE_BLOCKS_PER_SM")) {
      const int v = atoi(e);
      if (v >= 1 && v <= per) want = v;
    }
    g_tree_blocks = sms * (want > 0 ? want : 1);
    if (g_tree_blocks > (int)TREE_GRID_MAX) g_tree_blocks = TREE_GRID_MAX;
  }
  TreeBuildArgs a;
  a.xs = xs; a.ys = ys; a.n = n;
  a.vxs = vxs; a.vys = vys; a.pxs = pxs; a.pys = pys;
  a.tiles = (n + TB_TILE - 1) / TB_TILE;
  a.cells_cap = t.cells_cap;
  a.keys = t.keys; a.keys_tmp = t.keys_tmp; a.sv = t.sv; a.sv_tmp = t.sv_tmp;
  a.perm = t.perm; a.perm_tmp = t.perm_tmp; a.lcpx = t.lcpx;
  a.cnt = t.cnt; a.base = t.base; a.run_end = t.run_end; a.leafd = t.leafd;
  a.frames = t.frames; a.cells = t.cells; a.skip = t.skip; a.parent = t.parent;
  a.counter = t.counter; a.leaf_of = t.leaf_of; a.pnch = t.pnch;
  a.parts = (BoxPart *)t.box_part;
  a.hist = t.hist;
  a.hist2 = t.hist + (size_t)a.tiles * 256;
  a.dtot = a.hist2 + (size_t)a.tiles * 256;
  a.bsum = a.dtot + 256;
  a.extent = t.extent; a.info = t.info; a.status = status;
  a.stamps = t.stamps;
  void *params[] = {&a};
  ++g_launches;
  if (cudaLaunchCooperativeKernel((const void *)k_tree_build, g_tree_blocks, TB_THREADS, params, 0,
                                  st) != cudaSuccess) {
    // report it: without the launch the cells, perm and leaf_of are stale,
    // so the passes that follow see an empty tree (info[1] = 0) and the
    // launch-failure mark (info[5] = 0xffffffff), which they check
    D3_LAUNCH(k_tree_failed, 1, 1, 0, st)(t.info, status);
  }
}

}  // namespace d3
