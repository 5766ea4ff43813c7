// tree.cu — d3-quadtree-identical tree build on the device.
//
// d3's tree is a function of the extent and the point set: a quadrant is a
// leaf exactly when all its points coincide (tree.zig:1-22). The build:
//   1. bounding box with addAll's first-wins comparisons, then d3's `cover`
//      (tree.zig:148-187, 230-248, 316-340);
//   2. 32-level Morton keys by d3's own midpoint test (tree.zig:252-284);
//   3. stable LSD radix sort of the keys, then a stable partition that moves
//      points with a NaN coordinate last (they are left out of the tree);
//   4. cells in closed form: every cell is identified by (first sorted point,
//      depth); cells starting at point k have consecutive depths d0..leaf, so
//      cell index = base[k] + depth - d0 with base the exclusive scan of the
//      per-point cell counts. This is d3's `visit` preorder (children 0..3).
//   5. below the 32 key levels (distinct points in one key) the reference's
//      stable midpoint partition runs serially per group (tree.zig:449-479).
#include "tree.cuh"

namespace d3 {

struct BoxPart {
  double v[4];   // min x, min y, max x, max y
  uint32_t i[4]; // index of the point that set each
  uint32_t m;    // points without a NaN coordinate
  uint32_t pad;
};

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

__device__ void block_box_reduce(double *v, uint32_t *ix, uint32_t &m) {
  __shared__ double sv[BOX_THREADS][4];
  __shared__ uint32_t si[BOX_THREADS][4];
  __shared__ uint32_t sm[BOX_THREADS];
  const unsigned t = threadIdx.x;
  for (int q = 0; q < 4; ++q) { sv[t][q] = v[q]; si[t][q] = ix[q]; }
  sm[t] = m;
  __syncthreads();
  for (unsigned s = BOX_THREADS / 2; s > 0; s >>= 1) {
    if (t < s) {
      double a[4];
      uint32_t ai[4];
      uint32_t am = sm[t];
      for (int q = 0; q < 4; ++q) { a[q] = sv[t][q]; ai[q] = si[t][q]; }
      box_merge(a, ai, am, sv[t + s], si[t + s], sm[t + s]);
      for (int q = 0; q < 4; ++q) { sv[t][q] = a[q]; si[t][q] = ai[q]; }
      sm[t] = am;
    }
    __syncthreads();
  }
  for (int q = 0; q < 4; ++q) { v[q] = sv[0][q]; ix[q] = si[0][q]; }
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
__global__ void k_keys(const double *xs, const double *ys, uint32_t n, const double *extent,
                       uint64_t *keys, uint32_t *sv) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
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
__global__ void k_runs(const double *xs, const double *ys, uint32_t n, const uint64_t *keys,
                       const uint32_t *sv, uint32_t *perm, int8_t *lcpx, const uint32_t *info,
                       uint32_t *leaf_of) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t p = sv[k] & 0x7fffffffu;
  perm[k] = p;
  uint32_t m = info[0];
  if (k >= m) {
    leaf_of[p] = NONE;
    return;
  }
  if (k == 0) {
    lcpx[0] = -1;
    return;
  }
  uint32_t q = sv[k - 1] & 0x7fffffffu;
  if (xs[p] == xs[q] && ys[p] == ys[q]) {
    lcpx[k] = 64;
    return;
  }
  uint64_t d = keys[k] ^ keys[k - 1];
  int l = d ? (__clzll(d) >> 1) : 32;
  lcpx[k] = (int8_t)(l < 32 ? l : 32);
}

__device__ inline bool is_start(const int8_t *lcpx, uint32_t k) {
  int l = lcpx[k];
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
                               uint32_t *parent, uint32_t *skip, uint32_t skip_after,
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
      }
      f.parent = me;
      // allSame by position (tree.zig:437-444); the depth guard of tree.zig:33
      bool same = true;
      uint32_t p0 = perm[f.lo];
      for (uint32_t k = f.lo + 1; k < f.hi; ++k) {
        uint32_t p = perm[k];
        if (xs[p] != xs[p0] || ys[p] != ys[p0]) { same = false; break; }
      }
      if (f.depth >= MAX_DEPTH || same) {
        if (write)
          for (uint32_t k = f.lo; k < f.hi; ++k) leaf_of[perm[k]] = me;
        continue;
      }
    }
    first = false;
    // split: stable partition of perm[lo, hi) by the midpoint quadrant
    double xm = (f.x0 + f.x1) / 2, ym = (f.y0 + f.y1) / 2;
    uint32_t counts[4] = {0, 0, 0, 0}, off[4], b[5];
    for (uint32_t k = f.lo; k < f.hi; ++k) {
      uint32_t p = perm[k];
      counts[quadrant(xs[p], ys[p], xm, ym)]++;
    }
    uint32_t sum = f.lo;
    for (int q = 0; q < 4; ++q) { off[q] = sum; b[q] = sum; sum += counts[q]; }
    b[4] = f.hi;
    for (uint32_t k = f.lo; k < f.hi; ++k) {
      uint32_t p = perm[k];
      perm_tmp[off[quadrant(xs[p], ys[p], xm, ym)]++] = p;
    }
    for (uint32_t k = f.lo; k < f.hi; ++k) perm[k] = perm_tmp[k];
    for (int q = 3; q >= 0; --q) {
      if (b[q] == b[q + 1]) continue;
      if (sp >= cap) return emitted;  // cannot happen: pending frames hold disjoint points
      Frame c;
      c.lo = b[q]; c.hi = b[q + 1]; c.depth = f.depth + 1; c.parent = f.parent; c.slot = q;
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
__global__ void k_count(const double *xs, const double *ys, const uint64_t *keys, const int8_t *lcpx,
                        const double *extent, uint32_t *perm, uint32_t *perm_tmp, Frame *frames,
                        uint32_t *cnt, uint32_t *run_end, uint8_t *leafd, const uint32_t *info,
                        uint32_t n) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t m = info[0];
  if (k >= m) {
    if (k < n) cnt[k] = 0;  // points with a NaN coordinate start no cell
    return;
  }
  if (!is_start(lcpx, k)) {
    cnt[k] = 0;
    return;
  }
  int d0 = k == 0 ? 0 : lcpx[k] + 1;
  uint32_t j = k + 1;
  while (j < m && lcpx[j] == 64) ++j;
  int lr = j < m ? lcpx[j] : -1;
  if (lr < 32) {
    int ld = lr + 1 > d0 ? lr + 1 : d0;
    leafd[k] = (uint8_t)ld;
    run_end[k] = j;
    cnt[k] = (uint32_t)(ld - d0 + 1);
    return;
  }
  uint32_t g1 = j;
  while (g1 < m && lcpx[g1] >= 32) ++g1;
  leafd[k] = 33;
  run_end[k] = g1;
  uint32_t deep = deep_group(false, k, g1, 0, keys[k], extent, xs, ys, perm, perm_tmp, frames,
                             nullptr, nullptr, nullptr, 0, nullptr, nullptr);
  cnt[k] = (uint32_t)(32 - d0 + 1) + deep;
}

// First index in [lo, hi) with keys[j] >= t (keys sorted).
__device__ inline uint32_t lower_bound(const uint64_t *keys, uint32_t lo, uint32_t hi, uint64_t t) {
  while (lo < hi) {
    uint32_t mid = lo + ((hi - lo) >> 1);
    if (keys[mid] < t) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// First index in [lo, hi) whose key's top 2d bits differ from pk (d >= 1).
__device__ inline uint32_t prefix_end(const uint64_t *keys, uint32_t lo, uint32_t hi, uint64_t pk,
                                      int d) {
  const int sh = 64 - 2 * d;
  while (lo < hi) {
    uint32_t mid = lo + ((hi - lo) >> 1);
    if ((keys[mid] >> sh) == pk) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void k_emit(const double *xs, const double *ys, const uint64_t *keys, const int8_t *lcpx,
                       const double *extent, uint32_t *perm, uint32_t *perm_tmp, Frame *frames,
                       const uint32_t *base, const uint32_t *run_end, const uint8_t *leafd,
                       Cell *cells, uint32_t *skip, uint32_t *parent, uint32_t *counter,
                       uint32_t cells_cap, uint32_t *info, uint32_t *status, uint32_t *leaf_of) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t m = info[0];
  uint32_t total = info[1];
  if (k >= m) return;
  if (total > cells_cap) {
    if (k == 0) { info[5] = 1; atomicOr(status, ST_DEEP_STACK); }
    return;
  }
  if (!is_start(lcpx, k)) return;
  const uint64_t key = keys[k];
  const int d0 = k == 0 ? 0 : lcpx[k] + 1;
  const int ld = leafd[k];
  const bool deep = ld == 33;
  const int dlast = deep ? 32 : ld;
  const uint32_t rend = run_end[k];
  double x0, y0, x1, y1;
  path_bounds(extent, key, d0, x0, y0, x1, y1);
  uint32_t c = base[k];
  if (k == 0) parent[0] = NONE;
  for (int d = d0; d <= dlast; ++d, ++c) {
    const bool leaf = !deep && d == ld;
    uint32_t end;
    if (leaf || (deep && d == 32)) end = rend;
    else if (d == 0) end = m;
    else end = prefix_end(keys, k, m, key >> (64 - 2 * d), d);
    Cell cell;
    cell.child[0] = cell.child[1] = cell.child[2] = cell.child[3] = NONE;
    cell.first = k;
    cell.count = end - k;
    cell.x0 = x0; cell.y0 = y0; cell.x1 = x1; cell.y1 = y1;
    cell.x = cell.y = cell.value = cell.r = 0;
    skip[c] = end < m ? base[end] : total;
    counter[c] = 0;
    if (!leaf && d < 32) {
      const uint64_t top = d == 0 ? 0 : (key >> (64 - 2 * d)) << (64 - 2 * d);
      uint32_t b[5];
      b[0] = k;
      b[4] = end;
      for (uint32_t q = 1; q < 4; ++q)
        b[q] = lower_bound(keys, b[q - 1], end, top | ((uint64_t)q << (62 - 2 * d)));
      for (int q = 0; q < 4; ++q) {
        if (b[q] == b[q + 1]) continue;
        uint32_t a = b[q];
        int cd0 = a == k ? d0 : lcpx[a] + 1;
        uint32_t ch = base[a] + (uint32_t)(d + 1 - cd0);
        cell.child[q] = ch;
        parent[ch] = c;
      }
    }
    cells[c] = cell;
    if (leaf)
      for (uint32_t p = k; p < rend; ++p) leaf_of[perm[p]] = c;
    // descend one level along the key
    uint32_t dg = (uint32_t)(key >> (62 - 2 * d)) & 3u;
    double xm = (x0 + x1) / 2, ym = (y0 + y1) / 2;
    if (dg & 1) x0 = xm; else x1 = xm;
    if (dg & 2) y0 = ym; else y1 = ym;
  }
  atomicMax(&info[2], (uint32_t)dlast);
  if (deep) {
    uint32_t c32 = base[k] + (uint32_t)(32 - d0);
    uint32_t after = rend < m ? base[rend] : total;
    uint32_t emitted = deep_group(true, k, rend, c32, key, extent, xs, ys, perm, perm_tmp, frames,
                                  cells, parent, skip, after, &info[2], leaf_of);
    for (uint32_t q = c32 + 1; q <= c32 + emitted; ++q) counter[q] = 0;
  }
}

int tree_reserve(TreeDev &t, uint32_t n) {
  if (!t.info) {
    D3_CUDA_OK(cudaMalloc(&t.info, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(t.info, 0, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMalloc(&t.extent, 4 * sizeof(double)));
    D3_CUDA_OK(cudaMalloc(&t.box_part, BOX_BLOCKS_MAX * sizeof(BoxPart)));
  }
  if (n <= t.cap && t.cap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  cudaFree(t.keys); cudaFree(t.keys_tmp); cudaFree(t.sv); cudaFree(t.sv_tmp); cudaFree(t.perm);
  cudaFree(t.perm_tmp); cudaFree(t.lcpx); cudaFree(t.cnt); cudaFree(t.base); cudaFree(t.run_end);
  cudaFree(t.leafd); cudaFree(t.frames); cudaFree(t.cells); cudaFree(t.skip); cudaFree(t.parent);
  cudaFree(t.counter); cudaFree(t.scan_part); cudaFree(t.hist); cudaFree(t.leaf_of);
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
  D3_CUDA_OK(cudaMalloc(&t.leaf_of, cap * 4ull));
  size_t sp = scan_partial_words(sort_hist_words(cap) > cap + 1 ? sort_hist_words(cap) : cap + 1);
  D3_CUDA_OK(cudaMalloc(&t.scan_part, sp * 4));
  D3_CUDA_OK(cudaMalloc(&t.hist, sort_hist_words(cap) * 4));
  t.cap = cap;
  t.cells_cap = (uint32_t)cells;
  return 0;
}

void tree_free(TreeDev &t) {
  cudaFree(t.keys); cudaFree(t.keys_tmp); cudaFree(t.sv); cudaFree(t.sv_tmp); cudaFree(t.perm);
  cudaFree(t.perm_tmp); cudaFree(t.lcpx); cudaFree(t.cnt); cudaFree(t.base); cudaFree(t.run_end);
  cudaFree(t.leafd); cudaFree(t.frames); cudaFree(t.cells); cudaFree(t.skip); cudaFree(t.parent);
  cudaFree(t.counter); cudaFree(t.scan_part); cudaFree(t.hist); cudaFree(t.info);
  cudaFree(t.leaf_of);
  cudaFree(t.extent); cudaFree(t.box_part);
  t = TreeDev();
}

void fast_box(TreeDev &t, const double *xs, const double *ys, uint32_t n, double *square,
              cudaStream_t st) {
  unsigned bb = blocks_for(n, BOX_THREADS * 4);
  if (bb > BOX_BLOCKS_MAX) bb = BOX_BLOCKS_MAX;
  D3_LAUNCH(k_box, bb, BOX_THREADS, 0, st)(xs, ys, n, (BoxPart *)t.box_part, t.extent, t.info,
                                           square);
}

void tree_build(TreeDev &t, const double *xs, const double *ys, uint32_t n, uint32_t *status,
                cudaStream_t st) {
  unsigned bb = blocks_for(n, BOX_THREADS * 4);
  if (bb > BOX_BLOCKS_MAX) bb = BOX_BLOCKS_MAX;
  D3_LAUNCH(k_box, bb, BOX_THREADS, 0, st)(xs, ys, n, (BoxPart *)t.box_part, t.extent, t.info,
                                           nullptr);
  if (n == 0) return;
  const unsigned T = 256, B = blocks_for(n, T);
  D3_LAUNCH(k_keys, B, T, 0, st)(xs, ys, n, t.extent, t.keys, t.sv);
  SortScratch ss{t.keys_tmp, t.sv_tmp, t.hist, t.scan_part};
  radix_sort_u64(t.keys, t.sv, n, 0, 8, true, ss, st);
  D3_LAUNCH(k_runs, B, T, 0, st)(xs, ys, n, t.keys, t.sv, t.perm, t.lcpx, t.info, t.leaf_of);
  D3_LAUNCH(k_count, B, T, 0, st)(xs, ys, t.keys, t.lcpx, t.extent, t.perm, t.perm_tmp, t.frames, t.cnt,
                           t.run_end, t.leafd, t.info, n);
  // cells before each start; the total lands in info[1]
  scan_u32(t.cnt, t.base, n, t.scan_part, t.info + 1, st);
  D3_LAUNCH(k_emit, B, T, 0, st)(xs, ys, t.keys, t.lcpx, t.extent, t.perm, t.perm_tmp, t.frames, t.base,
                          t.run_end, t.leafd, t.cells, t.skip, t.parent, t.counter, t.cells_cap,
                          t.info, status, t.leaf_of);
}

}  // namespace d3
