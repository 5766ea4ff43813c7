// fast.cu — fast-mode link (Jacobi sweep) and collide (uniform grid).
//
// Both are per-node Jacobi passes over a snapshot (link_fast.zig, grid.zig):
// every node writes only its own velocity, and each node's additions run in
// the reference's order (CSR row order; 3 x 3 cells, items by descending node
// index), so one thread per node reproduces the reference bit for bit.
#include <vector>

#include "fast.cuh"
#include "scan_sort.cuh"

namespace d3 {

constexpr uint32_t TARGET_BIT = 0x80000000u;
constexpr uint32_t NO_CELL = 0xffffffffu;
constexpr unsigned GRID_THREADS = 256;
constexpr unsigned GRID_BLOCKS_MAX = 592;

int fast_reserve(FastScratch &s, uint32_t n) {
  if (!s.seed) {
    D3_CUDA_OK(cudaMalloc(&s.seed, sizeof(double)));
    D3_CUDA_OK(cudaMalloc(&s.g_box, GRID_BLOCKS_MAX * 6 * sizeof(double)));
    D3_CUDA_OK(cudaMalloc(&s.g_info, 8 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(s.g_info, 0, 8 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMalloc(&s.g_geom, 4 * sizeof(double)));
  }
  if (n <= s.cap && s.cap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  cudaFree(s.g_keys); cudaFree(s.g_keys_tmp); cudaFree(s.g_items); cudaFree(s.g_items_tmp);
  cudaFree(s.g_cell_of); cudaFree(s.g_start); cudaFree(s.g_hist); cudaFree(s.g_part);
  D3_CUDA_OK(cudaMalloc(&s.g_keys, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.g_keys_tmp, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.g_items, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.g_items_tmp, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.g_cell_of, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.g_start, (4ull * cap + 24) * 4));
  D3_CUDA_OK(cudaMalloc(&s.g_hist, sort_hist_words(cap) * 4));
  D3_CUDA_OK(cudaMalloc(&s.g_part, scan_partial_words(sort_hist_words(cap)) * 4));
  s.cap = cap;
  return 0;
}

void fmm_free(FastScratch &s);

void fast_free(FastScratch &s) {
  cudaFree(s.seed); cudaFree(s.g_keys); cudaFree(s.g_keys_tmp); cudaFree(s.g_items);
  cudaFree(s.g_items_tmp); cudaFree(s.g_cell_of); cudaFree(s.g_start); cudaFree(s.g_hist);
  cudaFree(s.g_part); cudaFree(s.g_box); cudaFree(s.g_info); cudaFree(s.g_geom);
  fmm_free(s);
  fmm_tc_free(s);
  s = FastScratch();
}

__global__ void k_draw_seed(Rng *rng, double *seed) {
  uint32_t st = lcg_step(rng->lcg);
  rng->lcg = st;
  *seed = lcg_value(st);
}

__global__ void k_set_seed(double *seed, double v) { *seed = v; }

void draw_seed(Rng *rng, double *seed, cudaStream_t st) { D3_LAUNCH(k_draw_seed, 1, 1, 0, st)(rng, seed); }
void set_seed(double *seed, double value, cudaStream_t st) {
  D3_LAUNCH(k_set_seed, 1, 1, 0, st)(seed, value);
}

__device__ inline uint64_t seed_bits(const double *seed) {
  return (uint64_t)__double_as_longlong(*seed);
}

// ---- link_fast.zig --------------------------------------------------------

int fast_link_build(FastLink &c, const uint32_t *src, const uint32_t *tgt, uint32_t m, uint32_t n) {
  // link_fast.zig:105-130
  std::vector<uint32_t> row(n + 1, 0), adj(m ? 2 * (size_t)m : 1);
  for (uint32_t e = 0; e < m; ++e) {
    row[src[e] + 1]++;
    row[tgt[e] + 1]++;
  }
  for (uint32_t i = 1; i <= n; ++i) row[i] += row[i - 1];
  for (uint32_t e = 0; e < m; ++e) {
    adj[row[src[e] + 1] - 1] = e;
    row[src[e] + 1]--;
    adj[row[tgt[e] + 1] - 1] = e | TARGET_BIT;
    row[tgt[e] + 1]--;
  }
  for (uint32_t i = 0; i < n; ++i) row[i] = row[i + 1];
  row[n] = 2 * m;
  std::vector<uint32_t> other(adj.size(), 0);
  for (size_t a = 0; a < 2 * (size_t)m; ++a) {
    const uint32_t e = adj[a] & ~TARGET_BIT;
    other[a] = (adj[a] & TARGET_BIT) ? src[e] : tgt[e];
  }
  fast_link_free(c);
  D3_CUDA_OK(cudaMalloc(&c.row, row.size() * 4));
  D3_CUDA_OK(cudaMalloc(&c.adj, adj.size() * 4));
  D3_CUDA_OK(cudaMalloc(&c.other, other.size() * 4));
  D3_CUDA_OK(cudaMalloc(&c.scal, 3 * adj.size() * sizeof(double)));
  D3_CUDA_OK(cudaMemcpy(c.row, row.data(), row.size() * 4, cudaMemcpyHostToDevice));
  D3_CUDA_OK(cudaMemcpy(c.adj, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice));
  D3_CUDA_OK(cudaMemcpy(c.other, other.data(), other.size() * 4, cudaMemcpyHostToDevice));
  c.n = n;
  c.m = m;
  c.gathered = false;
  return 0;
}

void fast_link_free(FastLink &c) {
  cudaFree(c.row);
  cudaFree(c.adj);
  cudaFree(c.other);
  cudaFree(c.scal);
  c = FastLink();
}

// scal[plane * 2m + a] = the distance / strength / bias of entry a's link.
__global__ void k_link_gather(LinkArrays l, const uint32_t *adj, uint32_t entries, double *scal) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= entries) return;
  const uint32_t e = adj[a] & ~TARGET_BIT;
  scal[a] = l.distance[e];
  scal[(size_t)entries + a] = l.strength[e];
  scal[2 * (size_t)entries + a] = l.bias[e];
}

__global__ void k_shift2(const double *x, const double *y, const double *vx, const double *vy,
                         double *px, double *py, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  px[i] = x[i] + vx[i];
  py[i] = y[i] + vy[i];
}

// link_fast.zig:60-99. A thread per node over its adjacency in CSR order;
// the entries' other endpoints and link scalars are read from the
// adjacency-ordered copies (contiguous per node), four entries at a time
// with the position loads issued together, and applied in adjacency order as
// the serial loop does.
constexpr uint32_t LINK_BATCH = 4;

__global__ void k_link_sweep(const double *px, const double *py, double *vxs, double *vys,
                             const uint32_t *row, const uint32_t *adj, const uint32_t *other,
                             const double *scal, uint32_t entries, double alpha,
                             const double *seedp, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t seed = seed_bits(seedp);
  double vx = vxs[i], vy = vys[i];
  const double pxi = px[i], pyi = py[i];
  const uint32_t a1 = row[i + 1];
  for (uint32_t a0 = row[i]; a0 < a1; a0 += LINK_BATCH) {
    uint32_t ent[LINK_BATCH];
    double xj[LINK_BATCH], yj[LINK_BATCH];
#pragma unroll
    for (uint32_t k = 0; k < LINK_BATCH; ++k)
      if (a0 + k < a1) {
        ent[k] = adj[a0 + k];
        const uint32_t j = other[a0 + k];
        xj[k] = px[j];
        yj[k] = py[j];
      }
#pragma unroll
    for (uint32_t k = 0; k < LINK_BATCH; ++k) {
      const uint32_t a = a0 + k;
      if (a >= a1) break;
      const uint32_t e = ent[k] & ~TARGET_BIT;
      const bool is_target = (ent[k] & TARGET_BIT) != 0;
      double x = is_target ? pxi - xj[k] : xj[k] - pxi;
      double y = is_target ? pyi - yj[k] : yj[k] - pyi;
      if (x == 0 || x != x) x = hash_jiggle(seed, e, 0, 0);
      if (y == 0 || y != y) y = hash_jiggle(seed, e, 0, 1);
      double len = sqrt(x * x + y * y);
      len = (len - scal[a]) / len * alpha * scal[(size_t)entries + a];
      x *= len;
      y *= len;
      const double b = scal[2 * (size_t)entries + a];
      if (is_target) {
        vx -= x * b;
        vy -= y * b;
      } else {
        vx += x * (1 - b);
        vy += y * (1 - b);
      }
    }
  }
  vxs[i] = vx;
  vys[i] = vy;
}

void fast_link(const NodeArrays &a, const LinkArrays &l, FastLink &c, double alpha,
               double iterations, const double *seed, cudaStream_t st) {
  const uint32_t n = a.n, entries = 2 * c.m;
  if (!c.gathered && entries) {
    D3_LAUNCH(k_link_gather, blocks_for(entries, 256), 256, 0, st)(l, c.adj, entries, c.scal);
    c.gathered = true;
  }
  for (double k = 0; k < iterations; k += 1) {
    D3_LAUNCH(k_shift2, blocks_for(n, 256), 256, 0, st)(a.x, a.y, a.vx, a.vy, a.px, a.py, n);
    D3_LAUNCH(k_link_sweep, blocks_for(n, 128), 128, 0, st)(a.px, a.py, a.vx, a.vy, c.row, c.adj,
                                                           c.other, c.scal, entries, alpha, seed,
                                                           n);
  }
}

// ---- grid.zig --------------------------------------------------------------

// Shifted positions, bounds, largest radius and point count; the last block
// sizes the grid (grid.zig:66-91, 224-258).
__global__ void __launch_bounds__(GRID_THREADS) k_grid_bounds(const double *x, const double *y,
                                                              const double *vx, const double *vy,
                                                              double *px, double *py,
                                                              const double *radii, uint32_t n,
                                                              double *part, uint32_t *info,
                                                              double *geom) {
  double b[5] = {INFINITY, INFINITY, -INFINITY, -INFINITY, 0};
  uint32_t m = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double xx = x[i] + vx[i], yy = y[i] + vy[i];
    px[i] = xx;
    py[i] = yy;
    if (xx != xx || yy != yy) continue;
    ++m;
    if (xx < b[0]) b[0] = xx;
    if (xx > b[2]) b[2] = xx;
    if (yy < b[1]) b[1] = yy;
    if (yy > b[3]) b[3] = yy;
    double rad = radii[i];
    if (rad > b[4]) b[4] = rad;
  }
  __shared__ double sb[GRID_THREADS][5];
  __shared__ uint32_t sm[GRID_THREADS];
  const unsigned t = threadIdx.x;
  for (int q = 0; q < 5; ++q) sb[t][q] = b[q];
  sm[t] = m;
  __syncthreads();
  for (unsigned s = GRID_THREADS / 2; s > 0; s >>= 1) {
    if (t < s) {
      if (sb[t + s][0] < sb[t][0]) sb[t][0] = sb[t + s][0];
      if (sb[t + s][1] < sb[t][1]) sb[t][1] = sb[t + s][1];
      if (sb[t + s][2] > sb[t][2]) sb[t][2] = sb[t + s][2];
      if (sb[t + s][3] > sb[t][3]) sb[t][3] = sb[t + s][3];
      if (sb[t + s][4] > sb[t][4]) sb[t][4] = sb[t + s][4];
      sm[t] += sm[t + s];
    }
    __syncthreads();
  }
  __shared__ bool last;
  if (t == 0) {
    for (int q = 0; q < 5; ++q) part[blockIdx.x * 6 + q] = sb[0][q];
    ((uint32_t *)&part[blockIdx.x * 6 + 5])[0] = sm[0];
    __threadfence();
    last = atomicAdd(&info[5], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || t != 0) return;
  __threadfence();
  double a0 = INFINITY, a1 = INFINITY, a2 = -INFINITY, a3 = -INFINITY, rmax = 0;
  uint32_t mm = 0;
  for (unsigned k = 0; k < gridDim.x; ++k) {
    const volatile double *p = &part[k * 6];
    uint32_t pm = ((const volatile uint32_t *)&part[k * 6 + 5])[0];
    if (pm == 0) continue;
    mm += pm;
    if (p[0] < a0) a0 = p[0];
    if (p[2] > a2) a2 = p[2];
    if (p[1] < a1) a1 = p[1];
    if (p[3] > a3) a3 = p[3];
    if (p[4] > rmax) rmax = p[4];
  }
  info[5] = 0;
  info[3] = mm;
  if (mm < 2 || !(rmax > 0)) {
    info[4] = 0;
    return;
  }
  double h = 2 * rmax;
  uint32_t gx = (uint32_t)(floor((a2 - a0) / h) + 1);
  uint32_t gy = (uint32_t)(floor((a3 - a1) / h) + 1);
  while ((uint64_t)gx * gy > 4 * (uint64_t)n + 16) {
    h *= 2;
    gx = (uint32_t)(floor((a2 - a0) / h) + 1);
    gy = (uint32_t)(floor((a3 - a1) / h) + 1);
  }
  info[0] = gx;
  info[1] = gy;
  info[2] = gx * gy;
  info[4] = 1;
  geom[0] = a0;
  geom[1] = a1;
  geom[2] = 1 / h;
}

// grid.zig:95-111: sort input in descending node order, keyed by cell.
__global__ void k_grid_bin(const double *px, const double *py, uint32_t n, const uint32_t *info,
                           const double *geom, uint64_t *keys, uint32_t *items, uint32_t *cell_of) {
  if (info[4] == 0) return;
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t gx = info[0], cells = info[2];
  const uint32_t i = n - 1 - k;
  uint32_t cell = cells;
  if (px[i] == px[i] && py[i] == py[i]) {
    uint32_t cx = (uint32_t)floor((px[i] - geom[0]) * geom[2]);
    uint32_t cy = (uint32_t)floor((py[i] - geom[1]) * geom[2]);
    cell = cy * gx + cx;
  }
  cell_of[i] = cell >= cells ? NO_CELL : cell;
  keys[k] = cell;
  items[k] = i;
}

// start[c] = first sorted position whose cell is >= c (grid.zig:115-127, 263-267).
__global__ void k_grid_starts(const uint64_t *keys, uint32_t n, const uint32_t *info,
                              uint32_t *start) {
  if (info[4] == 0) return;
  const uint32_t cells = info[2], m = info[3];
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= cells; c += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
      uint32_t mid = lo + ((hi - lo) >> 1);
      if (keys[mid] < c) lo = mid + 1; else hi = mid;
    }
    start[c] = c == cells ? m : (lo < m ? lo : m);
  }
}

// grid.zig:129-195
__global__ void k_grid_sweep(const double *px, const double *py, double *vxs, double *vys,
                             const double *radii, double strength, const double *seedp, uint32_t n,
                             const uint32_t *info, const uint32_t *start, const uint32_t *items,
                             const uint32_t *cell_of) {
  if (info[4] == 0) return;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t ci = cell_of[i];
  if (ci == NO_CELL) return;
  const uint64_t seed = seed_bits(seedp);
  const uint32_t gx = info[0], gy = info[1];
  const double ri = radii[i], ri2 = ri * ri;
  const double xi = px[i], yi = py[i];
  double vx = vxs[i], vy = vys[i];
  const uint32_t cxi = ci % gx, cyi = ci / gx;
  const uint32_t xa = cxi > 0 ? cxi - 1 : 0, xb = cxi + 1 < gx - 1 ? cxi + 1 : gx - 1;
  const uint32_t ya = cyi > 0 ? cyi - 1 : 0, yb = cyi + 1 < gy - 1 ? cyi + 1 : gy - 1;
  for (uint32_t cy = ya; cy <= yb; ++cy) {
    for (uint32_t cx = xa; cx <= xb; ++cx) {
      const uint32_t cell = cy * gx + cx;
      for (uint32_t kk = start[cell]; kk < start[cell + 1]; ++kk) {
        const uint32_t j = items[kk];
        if (j == i) continue;
        const double rj = radii[j];
        double rr = ri + rj;
        double x = xi - px[j], y = yi - py[j];
        double l = x * x + y * y;
        if (l < rr * rr) {
          if (x == 0 || y == 0) {
            const uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
            const double sign = i == lo ? 1 : -1;
            if (x == 0) { x = sign * hash_jiggle(seed, lo, hi, 0); l += x * x; }
            if (y == 0) { y = sign * hash_jiggle(seed, lo, hi, 1); l += y * y; }
          }
          l = sqrt(l);
          l = (rr - l) / l * strength;
          x *= l;
          y *= l;
          rr = rj * rj / (ri2 + rj * rj);
          vx += x * rr;
          vy += y * rr;
        }
      }
    }
  }
  vxs[i] = vx;
  vys[i] = vy;
}

void fast_collide(FastScratch &s, const NodeArrays &a, const double *radii, double strength,
                  double iterations, const double *seed, cudaStream_t st) {
  const uint32_t n = a.n;
  if (n == 0) return;
  unsigned gb = blocks_for(n, GRID_THREADS * 4);
  if (gb > GRID_BLOCKS_MAX) gb = GRID_BLOCKS_MAX;
  SortScratch ss{s.g_keys_tmp, s.g_items_tmp, s.g_hist, s.g_part};
  for (double k = 0; k < iterations; k += 1) {
    D3_LAUNCH(k_grid_bounds, gb, GRID_THREADS, 0, st)(a.x, a.y, a.vx, a.vy, a.px, a.py, radii, n, s.g_box,
                                                s.g_info, s.g_geom);
    D3_LAUNCH(k_grid_bin, blocks_for(n, 256), 256, 0, st)(a.px, a.py, n, s.g_info, s.g_geom, s.g_keys,
                                                   s.g_items, s.g_cell_of);
    radix_sort_u64(s.g_keys, s.g_items, n, 0, 4, false, ss, st);
    D3_LAUNCH(k_grid_starts, blocks_for(4ull * n + 17, 256), 256, 0, st)(s.g_keys, n, s.g_info, s.g_start);
    D3_LAUNCH(k_grid_sweep, blocks_for(n, 128), 128, 0, st)(a.px, a.py, a.vx, a.vy, radii, strength, seed, n,
                                                     s.g_info, s.g_start, s.g_items, s.g_cell_of);
  }
}

}  // namespace d3
