// forces.cu — exact-mode forces on the device, bit-exact with d3-force.
//
// All arithmetic keeps d3's statement order (no FMA contraction: the file is
// built with -fmad=false). Traversals are stackless: cells are in d3's visit
// preorder, so "descend" is c + 1 and "do not descend" is skip[c].
#include <climits>
#include <cstdlib>
#include <vector>

#include <cooperative_groups.h>

#include "forces.cuh"
#include "scan_sort.cuh"

namespace cg = cooperative_groups;

namespace d3 {

size_t csum_rec_bytes(uint32_t n);
size_t csum_count_words(uint32_t n);
size_t csum_part_words(uint32_t n);

int scratch_reserve(ForceScratch &s, uint32_t n) {
  if (!s.counters) {
    D3_CUDA_OK(cudaMalloc(&s.counters, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(s.counters, 0, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMalloc(&s.center, 2 * sizeof(double)));
    D3_CUDA_OK(cudaMalloc(&s.csum_stamps, 8 * sizeof(unsigned long long)));
    D3_CUDA_OK(cudaMemset(s.csum_stamps, 0, 8 * sizeof(unsigned long long)));
  }
  if (n <= s.cap && s.cap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  cudaFree(s.draws); cudaFree(s.offsets); cudaFree(s.scan_part);
  cudaFree(s.csum_recs); cudaFree(s.csum_counts); cudaFree(s.csum_part); cudaFree(s.csum_scan_part);
  D3_CUDA_OK(cudaMalloc(&s.csum_recs, csum_rec_bytes(cap)));
  D3_CUDA_OK(cudaMalloc(&s.csum_counts, 2 * csum_count_words(cap) * 4));  // counts, offsets
  D3_CUDA_OK(cudaMalloc(&s.csum_part, csum_part_words(cap) * 8));
  D3_CUDA_OK(cudaMalloc(&s.csum_scan_part, scan_partial_words(csum_count_words(cap)) * 4));
  D3_CUDA_OK(cudaMalloc(&s.draws, (cap + 1) * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.offsets, (cap + 1) * 4ull));
  // also the grid partials of k_mb_draws (one word per block)
  const size_t sp = scan_partial_words(cap + 1);
  D3_CUDA_OK(cudaMalloc(&s.scan_part, (sp > 1024 ? sp : 1024) * 4));
  s.cap = cap;
  return 0;
}

void scratch_free(ForceScratch &s) {
  cudaFree(s.draws); cudaFree(s.offsets); cudaFree(s.scan_part); cudaFree(s.counters);
  cudaFree(s.center); cudaFree(s.csum_recs); cudaFree(s.csum_counts); cudaFree(s.csum_part);
  cudaFree(s.csum_scan_part); cudaFree(s.csum_stamps);
  s = ForceScratch();
}

// ---------------------------------------------------------------------------
// Bottom-up passes (visitAfter). The many-body accumulation: the last child to
// finish computes its parent. The collide radii: a maximum, so each leaf
// raises its ancestors directly.
// ---------------------------------------------------------------------------

__device__ inline double ld_cg(const double *p) { return __ldcg(p); }

// A cell as the exact many-body traversal reads it, in one 64-byte load.
struct alignas(64) MRec {
  double x, y, value;
  double wt;              // (x1 - x0)^2 / theta2, as the opening test forms it
  uint32_t skip, head;    // head: the leaf's head node; NONE for an internal cell
  uint32_t first, count;  // the leaf's points in perm
};
static_assert(sizeof(MRec) == 64, "record layout");

// A parent's step of the accumulation: its children are the ones listed
// in its cell (several), or only the child just finished (one: no counter,
// and the child's values are still in registers).
struct Climb {
  uint32_t p;      // the parent (NONE at the root)
  uint32_t nch;    // its child count
};

__device__ inline Climb climb_up(const uint32_t *parent, const uint8_t *pnch, uint32_t cur) {
  Climb c;
  c.p = parent[cur];
  c.nch = pnch[cur];
  return c;
}

// A child's arrival at its parent: release orders the child's values before
// the count, acquire makes the earlier children's values visible to the last
// one (the counts on one parent form a release sequence).
__device__ inline uint32_t arrive_acq_rel(uint32_t *p) {
  uint32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}

// many_body.zig:101-135 (accumulate). Leaf: head position, strength summed
// over the chain from perm[first + count - 1] down. Internal: children 0..3
// with a truthy |value|. Every cell's traversal record: the thread visiting
// an internal cell writes its fixed part (width test, skip link); the climb
// writes its centroid and charge.
__global__ void k_mb_accumulate(Cell *cells, const uint32_t *parent, const uint8_t *pnch,
                                uint32_t *counter, const uint32_t *perm, const uint32_t *skip,
                                const double *xs, const double *ys, const double *strengths,
                                double theta2, MRec *rec, const uint32_t *info) {
  const uint32_t len = info[1];
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < len; c += gridDim.x * blockDim.x) {
    Cell *q = &cells[c];
    if (!is_leaf(*q)) {
      const double w = q->x1 - q->x0;
      rec[c].wt = w * w / theta2;
      rec[c].skip = skip[c];
      rec[c].head = NONE;
      rec[c].first = 0;
      rec[c].count = 0;
      continue;
    }
    const uint32_t first = q->first, count = q->count;
    uint32_t head = perm[first + count - 1];
    double strength = 0;
    for (uint32_t k = first + count; k > first;) {
      --k;
      strength += strengths[perm[k]];
    }
    double cx = xs[head], cy = ys[head], cv = strength;
    q->x = cx;
    q->y = cy;
    q->value = cv;
    {
      const double w = q->x1 - q->x0;
      MRec r;
      r.x = cx; r.y = cy; r.value = cv; r.wt = w * w / theta2;
      r.skip = skip[c]; r.head = head; r.first = first; r.count = count;
      rec[c] = r;
    }
    auto finish = [&](uint32_t x) {
      cells[x].x = cx;
      cells[x].y = cy;
      cells[x].value = cv;
      rec[x].x = cx;
      rec[x].y = cy;
      rec[x].value = cv;
    };
    Climb up = climb_up(parent, pnch, c);
    for (;;) {
      const uint32_t p = up.p;
      if (p == NONE) break;
      if (up.nch == 1) {
        // A run of only children: p's only child is done, so p, p - 1, ...
        // (in preorder an only child follows its parent) while each is an
        // only child itself; their child counts read 8 at a time.
        uint8_t pk[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) pk[t] = (uint32_t)t <= p ? pnch[p - t] : 0;
        bool out = false;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const uint32_t x = p - t;
          double st = 0, weight = 0, sx = 0, sy = 0;
          const double w = fabs(cv);
          if (w > 0) {
            st += cv;
            weight += w;
            sx += w * cx;
            sy += w * cy;
          }
          cx = sx / weight;
          cy = sy / weight;
          cv = st;
          finish(x);
          if (pk[t] != 1) {
            up = climb_up(parent, pnch, x);
            out = true;
            break;
          }
        }
        if (!out) {
          up.p = p - 8;  // the eighth cell was an only child too
          up.nch = 1;
        }
        continue;
      }
      // The parent's links and child list were written by the tree build:
      // loaded before the arrival, so only the children's values wait on it.
      const Climb next = climb_up(parent, pnch, p);
      uint32_t ch[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) ch[k] = cells[p].child[k];
      if (arrive_acq_rel(&counter[p]) != up.nch - 1) break;
      double2 cxy[4], cvw[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (ch[k] == NONE) continue;
        cxy[k] = __ldcg((const double2 *)&rec[ch[k]].x);
        cvw[k] = __ldcg((const double2 *)&rec[ch[k]].value);
      }
      double st = 0, weight = 0, x = 0, y = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (ch[k] == NONE) continue;
        double v = cvw[k].x;
        double w = fabs(v);
        if (w > 0) {
          st += v;
          weight += w;
          x += w * cxy[k].x;
          y += w * cxy[k].y;
        }
      }
      cx = x / weight;
      cy = y / weight;
      cv = st;
      finish(p);
      up = next;
    }
  }
}

// collide.zig:117-129 (prepare): leaf radius of its head, internal the largest
// child radius (strict >, from 0). The internal rule makes a cell's radius
// max(+0, the positive radii of the leaf heads below it): a maximum, exact in
// any order. So no cell waits for its children: the tree build leaves every
// radius +0, each leaf with a positive radius raises its ancestors by 64-bit
// atomic maxima on the radius bits (the bit order of positive doubles is their
// numeric order), and stops at the first ancestor that already holds at least
// as much (whoever raised that one goes on from there). NaN, negative and zero
// leaf radii raise nothing, as in the strict comparison from 0.
__global__ void k_collide_prep(Cell *cells, const uint32_t *parent, const uint32_t *perm,
                               const double *radii, const uint32_t *info) {
  const uint32_t len = info[1];
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < len; c += gridDim.x * blockDim.x) {
    Cell *q = &cells[c];
    if (!is_leaf(*q)) continue;
    const double cr = radii[perm[q->first + q->count - 1]];
    q->r = cr;
    if (!(cr > 0)) continue;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(cr);
    uint32_t p = parent[c];
    while (p != NONE) {
      // the next link is static: loaded alongside the maximum
      const uint32_t pp = parent[p];
      const unsigned long long old =
          atomicMax(reinterpret_cast<unsigned long long *>(&cells[p].r), bits);
      if (old >= bits) break;
      p = pp;
    }
  }
}

// ---------------------------------------------------------------------------
// Exact many-body traversal (many_body.zig:176-263)
// ---------------------------------------------------------------------------

// One target. RECORD: stop accumulating at the first zero delta d3 would
// jiggle, count the draws it would make, and do not write. Otherwise draws
// come from the stream at `draw0`.
template <bool RECORD>
__device__ inline uint32_t mb_node(const MRec *rec, const uint32_t *perm,
                                   uint32_t len, const double *xs, const double *ys,
                                   double *vxs, double *vys, const double *strengths,
                                   const ManyBodyParams p, uint32_t i, const Rng *rng,
                                   uint64_t draw0) {
  const double nx = xs[i], ny = ys[i];
  double vx = vxs[i], vy = vys[i];
  uint32_t draws = 0;
  bool flagged = false;
  // The next cell follows from the current record alone (its skip link when
  // the cell is empty or far enough, else c + 1), so its load is issued
  // before this cell's arithmetic.
  uint32_t c = 0;
  MRec q;
  if (len) q = rec[0];
  while (c < len) {
    const MRec cq = q;
    const double value = cq.value;
    const bool live = value != 0 && value == value;
    double x = cq.x - nx, y = cq.y - ny;
    double l = x * x + y * y;
    const bool far = live && cq.wt < l;
    const uint32_t next = !live || far ? cq.skip : c + 1;
    if (next < len) q = rec[next];
    c = next;
    if (!live) continue;
    if (far) {
      if (l < p.dmax2) {
        if (RECORD && (x == 0 || y == 0)) {
          flagged = true;
          draws += (x == 0) + (y == 0);
        } else if (!flagged) {
          if (!RECORD) {
            if (x == 0) { x = (rng_draw_at(*rng, draw0 + draws++) - 0.5) * 1e-6; l += x * x; }
            if (y == 0) { y = (rng_draw_at(*rng, draw0 + draws++) - 0.5) * 1e-6; l += y * y; }
          }
          if (l < p.dmin2) l = sqrt(p.dmin2 * l);
          vx += x * value * p.alpha / l;
          vy += y * value * p.alpha / l;
        }
      }
      continue;
    }
    if (cq.head == NONE) continue;
    if (l >= p.dmax2) continue;
    const uint32_t first = cq.first, count = cq.count;
    const uint32_t head = cq.head;
    if (head != i || count > 1) {
      if (RECORD && (x == 0 || y == 0)) {
        flagged = true;
        draws += (x == 0) + (y == 0);
      } else if (!flagged) {
        if (!RECORD) {
          if (x == 0) { x = (rng_draw_at(*rng, draw0 + draws++) - 0.5) * 1e-6; l += x * x; }
          if (y == 0) { y = (rng_draw_at(*rng, draw0 + draws++) - 0.5) * 1e-6; l += y * y; }
        }
        if (l < p.dmin2) l = sqrt(p.dmin2 * l);
      }
    }
    if (!flagged) {
      for (uint32_t k = first + count; k > first;) {
        --k;
        const uint32_t j = perm[k];
        if (j != i) {
          const double wj = strengths[j] * p.alpha / l;
          vx += x * wj;
          vy += y * wj;
        }
      }
    }
  }
  if (!flagged) {
    vxs[i] = vx;
    vys[i] = vy;
  }
  return flagged ? draws : 0;
}

// Record pass over all nodes in Morton order (perm, then the NaN nodes).
__global__ void __launch_bounds__(128) k_mb_traverse(const MRec *rec,
                                                     const uint32_t *perm, const uint32_t *info,
                                                     const double *xs, const double *ys, double *vxs,
                                                     double *vys, const double *strengths,
                                                     ManyBodyParams p, uint32_t n, uint32_t *draws,
                                                     uint32_t *counters) {
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n) return;
  // no tree this call (cell buffer overflow or a failed build launch): perm
  // may be stale, the velocities stay as they are
  if (info[5]) return;
  const uint32_t len = info[1];
  const uint32_t i = perm[pos];
  uint32_t d = len ? mb_node<true>(rec, perm, len, xs, ys, vxs, vys, strengths, p, i,
                                   nullptr, 0)
                   : 0;
  draws[i] = d;
  if (d) atomicAdd(&counters[1], 1u);
}

// Flagged nodes again, each from its own offset in the draw stream (the
// exclusive scan of draws over node index = d3's draw order).
__global__ void __launch_bounds__(128) k_mb_rerun(const MRec *rec,
                                                  const uint32_t *perm, const uint32_t *info,
                                                  const double *xs, const double *ys, double *vxs,
                                                  double *vys, const double *strengths,
                                                  ManyBodyParams p, uint32_t n,
                                                  const uint32_t *draws, const uint32_t *offsets,
                                                  const uint32_t *counters, const Rng *rng) {
  if (counters[1] == 0 || info[5]) return;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || draws[i] == 0) return;
  mb_node<false>(rec, perm, info[1], xs, ys, vxs, vys, strengths, p, i, rng, offsets[i]);
}

// The jiggle draws of the flagged targets, after the record pass, in one
// cooperative launch (device LCG): the exclusive scan of the draw counts over
// node index (d3's draw order), the flagged targets again from their stream
// positions, then the LCG advanced past all the draws. Nothing to do (the
// usual case) is decided by every block alike from the flagged count.
__global__ void __launch_bounds__(256) k_mb_draws(const MRec *rec, const uint32_t *perm,
                                                  const uint32_t *info, const double *xs,
                                                  const double *ys, double *vxs, double *vys,
                                                  const double *strengths, ManyBodyParams p,
                                                  uint32_t n, const uint32_t *draws,
                                                  uint32_t *offsets, uint32_t *counters,
                                                  uint32_t *bsum, Rng *rng) {
  if (__ldcg(&counters[1]) == 0 || __ldcg(&info[5])) return;
  cg::grid_group g = cg::this_grid();
  const uint32_t total = grid_excl_scan(g, draws, offsets, n, bsum);
  g.sync();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t len = info[1];
  for (uint32_t i = tid; i < n; i += nth)
    if (__ldcg(&draws[i]))
      mb_node<false>(rec, perm, len, xs, ys, vxs, vys, strengths, p, i, rng, __ldcg(&offsets[i]));
  g.sync();
  if (tid == 0) {
    counters[0] = total;
    if (rng->mode == 0) rng->lcg = lcg_skip(rng->lcg, total);
    else rng->pos += total;
  }
}

__global__ void k_rng_advance(Rng *rng, const uint32_t *total) {
  uint32_t t = *total;
  if (t == 0) return;
  if (rng->mode == 0) rng->lcg = lcg_skip(rng->lcg, t);
  else rng->pos += t;
}

static void climb_grid(unsigned &blocks, unsigned &threads, uint32_t cap) {
  threads = 256;
  blocks = blocks_for(cap, threads);
  if (blocks > 148 * 16) blocks = 148 * 16;
}

void many_body_exact(TreeDev &t, const NodeArrays &a, const double *strengths,
                     const ManyBodyParams &p, Rng *rng, ForceScratch &s, uint32_t *status,
                     bool host_draws, cudaStream_t st, const std::function<void(int)> &mark) {
  const uint32_t n = a.n;
  tree_build(t, a.x, a.y, n, status, st);
  if (mark) mark(0);
  if (n == 0) return;
  unsigned cb, ct;
  climb_grid(cb, ct, t.cells_cap);
  D3_LAUNCH(k_mb_accumulate, cb, ct, 0, st)(t.cells, t.parent, t.pnch, t.counter, t.perm, t.skip, a.x,
                                     a.y, strengths, p.theta2, (MRec *)t.rec, t.info);
  if (mark) mark(1);
  cudaMemsetAsync(s.counters, 0, 2 * sizeof(uint32_t), st);
  D3_LAUNCH(k_mb_traverse, blocks_for(n, 128), 128, 0, st)((const MRec *)t.rec, t.perm, t.info, a.x, a.y,
                                                    a.vx, a.vy, strengths, p, n, s.draws,
                                                    s.counters);
  if (host_draws) {
    scan_u32(s.draws, s.offsets, n, s.scan_part, s.counters, st);
    return;
  }
  static int blocks = 0;
  if (!blocks) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_mb_draws, 256, 0);
    blocks = sms * (per >= 2 ? 2 : (per > 0 ? per : 1));
  }
  const MRec *rec = (const MRec *)t.rec;
  const uint32_t *perm = t.perm, *info = t.info;
  const double *x = a.x, *y = a.y;
  double *vx = a.vx, *vy = a.vy;
  ManyBodyParams pp = p;
  uint32_t nn = n;
  const uint32_t *draws = s.draws;
  uint32_t *offsets = s.offsets, *counters = s.counters, *bsum = s.scan_part;
  void *params[] = {&rec, &perm, &info, &x, &y, &vx, &vy, &strengths, &pp, &nn, &draws, &offsets,
                    &counters, &bsum, &rng};
  ++g_launches;
  if (cudaLaunchCooperativeKernel((const void *)k_mb_draws, blocks, 256, params, 0, st) != cudaSuccess) {
    cudaGetLastError();
    scan_u32(s.draws, s.offsets, n, s.scan_part, s.counters, st);
    many_body_rerun(t, a, strengths, p, rng, s, st);
  }
}

void many_body_rerun(TreeDev &t, const NodeArrays &a, const double *strengths,
                     const ManyBodyParams &p, Rng *rng, ForceScratch &s, cudaStream_t st) {
  const uint32_t n = a.n;
  D3_LAUNCH(k_mb_rerun, blocks_for(n, 128), 128, 0, st)((const MRec *)t.rec, t.perm, t.info, a.x, a.y, a.vx,
                                                 a.vy, strengths, p, n, s.draws, s.offsets,
                                                 s.counters, rng);
  D3_LAUNCH(k_rng_advance, 1, 1, 0, st)(rng, s.counters);
}

// ---------------------------------------------------------------------------
// Exact link (link.zig:8-40)
// ---------------------------------------------------------------------------

int link_plan_build(LinkPlan &plan, const uint32_t *src, const uint32_t *tgt, uint32_t m) {
  // level(e) = 1 + the largest level of an earlier link sharing a node, so
  // every link sees exactly the velocities its predecessors wrote.
  uint32_t nmax = 0;
  for (uint32_t e = 0; e < m; ++e) {
    if (src[e] + 1 > nmax) nmax = src[e] + 1;
    if (tgt[e] + 1 > nmax) nmax = tgt[e] + 1;
  }
  std::vector<uint32_t> node_level(nmax, 0), level(m);
  uint32_t levels = 0;
  for (uint32_t e = 0; e < m; ++e) {
    uint32_t l = (node_level[src[e]] > node_level[tgt[e]] ? node_level[src[e]] : node_level[tgt[e]]) + 1;
    level[e] = l;
    node_level[src[e]] = l;
    node_level[tgt[e]] = l;
    if (l > levels) levels = l;
  }
  std::vector<uint32_t> start(levels + 2, 0), order(m > 0 ? m : 1);
  for (uint32_t e = 0; e < m; ++e) start[level[e]]++;
  uint32_t run = 0;
  for (uint32_t l = 0; l <= levels + 1; ++l) {
    uint32_t c = start[l];
    start[l] = run;
    run += c;
  }
  std::vector<uint32_t> fill(start.begin(), start.end());
  for (uint32_t e = 0; e < m; ++e) order[fill[level[e]]++] = e;
  // per link, how many earlier links touch its source and its target: it may
  // run once that many links on each have finished
  std::vector<uint32_t> seen(nmax, 0), need_e(2 * (size_t)m), need(2 * (size_t)(m > 0 ? m : 1));
  for (uint32_t e = 0; e < m; ++e) {
    need_e[2 * e] = seen[src[e]];
    need_e[2 * e + 1] = seen[tgt[e]];
    ++seen[src[e]];
    ++seen[tgt[e]];
  }
  for (uint32_t p = 0; p < m; ++p) {
    need[2 * p] = need_e[2 * order[p]];
    need[2 * p + 1] = need_e[2 * order[p] + 1];
  }
  link_plan_free(plan);
  D3_CUDA_OK(cudaMalloc(&plan.order, order.size() * 4));
  D3_CUDA_OK(cudaMalloc(&plan.level_start, start.size() * 4));
  D3_CUDA_OK(cudaMalloc(&plan.need, need.size() * 4));
  D3_CUDA_OK(cudaMalloc(&plan.done, (nmax > 0 ? nmax : 1) * 4ull));
  D3_CUDA_OK(cudaMemcpy(plan.order, order.data(), order.size() * 4, cudaMemcpyHostToDevice));
  D3_CUDA_OK(cudaMemcpy(plan.level_start, start.data(), start.size() * 4, cudaMemcpyHostToDevice));
  D3_CUDA_OK(cudaMemcpy(plan.need, need.data(), need.size() * 4, cudaMemcpyHostToDevice));
  plan.h_level_start = new uint32_t[start.size()];
  for (size_t k = 0; k < start.size(); ++k) plan.h_level_start[k] = start[k];
  plan.m = m;
  plan.levels = levels;
  plan.nodes = nmax;
  return 0;
}

void link_plan_free(LinkPlan &plan) {
  cudaFree(plan.order);
  cudaFree(plan.level_start);
  cudaFree(plan.need);
  cudaFree(plan.done);
  delete[] plan.h_level_start;
  plan = LinkPlan();
}

// One link, d3's statement order. Returns false (writing nothing) where d3
// would draw from `random`.
__device__ inline bool link_one(double *xs, double *ys, double *vxs, double *vys, const LinkArrays l,
                                uint32_t e, double alpha) {
  const uint32_t src = l.source[e], tgt = l.target[e];
  double x = xs[tgt] + vxs[tgt] - xs[src] - vxs[src];
  double y = ys[tgt] + vys[tgt] - ys[src] - vys[src];
  if (x == 0 || x != x || y == 0 || y != y) return false;
  double len = sqrt(x * x + y * y);
  len = (len - l.distance[e]) / len * alpha * l.strength[e];
  x *= len;
  y *= len;
  double b = l.bias[e];
  vxs[tgt] -= x * b;
  vys[tgt] -= y * b;
  b = 1 - b;
  vxs[src] += x * b;
  vys[src] += y * b;
  return true;
}

__global__ void k_link_level(double *xs, double *ys, double *vxs, double *vys, LinkArrays l,
                             const uint32_t *order, uint32_t lo, uint32_t hi, double alpha,
                             uint32_t *flag) {
  uint32_t k = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= hi) return;
  if (!link_one(xs, ys, vxs, vys, l, order[k], alpha)) atomicOr(flag, 1u);
}

__global__ void k_restore_v(double *vx, double *vy, const double *svx, const double *svy, uint32_t n,
                            const uint32_t *flag) {
  if (*flag == 0) return;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vx[i] = svx[i];
  vy[i] = svy[i];
}

__global__ void k_save_v(double *svx, double *svy, const double *vx, const double *vy, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  svx[i] = vx[i];
  svy[i] = vy[i];
}

// link.zig:8-40 on one thread, drawing from the device LCG.
__device__ void link_serial_lcg(const double *xs, const double *ys, double *vxs, double *vys,
                                const LinkArrays &l, double alpha, double iterations, Rng *rng,
                                uint32_t *status) {
  atomicOr(status, ST_LINK_JIGGLE);
  uint32_t s = rng->lcg;
  for (double k = 0; k < iterations; k += 1) {
    for (uint32_t i = 0; i < l.m; ++i) {
      const uint32_t src = l.source[i], tgt = l.target[i];
      double x = xs[tgt] + vxs[tgt] - xs[src] - vxs[src];
      if (x == 0 || x != x) { s = lcg_step(s); x = (lcg_value(s) - 0.5) * 1e-6; }
      double y = ys[tgt] + vys[tgt] - ys[src] - vys[src];
      if (y == 0 || y != y) { s = lcg_step(s); y = (lcg_value(s) - 0.5) * 1e-6; }
      double len = sqrt(x * x + y * y);
      len = (len - l.distance[i]) / len * alpha * l.strength[i];
      x *= len;
      y *= len;
      double b = l.bias[i];
      vxs[tgt] -= x * b;
      vys[tgt] -= y * b;
      b = 1 - b;
      vxs[src] += x * b;
      vys[src] += y * b;
    }
  }
  rng->lcg = s;
}

__global__ void k_link_serial(double *xs, double *ys, double *vxs, double *vys, LinkArrays l,
                              double alpha, double iterations, Rng *rng, const uint32_t *flag,
                              uint32_t *status) {
  if (*flag == 0) return;
  link_serial_lcg(xs, ys, vxs, vys, l, alpha, iterations, rng, status);
}

// The same with draws pulled by the host: resumes at (resume[0], resume[1]),
// stops before a link whose draws are not in the buffer yet.
__global__ void k_link_serial_host(double *xs, double *ys, double *vxs, double *vys, LinkArrays l,
                                   double alpha, double iterations, Rng *rng, uint32_t *resume) {
  uint64_t used = 0, avail = rng->avail - rng->pos;
  const double *buf = rng->buf + rng->pos;
  uint32_t it = resume[0], i0 = resume[1];
  for (double k = (double)it; k < iterations; k += 1, ++it, i0 = 0) {
    for (uint32_t i = i0; i < l.m; ++i) {
      const uint32_t src = l.source[i], tgt = l.target[i];
      double x = xs[tgt] + vxs[tgt] - xs[src] - vxs[src];
      double y = ys[tgt] + vys[tgt] - ys[src] - vys[src];
      uint32_t need = (x == 0 || x != x) + (y == 0 || y != y);
      if (used + need > avail) {
        resume[0] = it;
        resume[1] = i;
        resume[2] = (uint32_t)(used + need - avail);
        rng->pos += used;
        return;
      }
      if (x == 0 || x != x) x = (buf[used++] - 0.5) * 1e-6;
      if (y == 0 || y != y) y = (buf[used++] - 0.5) * 1e-6;
      double len = sqrt(x * x + y * y);
      len = (len - l.distance[i]) / len * alpha * l.strength[i];
      x *= len;
      y *= len;
      double b = l.bias[i];
      vxs[tgt] -= x * b;
      vys[tgt] -= y * b;
      b = 1 - b;
      vxs[src] += x * b;
      vys[src] += y * b;
    }
  }
  resume[2] = 0;
  rng->pos += used;
}

// A link with everything about it that does not change during the pass
// (e = NONE: no link).
struct LinkPre {
  uint32_t e, src, tgt;
  double dist, str, bias, xt, yt, xsrc, ysrc;
};

__device__ inline void link_params(const LinkArrays &l, uint32_t e, LinkPre &p) {
  p.e = e;
  if (e == NONE) return;
  p.src = l.source[e];
  p.tgt = l.target[e];
  p.dist = l.distance[e];
  p.str = l.strength[e];
  p.bias = l.bias[e];
}

__device__ inline void link_positions(const double *xs, const double *ys, LinkPre &p) {
  if (p.e == NONE) return;
  p.xt = xs[p.tgt];
  p.yt = ys[p.tgt];
  p.xsrc = xs[p.src];
  p.ysrc = ys[p.src];
}

struct LinkFlowArgs {
  const double *xs, *ys;
  double *vxs, *vys, *svx, *svy;
  LinkArrays l;
  const uint32_t *order, *need;
  uint32_t *done;
  uint32_t n, nodes;
  double alpha, iterations;
  uint32_t *flag;
  Rng *rng;           // with serial_lcg: the serial pass's draws
  uint32_t *status;
  int serial_lcg;     // a met jiggle is resolved in the launch (device LCG)
  unsigned sleep_ns;  // pause between polls of a wait (after the first eight)
};

__device__ inline unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A link's wait, bounded: until `ns` links on src and `nt` on tgt have
// finished. False if it gave up (20 ms): the pass is then restored and run
// serially.
__device__ inline uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// A finished link's count on a node, ordered after its velocity writes.
__device__ inline void red_release_add(uint32_t *p, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ inline bool link_wait(const uint32_t *done, uint32_t src, uint32_t ns, uint32_t tgt,
                                 uint32_t nt, unsigned sleep_ns) {
  // acquire loads: a count seen orders the counted links' writes before the
  // velocities this link reads
  if (ld_acquire_u32(&done[src]) >= ns && ld_acquire_u32(&done[tgt]) >= nt) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (uint32_t it = 0;; ++it) {
    if (ld_acquire_u32(&done[src]) >= ns && ld_acquire_u32(&done[tgt]) >= nt) return true;
    if (it >= 8 && sleep_ns) __nanosleep(sleep_ns);
    if ((it & 15) == 15 && globaltimer_ns() - t0 > 20000000ull) return false;
  }
}

// The pass as dataflow, in one cooperative launch: the pass-start snapshot,
// then every link (threads take them in level order) once the links before
// it on its two nodes have finished (per-node finished counts against the
// plan's per-link counts; a link's parameters and endpoint positions are
// loaded before its wait), then the snapshot back if a link met a zero or
// NaN delta or a wait gave up (the serial kernel then runs the pass).
__global__ void __launch_bounds__(256) k_link_flow(LinkFlowArgs a) {
  cg::grid_group g = cg::this_grid();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  if (tid == 0) *a.flag = 0;
  for (uint32_t i = tid; i < a.n; i += nth) {
    a.svx[i] = a.vxs[i];
    a.svy[i] = a.vys[i];
  }
  const uint32_t m = a.l.m;
  bool bad = false;
  for (double k = 0; k < a.iterations; k += 1) {
    for (uint32_t i = tid; i < a.nodes; i += nth) a.done[i] = 0;
    g.sync();  // the snapshot and the counts before any link runs
    for (uint32_t p = tid; p < m; p += nth) {
      LinkPre c;
      link_params(a.l, a.order[p], c);
      link_positions(a.xs, a.ys, c);
      const uint32_t ns = a.need[2 * p], nt = a.need[2 * p + 1];
      if (!link_wait(a.done, c.src, ns, c.tgt, nt, a.sleep_ns)) bad = true;
      const double vxt = __ldcg(&a.vxs[c.tgt]), vyt = __ldcg(&a.vys[c.tgt]);
      const double vxsrc = __ldcg(&a.vxs[c.src]), vysrc = __ldcg(&a.vys[c.src]);
      double x = c.xt + vxt - c.xsrc - vxsrc;
      double y = c.yt + vyt - c.ysrc - vysrc;
      if (x == 0 || x != x || y == 0 || y != y) {
        bad = true;
      } else {
        double len = sqrt(x * x + y * y);
        len = (len - c.dist) / len * a.alpha * c.str;
        x *= len;
        y *= len;
        double b = c.bias;
        a.vxs[c.tgt] = vxt - x * b;
        a.vys[c.tgt] = vyt - y * b;
        b = 1 - b;
        a.vxs[c.src] = vxsrc + x * b;
        a.vys[c.src] = vysrc + y * b;
      }
      red_release_add(&a.done[c.src], 1u);
      red_release_add(&a.done[c.tgt], 1u);
    }
    g.sync();
  }
  if (bad) atomicOr(a.flag, 1u);
  g.sync();
  if (__ldcg(a.flag)) {
    for (uint32_t i = tid; i < a.n; i += nth) {
      a.vxs[i] = __ldcg(&a.svx[i]);
      a.vys[i] = __ldcg(&a.svy[i]);
    }
    if (a.serial_lcg) {
      g.sync();
      if (tid == 0) link_serial_lcg(a.xs, a.ys, a.vxs, a.vys, a.l, a.alpha, a.iterations, a.rng, a.status);
    }
  }
}

static int g_link_blocks = 0;

void link_exact(const NodeArrays &a, const LinkArrays &l, const LinkPlan &plan, double alpha,
                double iterations, Rng *rng, uint32_t *flag, uint32_t *status, bool serial_lcg,
                cudaStream_t st) {
  if (l.m == 0) return;
  const uint32_t n = a.n;
  if (!g_link_blocks) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_link_flow, 256, 0);
    // blocks per SM: at most 2, or D3_LINK_BLOCKS_PER_SM (1 .. occupancy)
    int want = per >= 2 ? 2 : 1;
    if (const char *e = getenv("D3_LINK_BLOCKS_PER_SM")) {
      const int v = atoi(e);
      if (v >= 1 && v <= per) want = v;
    }
    g_link_blocks = sms * want;
  }
  {
    LinkFlowArgs c;
    c.xs = a.x; c.ys = a.y; c.vxs = a.vx; c.vys = a.vy; c.svx = a.snap_vx; c.svy = a.snap_vy;
    c.l = l; c.order = plan.order; c.need = plan.need; c.done = plan.done;
    c.n = n; c.nodes = plan.nodes; c.alpha = alpha; c.iterations = iterations; c.flag = flag;
    c.sleep_ns = wait_sleep_ns();
    c.rng = rng; c.status = status; c.serial_lcg = serial_lcg;
    void *params[] = {&c};
    ++g_launches;
    if (cudaLaunchCooperativeKernel((const void *)k_link_flow, g_link_blocks, 256, params, 0, st) ==
        cudaSuccess)
      return;
    cudaGetLastError();
  }
  // (without a cooperative launch: one launch per level)
  cudaMemsetAsync(flag, 0, sizeof(uint32_t), st);
  D3_LAUNCH(k_save_v, blocks_for(n, 256), 256, 0, st)(a.snap_vx, a.snap_vy, a.vx, a.vy, n);
  for (double k = 0; k < iterations; k += 1) {
    for (uint32_t lv = 1; lv <= plan.levels; ++lv) {
      uint32_t lo = plan.h_level_start[lv], hi = plan.h_level_start[lv + 1];
      if (hi > lo)
        D3_LAUNCH(k_link_level, blocks_for(hi - lo, 128), 128, 0, st)(a.x, a.y, a.vx, a.vy, l, plan.order,
                                                                lo, hi, alpha, flag);
    }
  }
  D3_LAUNCH(k_restore_v, blocks_for(n, 256), 256, 0, st)(a.vx, a.vy, a.snap_vx, a.snap_vy, n, flag);
  if (serial_lcg) link_fallback_lcg(a, l, alpha, iterations, rng, flag, status, st);
}

void link_serial_host(const NodeArrays &a, const LinkArrays &l, double alpha, double iterations,
                      Rng *rng, uint32_t *resume, cudaStream_t st) {
  D3_LAUNCH(k_link_serial_host, 1, 1, 0, st)(a.x, a.y, a.vx, a.vy, l, alpha, iterations, rng, resume);
}

// Serial link on the device LCG, after a DAG pass that met a jiggle.
void link_fallback_lcg(const NodeArrays &a, const LinkArrays &l, double alpha, double iterations,
                       Rng *rng, const uint32_t *flag, uint32_t *status, cudaStream_t st) {
  D3_LAUNCH(k_link_serial, 1, 1, 0, st)(a.x, a.y, a.vx, a.vy, l, alpha, iterations, rng, flag, status);
}

// ---------------------------------------------------------------------------
// Exact collide (collide.zig:17-102), serial node order
// ---------------------------------------------------------------------------

__global__ void k_shift(const double *x, const double *y, const double *vx, const double *vy,
                        double *px, double *py, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  px[i] = x[i] + vx[i];
  py[i] = y[i] + vy[i];
}

// The node loop of collide.zig:47-100 from node i0. In host-draw mode a turn
// first counts its draws (decided by the state at the turn's start) and stops
// before the turn when the buffer is short.
__global__ void k_collide_serial(const Cell *cells, const uint32_t *skip, const uint32_t *perm,
                                 const uint32_t *info, const double *xs, const double *ys, double *vxs,
                                 double *vys, const double *radii, double strength, uint32_t n,
                                 Rng *rng, bool host_draws, uint32_t *resume) {
  const uint32_t len = info[1];
  if (len == 0) {
    if (resume) resume[2] = 0;
    return;
  }
  uint32_t s = rng->lcg;
  uint64_t used = 0, avail = host_draws ? rng->avail - rng->pos : 0;
  const double *buf = host_draws ? rng->buf + rng->pos : nullptr;
  uint32_t i0 = resume ? resume[0] : 0;
  for (uint32_t i = i0; i < n; ++i) {
    const double ri = radii[i], ri2 = ri * ri;
    const double xi = xs[i] + vxs[i], yi = ys[i] + vys[i];
    if (host_draws) {
      uint32_t need = 0;
      for (uint32_t c = 0; c < len;) {
        const Cell &q = cells[c];
        double r = ri + q.r;
        if (is_leaf(q)) {
          uint32_t j = perm[q.first + q.count - 1];
          if (j > i) {
            double x = xi - xs[j] - vxs[j], y = yi - ys[j] - vys[j];
            if (x * x + y * y < r * r) need += (x == 0) + (y == 0);
          }
          c = c + 1;
          continue;
        }
        if (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r) c = skip[c];
        else c = c + 1;
      }
      if (used + need > avail) {
        resume[0] = i;
        resume[2] = (uint32_t)(used + need - avail);
        rng->pos += used;
        return;
      }
    }
    for (uint32_t c = 0; c < len;) {
      const Cell &q = cells[c];
      double rj = q.r;
      double r = ri + rj;
      if (is_leaf(q)) {
        const uint32_t j = perm[q.first + q.count - 1];
        if (j > i) {
          double x = xi - xs[j] - vxs[j];
          double y = yi - ys[j] - vys[j];
          double l = x * x + y * y;
          if (l < r * r) {
            if (x == 0) {
              double u;
              if (host_draws) u = buf[used++]; else { s = lcg_step(s); u = lcg_value(s); }
              x = (u - 0.5) * 1e-6;
              l += x * x;
            }
            if (y == 0) {
              double u;
              if (host_draws) u = buf[used++]; else { s = lcg_step(s); u = lcg_value(s); }
              y = (u - 0.5) * 1e-6;
              l += y * y;
            }
            l = sqrt(l);
            l = (r - l) / l * strength;
            x *= l;
            y *= l;
            rj *= rj;
            r = rj / (ri2 + rj);
            vxs[i] += x * r;
            vys[i] += y * r;
            r = 1 - r;
            vxs[j] -= x * r;
            vys[j] -= y * r;
          }
        }
        c = c + 1;
        continue;
      }
      if (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r) c = skip[c];
      else c = c + 1;
    }
  }
  if (host_draws) rng->pos += used;
  else rng->lcg = s;
  if (resume) resume[2] = 0;
}

void shift_positions(const NodeArrays &a, cudaStream_t st) {
  if (a.n == 0) return;
  D3_LAUNCH(k_shift, blocks_for(a.n, 256), 256, 0, st)(a.x, a.y, a.vx, a.vy, a.px, a.py, a.n);
}

void collide_setup(TreeDev &t, const NodeArrays &a, const double *radii, uint32_t *status,
                   cudaStream_t st) {
  const uint32_t n = a.n;
  tree_build_shifted(t, a.x, a.y, a.vx, a.vy, a.px, a.py, n, status, st);
  if (n == 0) return;
  unsigned cb, ct;
  climb_grid(cb, ct, t.cells_cap);
  D3_LAUNCH(k_collide_prep, cb, ct, 0, st)(t.cells, t.parent, t.perm, radii, t.info);
}

void collide_serial(TreeDev &t, const NodeArrays &a, const double *radii, double strength, Rng *rng,
                    bool host_draws, uint32_t *resume, cudaStream_t st) {
  if (a.n == 0) return;
  D3_LAUNCH(k_collide_serial, 1, 1, 0, st)(t.cells, t.skip, t.perm, t.info, a.x, a.y, a.vx, a.vy, radii,
                                    strength, a.n, rng, host_draws, resume);
}

// ---------------------------------------------------------------------------
// center, x, y, radial, integrate (simple.zig)
// ---------------------------------------------------------------------------

// simple.zig:14-31: sx += x[i] for i = 0..n-1 (and sy), reproduced exactly
// in parallel. While the running sum s stays inside one binade [2^e, 2^e+1)
// (or its negative) and never meets a rounding tie, fl(s + v) = s + R(v) u
// with u = 2^(e-52) the ulp there and R(v) = v / u rounded to the nearest
// integer: the chain is an integer prefix sum. The launches:
//  part     approximate sums of chunks of values (a warp per chunk);
//  records  per chunk (a thread each), from the approximate prefix, the chunk
//           as records {lo, hi, a}, each applied as "s must lie in [lo, hi];
//           s += a" — run twice, to count and then to write at the scanned
//           offsets. A stretch record covers a run where the approximate sum
//           stays in one binade: [lo, hi] holds the exact entry sums for which
//           every partial sum provably stays there, and a = T, the run's exact
//           total (s + T is itself exact: both are multiples of u and the
//           result lies in the binade). A value record adds one value (binade
//           crossings, ties, short runs) and always applies.
//  walk     one thread per axis applies the records in order with the exact s,
//           streaming them into shared memory by bulk async copies
//           (cp.async.bulk, completion on an mbarrier). A batch runs first
//           with the entry tests off the dependent chain (one add per record);
//           if any test failed, the batch reruns from its entry sum, adding a
//           failed stretch's values one by one from global memory.
constexpr unsigned CSUM_CHUNK_MIN = 128;   // values per chunk (at least)
constexpr unsigned CSUM_MAX_CHUNKS = 8192; // chunks per axis (at most)
constexpr unsigned CSUM_BUFS = 4;          // record copies in flight per axis
constexpr unsigned CSUM_BATCH = 256;       // records per copy
constexpr unsigned CSUM_MIN_RUN = 2;       // shorter runs go into value records
constexpr unsigned long long CSUM_WAIT_NS = 20000000ull;  // 20 ms per copy, far above need

__device__ inline uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ inline unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A record; meta = (start << 16) | len for a stretch, 0 for a value.
struct CsumRec {
  double lo, hi, a;
  unsigned long long meta;
};

struct CsumGeom {
  uint32_t L, nc;  // values per chunk, chunks
};

__host__ __device__ inline CsumGeom csum_geom(uint32_t n) {
  CsumGeom g;
  uint32_t L = CSUM_CHUNK_MIN;
  if ((n + L - 1) / L > CSUM_MAX_CHUNKS) L = ((n + CSUM_MAX_CHUNKS - 1) / CSUM_MAX_CHUNKS + 31) / 32 * 32;
  g.L = L;
  g.nc = (n + L - 1) / L;
  return g;
}

// Every record covers at least one value: at most n records per axis.
size_t csum_rec_bytes(uint32_t n) { return 2ull * ((size_t)n + 1) * sizeof(CsumRec); }
size_t csum_count_words(uint32_t n) { return 2ull * csum_geom(n).nc + 1; }
size_t csum_part_words(uint32_t n) { return 2ull * csum_geom(n).nc; }

__device__ inline int binade_of(double s) {
  int e;
  frexp(s, &e);  // s = f 2^e, f in [0.5, 1): binade [2^(e-1), 2^e)
  return e - 1;
}

// part[ax * nc + c]: the sum of chunk c, in any order.
__global__ void k_csum_part(const double *x, const double *y, uint32_t n, CsumGeom g, double *part) {
  const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31;
  if (c >= g.nc) return;
  const uint32_t k0 = c * g.L, k1 = min(n, k0 + g.L);
  double ax = 0, ay = 0;
  for (uint32_t k = k0 + lane; k < k1; k += 32) {
    ax += x[k];
    ay += y[k];
  }
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
  }
  if (lane == 0) {
    part[c] = ax;
    part[g.nc + c] = ay;
  }
}

// One thread per chunk, both axes. WRITE false: counts[ax nc + c] = the
// chunk's records; WRITE true: the records at out + offsets[ax nc + c].
template <bool WRITE>
__global__ void __launch_bounds__(256) k_csum_records(const double *x, const double *y, uint32_t n,
                                                      CsumGeom g, const double *part,
                                                      uint32_t *counts, const uint32_t *offsets,
                                                      CsumRec *out, uint32_t *status) {
  __shared__ double sred[2][8];
  __shared__ double swarp[2][8];
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t c0 = blockIdx.x * blockDim.x;
  // approximate prefix: the chunks before this block, then a block scan
  double before[2] = {0, 0};
  for (int ax = 0; ax < 2; ++ax) {
    double a = 0;
    for (uint32_t k = t; k < c0; k += blockDim.x) a += part[ax * g.nc + k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) sred[ax][warp] = a;
  }
  __syncthreads();
  for (int ax = 0; ax < 2; ++ax) {
    double b = 0;
    for (unsigned w = 0; w < blockDim.x / 32; ++w) b += sred[ax][w];
    before[ax] = b;
  }
  double start[2];
  for (int ax = 0; ax < 2; ++ax) {
    const double mine = c < g.nc ? part[ax * g.nc + c] : 0;
    double incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
      const double yv = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (unsigned)o) incl += yv;
    }
    if (lane == 31) swarp[ax][warp] = incl;
    __syncthreads();
    double wpre = 0;
    for (unsigned w = 0; w < warp; ++w) wpre += swarp[ax][w];
    start[ax] = before[ax] + wpre + incl - mine;
    __syncthreads();
  }
  if (c >= g.nc) return;
  const long long LO = (1ll << 52) + 1, HI = (1ll << 53) - 1;
  const uint32_t k0 = c * g.L, k1 = min(n, k0 + g.L);
  for (int ax = 0; ax < 2; ++ax) {
    const double *v = ax ? y : x;
    CsumRec *o = nullptr;
    uint32_t limit = 0;
    if (WRITE) {
      o = out + offsets[ax * g.nc + c];
      limit = counts[ax * g.nc + c];
    }
    uint32_t count = 0;
    auto put = [&](const CsumRec &r) {
      if (WRITE) {
        if (count < limit) o[count] = r;
        else atomicOr(status, ST_CENTER_RECORDS);  // cannot happen: both passes agree
      }
      ++count;
    };
    double run = start[ax];
    bool open = false, neg = false;
    double scale = 0, u = 0, blo = 0, bhi = 0;  // 1 / u, u, binade [blo, bhi)
    long long tot = 0, pmin = 0, pmax = 0;
    uint32_t st0 = 0;
    auto start_at = [&](uint32_t k) {
      open = false;
      if (!(run != 0) || !isfinite(run)) return;
      const int e = binade_of(run);
      if (!(e > -1000 && e < 1000)) return;
      neg = run < 0;
      st0 = k;
      tot = pmin = pmax = 0;
      scale = ldexp(1.0, 52 - e);
      u = ldexp(1.0, e - 52);
      blo = ldexp(1.0, e);
      bhi = ldexp(1.0, e + 1);
      open = true;
    };
    // closes the open run [st0, end): a stretch record, or its values
    auto close = [&](uint32_t end) {
      if (!open) return;
      open = false;
      if (end - st0 >= CSUM_MIN_RUN) {
        // entry S (|s| = S u) keeps every partial S +- P in [LO, HI]
        long long a, b;
        if (!neg) { a = LO - pmin; b = HI - pmax; }
        else { a = LO + pmax; b = HI + pmin; }
        if (a <= b && a >= LO && b <= HI) {
          CsumRec r;
          if (!neg) { r.lo = (double)a * u; r.hi = (double)b * u; }
          else { r.lo = -(double)b * u; r.hi = -(double)a * u; }
          r.a = (double)tot * u;
          r.meta = ((unsigned long long)st0 << 16) | (unsigned long long)(end - st0);
          put(r);
          return;
        }
      }
      for (uint32_t k = st0; k < end; ++k) put(CsumRec{-INFINITY, INFINITY, v[k], 0ull});
    };
    start_at(k0);
    for (uint32_t k = k0; k < k1; ++k) {
      const double vv = v[k];
      run += vv;
      if (open) {
        const double q = vv * scale;  // exact: a power-of-two scaling in range
        const double ar = fabs(run);
        if (fabs(q) < 4.0e15 && fabs(q - trunc(q)) != 0.5 && ar >= blo && ar < bhi &&
            (run < 0) == neg) {
          tot += (long long)rint(q);
          pmin = tot < pmin ? tot : pmin;
          pmax = tot > pmax ? tot : pmax;
          continue;
        }
      }
      close(k);
      put(CsumRec{-INFINITY, INFINITY, vv, 0ull});  // element k is added on its own
      start_at(k + 1);
    }
    close(k1);
    if (!WRITE) counts[ax * g.nc + c] = count;
  }
}

__device__ inline bool mbar_test(uint32_t a, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{ .reg .pred p; mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2; "
      "selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits on an mbarrier phase with a time budget; false if it ran out. It
// spins on the test first, then polls against the timer.
__device__ bool mbar_wait_for(uint64_t *bar, uint32_t parity, unsigned long long budget_ns) {
  const uint32_t a = smem_addr(bar);
  for (int k = 0; k < 4096; ++k)
    if (mbar_test(a, parity)) return true;
  const unsigned long long t0 = gtimer_ns();
  for (;;) {
    if (mbar_test(a, parity)) return true;
    if (gtimer_ns() - t0 > budget_ns) return false;
    __nanosleep(32);
  }
}

__device__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, CSUM_WAIT_NS);
}

// The bounded wait's failure path, on purpose: a wait on an mbarrier that
// nothing arrives at (no copy is issued), with a short budget. The wait gives
// up, the status word records it, and the kernel returns.
__global__ void k_wait_selftest(uint32_t *status, unsigned long long budget_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  if (!mbar_wait_for(&bar, 0, budget_ns)) atomicOr(status, ST_WAIT_TIMEOUT);
}

void wait_selftest(uint32_t *status, uint32_t budget_us, cudaStream_t st) {
  D3_LAUNCH(k_wait_selftest, 1, 32, 0, st)(status, (unsigned long long)budget_us * 1000ull);
}

// A buffer is refilled only after this thread has used the values it read
// from it, so the copy needs no proxy fence before it.
__device__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

constexpr size_t CSUM_WALK_SMEM = 2ull * CSUM_BUFS * CSUM_BATCH * sizeof(CsumRec);

// One block: thread 0 walks x and thread 32 walks y, over the records
// [offsets[ax nc], offsets[(ax + 1) nc]).
// stamps (globaltimer ns): 0-2 walk start, 3 / 4 end of the x / y walk;
// 5 / 6 / 7 the x walk's batches rerun / stretches added one by one /
// records in all.
__global__ void k_csum_walk(const double *x, const double *y, CsumGeom g, const CsumRec *recs,
                            const uint32_t *offsets, double *out, uint32_t *status,
                            unsigned long long *stamps) {
  extern __shared__ __align__(128) unsigned char csum_smem[];
  __shared__ __align__(8) uint64_t bars[2][CSUM_BUFS];
  const unsigned t = threadIdx.x;
  if ((t & 31) != 0) return;
  const int ax = t >> 5;
  if (ax > 1) return;
  if (ax == 0) stamps[0] = stamps[1] = stamps[2] = gtimer_ns();
  CsumRec *bufs = reinterpret_cast<CsumRec *>(csum_smem) + (size_t)ax * CSUM_BUFS * CSUM_BATCH;
  uint64_t *bar = bars[ax];
  for (uint32_t q = 0; q < CSUM_BUFS; ++q)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[q])) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  const double *v = ax ? y : x;
  const uint32_t r0 = offsets[ax * g.nc], r1 = offsets[(ax + 1) * g.nc];
  const uint32_t nrec = r1 - r0, nb = (nrec + CSUM_BATCH - 1) / CSUM_BATCH;
  const CsumRec *rec = recs + r0;
  auto issue = [&](uint32_t b) {
    const uint32_t m = min(CSUM_BATCH, nrec - b * CSUM_BATCH);
    bulk_copy(bufs + (size_t)(b % CSUM_BUFS) * CSUM_BATCH, rec + (size_t)b * CSUM_BATCH,
              m * (uint32_t)sizeof(CsumRec), &bar[b % CSUM_BUFS]);
  };
  for (uint32_t b = 0; b < CSUM_BUFS && b < nb; ++b) issue(b);
  bool ok = true;
  double s = 0;
  uint32_t reruns = 0, failed = 0;
  uint32_t b = 0;
  for (; b < nb; ++b) {
    if (!mbar_wait(&bar[b % CSUM_BUFS], (b / CSUM_BUFS) & 1u)) {
      ok = false;
      break;
    }
    const CsumRec *r = bufs + (size_t)(b % CSUM_BUFS) * CSUM_BATCH;
    const uint32_t m = min(CSUM_BATCH, nrec - b * CSUM_BATCH);
    // the tests do not feed the chain: one dependent add per record
    const double s_in = s;
    bool bad = false;
#pragma unroll 4
    for (uint32_t k = 0; k < m; ++k) {
      const double lo = r[k].lo, hi = r[k].hi, a = r[k].a;
      bad |= !(s >= lo && s <= hi);
      s += a;
    }
    if (bad) {
      // some entry test failed (or s is not finite): rerun with the tests
      ++reruns;
      s = s_in;
      for (uint32_t k = 0; k < m; ++k) {
        const CsumRec d = r[k];
        if (d.meta == 0 || (s >= d.lo && s <= d.hi)) {
          s += d.a;
        } else {
          const uint32_t i0 = (uint32_t)(d.meta >> 16), len = (uint32_t)(d.meta & 0xffffu);
          for (uint32_t i = i0; i < i0 + len; ++i) s += v[i];
          ++failed;
        }
      }
    }
    if (b + CSUM_BUFS < nb) issue(b + CSUM_BUFS);
  }
  // every copy in flight lands before the block exits
  for (uint32_t q = b; q < nb && q < b + CSUM_BUFS; ++q)
    mbar_wait(&bar[q % CSUM_BUFS], (q / CSUM_BUFS) & 1u);
  if (!ok) atomicOr(status, ST_WAIT_TIMEOUT);
  out[ax] = s;
  stamps[3 + ax] = gtimer_ns();
  if (ax == 0) {
    stamps[5] = reruns;
    stamps[6] = failed;
    stamps[7] = nrec;
  }
}

// Small node counts: the two serial sums themselves, one warp on one SM
// (lane 0 x, lane 1 y, in lockstep: one dependent add per value), the values
// staged into shared memory by bulk copies. At 50k values this is ~0.27 ms
// and overlaps the forces entirely, where the record pipeline above spreads
// over many SMs and launches and, on a running sum that keeps crossing zero
// (short stretches), walks nearly as many records as values.
constexpr uint32_t CSUM_SERIAL_MAX = 1u << 16;
constexpr unsigned CSUM_TILE = 1024;  // values per copy and axis (8 KB)
constexpr unsigned CSUM_STAGES = 4;
constexpr size_t CSUM_SERIAL_SMEM = 2ull * CSUM_STAGES * CSUM_TILE * sizeof(double);

// stamps as k_csum_walk's (5-7 zero: no records).
__global__ void __launch_bounds__(32) k_csum_serial(const double *x, const double *y, uint32_t n,
                                                    double *out, uint32_t *status,
                                                    unsigned long long *stamps) {
  extern __shared__ __align__(128) unsigned char csum_smem[];
  __shared__ __align__(8) uint64_t bar[CSUM_STAGES];
  double *buf = reinterpret_cast<double *>(csum_smem);  // [stage][axis][CSUM_TILE]
  const unsigned lane = threadIdx.x;
  if (lane == 0) {
    stamps[0] = stamps[1] = stamps[2] = gtimer_ns();
    for (unsigned q = 0; q < CSUM_STAGES; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const uint32_t nt = (n + CSUM_TILE - 1) / CSUM_TILE;
  // tile t: its even-length head by two bulk copies (sizes in 16-byte
  // units), an odd last value by a plain load
  auto issue = [&](uint32_t t) {
    const uint32_t k0 = t * CSUM_TILE, m = min(CSUM_TILE, n - k0), mb = m & ~1u;
    uint64_t *b = &bar[t % CSUM_STAGES];
    double *d = buf + (size_t)(t % CSUM_STAGES) * 2 * CSUM_TILE;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
                 "r"(mb * 16u)
                 : "memory");
    if (mb) {
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(d)),
          "l"(x + k0), "r"(mb * 8u), "r"(smem_addr(b))
          : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(d + CSUM_TILE)),
          "l"(y + k0), "r"(mb * 8u), "r"(smem_addr(b))
          : "memory");
    }
  };
  if (lane == 0)
    for (uint32_t t = 0; t < CSUM_STAGES && t < nt; ++t) issue(t);
  __syncwarp();
  const double *v = lane == 1 ? y : x;
  double s = 0;
  bool ok = true;
  uint32_t t = 0;
  for (; t < nt; ++t) {
    bool w = true;
    if (lane < 2) w = mbar_wait(&bar[t % CSUM_STAGES], (t / CSUM_STAGES) & 1u);
    if (!__all_sync(0xffffffffu, w)) {
      ok = false;
      break;
    }
    const uint32_t k0 = t * CSUM_TILE, m = min(CSUM_TILE, n - k0), mb = m & ~1u;
    if (lane < 2) {
      const double *d = buf + ((size_t)(t % CSUM_STAGES) * 2 + lane) * CSUM_TILE;
      if (mb == CSUM_TILE) {
#pragma unroll 16
        for (uint32_t k = 0; k < CSUM_TILE; ++k) s += d[k];
      } else {
        for (uint32_t k = 0; k < mb; ++k) s += d[k];
      }
      if (mb < m) s += v[k0 + mb];
    }
    // the stage is refilled after both lanes have added its values
    __syncwarp();
    if (lane == 0 && t + CSUM_STAGES < nt) issue(t + CSUM_STAGES);
  }
  // every copy in flight lands before the block exits
  if (lane == 0)
    for (uint32_t q = t; q < nt && q < t + CSUM_STAGES; ++q)
      mbar_wait(&bar[q % CSUM_STAGES], (q / CSUM_STAGES) & 1u);
  if (lane < 2) {
    out[lane] = s;
    stamps[3 + lane] = gtimer_ns();
  }
  if (lane == 0) {
    stamps[5] = stamps[6] = stamps[7] = 0;
    if (!ok) atomicOr(status, ST_WAIT_TIMEOUT);
  }
}

__global__ void k_center_apply(double *x, double *y, uint32_t n, const double *sums, double cx,
                               double cy, double strength) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double nf = (double)n;
  const double sx = (sums[0] / nf - cx) * strength;
  const double sy = (sums[1] / nf - cy) * strength;
  x[i] -= sx;
  y[i] -= sy;
}

__global__ void k_set_status(uint32_t *status, uint32_t bits) { atomicOr(status, bits); }

void set_status(uint32_t *status, uint32_t bits, cudaStream_t st) {
  D3_LAUNCH(k_set_status, 1, 1, 0, st)(status, bits);
}

void center_sum(const NodeArrays &a, ForceScratch &s, uint32_t *status, cudaStream_t st) {
  if (a.n == 0) return;
  if (a.n <= CSUM_SERIAL_MAX && ((uintptr_t)a.x & 15) == 0 && ((uintptr_t)a.y & 15) == 0) {
    static bool sattr = [] {
      return cudaFuncSetAttribute(k_csum_serial, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)CSUM_SERIAL_SMEM) == cudaSuccess;
    }();
    D3_LAUNCH(k_csum_serial, 1, 32, CSUM_SERIAL_SMEM, st)(a.x, a.y, a.n, s.center, status,
                                                          s.csum_stamps);
    if (!sattr || cudaGetLastError() != cudaSuccess) set_status(status, ST_CENTER_RECORDS, st);
    return;
  }
  static bool attr = [] {
    return cudaFuncSetAttribute(k_csum_walk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)CSUM_WALK_SMEM) == cudaSuccess;
  }();
  const CsumGeom g = csum_geom(a.n);
  CsumRec *recs = static_cast<CsumRec *>(s.csum_recs);
  uint32_t *counts = s.csum_counts, *offsets = s.csum_counts + 2 * g.nc + 1;
  const unsigned cb = blocks_for(g.nc, 256);
  D3_LAUNCH(k_csum_part, blocks_for((size_t)g.nc * 32, 256), 256, 0, st)(a.x, a.y, a.n, g, s.csum_part);
  D3_LAUNCH(k_csum_records<false>, cb, 256, 0, st)(a.x, a.y, a.n, g, s.csum_part, counts, nullptr,
                                                   nullptr, status);
  // offsets of both axes' records; offsets[2 nc] = the total
  scan_u32(counts, offsets, 2 * g.nc, s.csum_scan_part, offsets + 2 * g.nc, st);
  D3_LAUNCH(k_csum_records<true>, cb, 256, 0, st)(a.x, a.y, a.n, g, s.csum_part, counts, offsets,
                                                  recs, status);
  D3_LAUNCH(k_csum_walk, 1, 64, CSUM_WALK_SMEM, st)(a.x, a.y, g, recs, offsets, s.center, status,
                                                    s.csum_stamps);
  // a launch that did not happen leaves stale sums: report it as a failure
  if (!attr || cudaGetLastError() != cudaSuccess) set_status(status, ST_CENTER_RECORDS, st);
}

// One block: s.center = the sums of the chunk sums in chunk order (a fixed
// tree: lane-strided partials, then a shuffle tree).
__global__ void __launch_bounds__(1024) k_csum_tree(const double *part, uint32_t nc, double *out) {
  __shared__ double wx[32], wy[32];
  double ax = 0, ay = 0;
  for (uint32_t c = threadIdx.x; c < nc; c += blockDim.x) {
    ax += part[c];
    ay += part[nc + c];
  }
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
  }
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    wx[warp] = ax;
    wy[warp] = ay;
  }
  __syncthreads();
  if (warp == 0) {
    const unsigned nw = blockDim.x >> 5;
    ax = lane < nw ? wx[lane] : 0.0;
    ay = lane < nw ? wy[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      ax += __shfl_xor_sync(0xffffffffu, ax, o);
      ay += __shfl_xor_sync(0xffffffffu, ay, o);
    }
    if (lane == 0) {
      out[0] = ax;
      out[1] = ay;
    }
  }
}

void center_sum_tree(const NodeArrays &a, ForceScratch &s, cudaStream_t st) {
  if (a.n == 0) return;
  const CsumGeom g = csum_geom(a.n);
  D3_LAUNCH(k_csum_part, blocks_for((size_t)g.nc * 32, 256), 256, 0, st)(a.x, a.y, a.n, g, s.csum_part);
  D3_LAUNCH(k_csum_tree, 1, 1024, 0, st)(s.csum_part, g.nc, s.center);
}

void center_apply(const NodeArrays &a, double cx, double cy, double strength, ForceScratch &s,
                  cudaStream_t st) {
  if (a.n == 0) return;
  D3_LAUNCH(k_center_apply, blocks_for(a.n, 256), 256, 0, st)(a.x, a.y, a.n, s.center, cx, cy, strength);
}

// src/core.js:130 on the device: fixed = (fx set) | (fy set) << 1, a missing
// value being NaN.
__global__ void k_fixed_from_f(const double *fx, const double *fy, uint8_t *fixed, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = fx[i], b = fy[i];
  fixed[i] = (uint8_t)((a == a ? 1u : 0u) | (b == b ? 2u : 0u));
}

void fixed_from_f(const double *fx, const double *fy, uint8_t *fixed, uint32_t n, cudaStream_t st) {
  if (n == 0) return;
  D3_LAUNCH(k_fixed_from_f, blocks_for(n, 256), 256, 0, st)(fx, fy, fixed, n);
}

// simulation.js:157-178 (find). The serial scan keeps the first node whose d2
// is strictly below its best so far (starting at radius^2): the lowest index
// of the least d2 below radius^2. One block: each thread runs that scan over
// its own nodes (ascending indices), then the block keeps the least (d2,
// index) pair. A NaN d2 never passes the strict test.
constexpr unsigned FIND_THREADS = 1024;

__device__ inline void find_merge(double &d, uint32_t &i, double d2, uint32_t i2) {
  if (i2 != NONE && (i == NONE || d2 < d || (d2 == d && i2 < i))) {
    d = d2;
    i = i2;
  }
}

__global__ void __launch_bounds__(FIND_THREADS) k_find(const double *xs, const double *ys, uint32_t n,
                                                       double x, double y, double r2,
                                                       uint32_t *out) {
  __shared__ double sd[FIND_THREADS / 32];
  __shared__ uint32_t si[FIND_THREADS / 32];
  double best = r2;
  uint32_t bi = NONE;
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    const double dx = x - xs[k], dy = y - ys[k];
    const double d2 = dx * dx + dy * dy;
    if (d2 < best) {
      best = d2;
      bi = k;
    }
  }
  for (int o = 16; o > 0; o >>= 1)
    find_merge(best, bi, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, bi, o));
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sd[warp] = best;
    si[warp] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (unsigned w = 1; w < blockDim.x / 32; ++w) find_merge(best, bi, sd[w], si[w]);
    *out = bi;
  }
}

void find_closest(const NodeArrays &a, double x, double y, double r2, uint32_t *out,
                  cudaStream_t st) {
  D3_LAUNCH(k_find, 1, FIND_THREADS, 0, st)(a.x, a.y, a.n, x, y, r2, out);
}

// simple.zig:51-62
__global__ void k_axis(double *pos, double *v, const double *strength, const double *target,
                       double alpha, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  v[i] += (target[i] - pos[i]) * strength[i] * alpha;
}

void axis_force(const NodeArrays &a, const double *strength, const double *target, double alpha,
                int dim, cudaStream_t st) {
  if (a.n == 0) return;
  D3_LAUNCH(k_axis, blocks_for(a.n, 256), 256, 0, st)(dim ? a.y : a.x, dim ? a.vy : a.vx, strength, target,
                                               alpha, a.n);
}

// simple.zig:64-86
__global__ void k_radial(const double *x, const double *y, double *vx, double *vy,
                         const double *strength, const double *radius, double cx, double cy,
                         double alpha, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dx = x[i] - cx;
  if (dx == 0 || dx != dx) dx = 1e-6;
  double dy = y[i] - cy;
  if (dy == 0 || dy != dy) dy = 1e-6;
  double l = sqrt(dx * dx + dy * dy);
  double k = (radius[i] - l) * strength[i] * alpha / l;
  vx[i] += dx * k;
  vy[i] += dy * k;
}

void radial_force(const NodeArrays &a, const double *strength, const double *radius, double cx,
                  double cy, double alpha, cudaStream_t st) {
  if (a.n == 0) return;
  D3_LAUNCH(k_radial, blocks_for(a.n, 256), 256, 0, st)(a.x, a.y, a.vx, a.vy, strength, radius, cx, cy,
                                                 alpha, a.n);
}

// simple.zig:90-123
__global__ void k_integrate(double *x, double *y, double *vx, double *vy, const double *fx,
                            const double *fy, const uint8_t *fixed, double decay, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t f = fixed[i];
  if ((f & 1) == 0) {
    double v = vx[i] * decay;
    vx[i] = v;
    x[i] += v;
  } else {
    x[i] = fx[i];
    vx[i] = 0;
  }
  if ((f & 2) == 0) {
    double v = vy[i] * decay;
    vy[i] = v;
    y[i] += v;
  } else {
    y[i] = fy[i];
    vy[i] = 0;
  }
}

// k_center_apply then k_integrate, per node in one pass (both are per node).
__global__ void k_center_integrate(double *x, double *y, double *vx, double *vy, const double *fx,
                                   const double *fy, const uint8_t *fixed, const double *sums,
                                   double cx, double cy, double strength, double decay,
                                   uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double nf = (double)n;
  const double sx = (sums[0] / nf - cx) * strength;
  const double sy = (sums[1] / nf - cy) * strength;
  const double x0 = x[i] - sx, y0 = y[i] - sy;
  const uint8_t f = fixed[i];
  if ((f & 1) == 0) {
    double v = vx[i] * decay;
    vx[i] = v;
    x[i] = x0 + v;
  } else {
    x[i] = fx[i];
    vx[i] = 0;
  }
  if ((f & 2) == 0) {
    double v = vy[i] * decay;
    vy[i] = v;
    y[i] = y0 + v;
  } else {
    y[i] = fy[i];
    vy[i] = 0;
  }
}

void center_apply_integrate(const NodeArrays &a, double cx, double cy, double strength,
                            ForceScratch &s, double decay, cudaStream_t st) {
  if (a.n == 0) return;
  D3_LAUNCH(k_center_integrate, blocks_for(a.n, 256), 256, 0, st)(a.x, a.y, a.vx, a.vy, a.fx, a.fy,
                                                           a.fixed, s.center, cx, cy, strength,
                                                           decay, a.n);
}

void integrate(const NodeArrays &a, double decay, cudaStream_t st) {
  if (a.n == 0) return;
  D3_LAUNCH(k_integrate, blocks_for(a.n, 256), 256, 0, st)(a.x, a.y, a.vx, a.vy, a.fx, a.fy, a.fixed, decay,
                                                    a.n);
}

}  // namespace d3
