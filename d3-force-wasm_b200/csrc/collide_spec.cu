// collide_spec.cu — exact forceCollide in parallel, bit-identical to the
// ordered node loop of collide.zig:47-100 (d3's collide.js).
//
// In the reference, node i's turn reads its own velocity and the velocity of
// every leaf head j > i it examines, and writes velocities only where it finds
// an overlap; later turns read what earlier turns wrote. Two turns commute
// unless one writes something the other reads or writes. The kernel runs the
// turns as a dependency DAG, in one cooperative launch:
//
//  G. Guess, per node, from the pass-start state and a margin `delta`: the heads
//     it may examine (R) and those it may overlap (W, a mask over R). A node
//     with W empty is inactive: it cannot write unless something moves by
//     `delta` before its turn.
//  E. Rounds over the active nodes: a node runs when no earlier unfinished
//     active node writes what it reads or accesses what it writes (per-node
//     "earliest accessor / writer" marks by 64-bit atomicMin, tagged with the
//     round so no reset is needed). A running node traverses exactly as d3
//     and writes only if everything it examined / overlapped was guessed.
//  V. Inactive nodes are checked with the push magnitudes the pass applied
//     (a node's position at its turn moved by at most the pushes it received
//     from earlier nodes): if i and every guessed head stayed within `delta`,
//     i's turn was a no-op, as guessed.
//  Any failure promotes the failing nodes (every guessed head may be written),
//  restores the pass-start velocities and runs E and V again; after 3
//  attempts, or when a turn would draw from `random` (a zero delta), block 0
//  runs the serial loop itself on the restored state.
#include <cooperative_groups.h>

#include "forces.cuh"

namespace cg = cooperative_groups;

namespace d3 {

constexpr int SPEC_CAP = 64;        // guessed heads per node (R)
constexpr int SPEC_ATTEMPTS = 3;
constexpr uint32_t SPEC_MAX_ROUNDS = 4096;
constexpr unsigned SPEC_THREADS = 256;

enum : uint32_t { C_ACTIVE = 0, C_DONE, C_FAIL, C_JIGGLE, C_OVERFLOW, C_ROUNDS, C_ATTEMPTS, C_SERIAL };

struct SpecArgs {
  const Cell *cells;
  const uint32_t *skip, *perm, *info;
  const double *xs, *ys, *px, *py, *radii;
  double *vxs, *vys, *svx, *svy;
  double strength, delta;
  uint32_t n;
  uint32_t *rlist;       // n * SPEC_CAP
  uint8_t *rcount;       // n
  uint64_t *wmask;       // n
  uint8_t *state;        // n: 0 inactive, 1 pending, 2 done
  uint32_t *active;      // active node list
  uint64_t *min_acc, *min_wr;  // tagged marks per node
  double *push;          // push magnitude received per node
  uint32_t *min_pusher;  // lowest pusher index per node
  uint32_t *counters;    // C_*
  Rng *rng;
};

// Mutable data is read through L2 (ld.global.cg): other SMs write it between
// the grid-wide barriers and L1 is not coherent across SMs.
__device__ inline double rd(const double *p) { return __ldcg(p); }
__device__ inline uint32_t rd(const uint32_t *p) { return __ldcg(p); }
__device__ inline uint64_t rd(const uint64_t *p) { return __ldcg((const unsigned long long *)p); }
__device__ inline uint8_t rd(const uint8_t *p) { return (uint8_t)__ldcg((const unsigned char *)p); }

// G: guessed heads (j > i) with pruning relaxed by `margin`, and a mask of the
// heads within r + margin of the pass-start positions.
__device__ bool spec_guess(const SpecArgs &a, uint32_t i, double margin, bool all_writes) {
  const uint32_t len = a.info[1];
  const double xi = a.px[i], yi = a.py[i], ri = a.radii[i];
  uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  uint32_t nr = 0;
  uint64_t wm = 0;
  a.rcount[i] = 0;
  a.wmask[i] = 0;
  for (uint32_t c = 0; c < len;) {
    const Cell &q = a.cells[c];
    const double r = ri + q.r;
    if (is_leaf(q)) {
      const uint32_t j = a.perm[q.first + q.count - 1];
      if (j > i) {
        if (nr == SPEC_CAP) return false;
        const double dx = xi - a.px[j], dy = yi - a.py[j];
        const double rr = r + margin;
        if (all_writes || dx * dx + dy * dy < rr * rr) wm |= 1ull << nr;
        rl[nr++] = j;
      }
      c = c + 1;
      continue;
    }
    if (q.x0 > xi + r + margin || q.x1 < xi - r - margin || q.y0 > yi + r + margin ||
        q.y1 < yi - r - margin)
      c = a.skip[c];
    else
      c = c + 1;
  }
  a.rcount[i] = (uint8_t)nr;
  a.wmask[i] = wm;
  return true;
}

__device__ inline int spec_find(const uint32_t *rl, uint32_t nr, uint32_t j) {
  for (uint32_t k = 0; k < nr; ++k)
    if (rd(&rl[k]) == j) return (int)k;
  return -1;
}

// E: node i's turn, exactly collide.zig:48-99; writes only if every examined
// head and every overlap was guessed and no zero delta occurs.
__device__ void spec_turn(const SpecArgs &a, uint32_t i) {
  const uint32_t len = a.info[1];
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  const double ri = a.radii[i], ri2 = ri * ri;
  double vi = rd(&a.vxs[i]), wi = rd(&a.vys[i]);
  const double xi = a.xs[i] + vi, yi = a.ys[i] + wi;
  uint32_t pj[SPEC_CAP];
  double pdx[SPEC_CAP], pdy[SPEC_CAP];
  uint32_t np = 0;
  for (uint32_t c = 0; c < len;) {
    const Cell &q = a.cells[c];
    double rj = q.r;
    double r = ri + rj;
    if (is_leaf(q)) {
      const uint32_t j = a.perm[q.first + q.count - 1];
      if (j > i) {
        const int k = spec_find(rl, nr, j);
        if (k < 0) {
          atomicAdd(&a.counters[C_FAIL], 1u);
          a.state[i] = 3;  // failed: promote
          return;
        }
        double x = xi - a.xs[j] - rd(&a.vxs[j]);
        double y = yi - a.ys[j] - rd(&a.vys[j]);
        double l = x * x + y * y;
        if (l < r * r) {
          if (!((wm >> k) & 1)) {
            atomicAdd(&a.counters[C_FAIL], 1u);
            a.state[i] = 3;
            return;
          }
          if (x == 0 || y == 0) {
            atomicAdd(&a.counters[C_JIGGLE], 1u);
            return;
          }
          l = sqrt(l);
          l = (r - l) / l * a.strength;
          x *= l;
          y *= l;
          rj *= rj;
          r = rj / (ri2 + rj);
          vi += x * r;
          wi += y * r;
          r = 1 - r;
          pj[np] = j;
          pdx[np] = x * r;
          pdy[np] = y * r;
          ++np;
        }
      }
      c = c + 1;
      continue;
    }
    if (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r) c = a.skip[c];
    else c = c + 1;
  }
  a.vxs[i] = vi;
  a.vys[i] = wi;
  for (uint32_t k = 0; k < np; ++k) {
    const uint32_t j = pj[k];
    a.vxs[j] = rd(&a.vxs[j]) - pdx[k];
    a.vys[j] = rd(&a.vys[j]) - pdy[k];
    atomicAdd(&a.push[j], sqrt(pdx[k] * pdx[k] + pdy[k] * pdy[k]));
    atomicMin(&a.min_pusher[j], i);
  }
}

__device__ bool spec_ready(const SpecArgs &a, uint32_t i, uint64_t tag) {
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  // self: read and written
  uint64_t v = __ldcg((const unsigned long long *)&a.min_acc[i]);
  if ((v >> 32) == tag && (uint32_t)v < i) return false;
  for (uint32_t k = 0; k < nr; ++k) {
    const uint32_t j = rd(&rl[k]);
    if ((wm >> k) & 1) {
      v = __ldcg((const unsigned long long *)&a.min_acc[j]);
      if ((v >> 32) == tag && (uint32_t)v < i) return false;
    } else {
      v = __ldcg((const unsigned long long *)&a.min_wr[j]);
      if ((v >> 32) == tag && (uint32_t)v < i) return false;
    }
  }
  return true;
}

__device__ void spec_mark(const SpecArgs &a, uint32_t i, uint64_t tag) {
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  const unsigned long long t = (tag << 32) | i;
  atomicMin((unsigned long long *)&a.min_acc[i], t);
  atomicMin((unsigned long long *)&a.min_wr[i], t);
  for (uint32_t k = 0; k < nr; ++k) {
    const uint32_t j = rd(&rl[k]);
    atomicMin((unsigned long long *)&a.min_acc[j], t);
    if ((wm >> k) & 1) atomicMin((unsigned long long *)&a.min_wr[j], t);
  }
}

// The serial loop (collide.zig:47-100) with draws from the device LCG.
__device__ void spec_serial(const SpecArgs &a) {
  const uint32_t len = a.info[1];
  uint32_t s = a.rng->lcg;
  for (uint32_t i = 0; i < a.n; ++i) {
    const double ri = a.radii[i], ri2 = ri * ri;
    const double xi = a.xs[i] + rd(&a.vxs[i]), yi = a.ys[i] + rd(&a.vys[i]);
    for (uint32_t c = 0; c < len;) {
      const Cell &q = a.cells[c];
      double rj = q.r;
      double r = ri + rj;
      if (is_leaf(q)) {
        const uint32_t j = a.perm[q.first + q.count - 1];
        if (j > i) {
          double x = xi - a.xs[j] - rd(&a.vxs[j]);
          double y = yi - a.ys[j] - rd(&a.vys[j]);
          double l = x * x + y * y;
          if (l < r * r) {
            if (x == 0) { s = lcg_step(s); x = (lcg_value(s) - 0.5) * 1e-6; l += x * x; }
            if (y == 0) { s = lcg_step(s); y = (lcg_value(s) - 0.5) * 1e-6; l += y * y; }
            l = sqrt(l);
            l = (r - l) / l * a.strength;
            x *= l;
            y *= l;
            rj *= rj;
            r = rj / (ri2 + rj);
            a.vxs[i] = rd(&a.vxs[i]) + x * r;
            a.vys[i] = rd(&a.vys[i]) + y * r;
            r = 1 - r;
            a.vxs[j] = rd(&a.vxs[j]) - x * r;
            a.vys[j] = rd(&a.vys[j]) - y * r;
          }
        }
        c = c + 1;
        continue;
      }
      if (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r) c = a.skip[c];
      else c = c + 1;
    }
  }
  a.rng->lcg = s;
}

__global__ void __launch_bounds__(SPEC_THREADS) k_collide_spec(SpecArgs a) {
  cg::grid_group g = cg::this_grid();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t n = a.n;
  if (tid < 8) a.counters[tid] = 0;
  g.sync();
  // G, plus per-node resets and the pass-start snapshot.
  for (uint32_t i = tid; i < n; i += nth) {
    a.svx[i] = a.vxs[i];
    a.svy[i] = a.vys[i];
    a.min_acc[i] = ~0ull;
    a.min_wr[i] = ~0ull;
    a.push[i] = 0;
    a.min_pusher[i] = NONE;
    if (!spec_guess(a, i, a.delta, false)) {
      atomicAdd(&a.counters[C_OVERFLOW], 1u);
      a.state[i] = 0;
      continue;
    }
    if (a.wmask[i]) {
      a.state[i] = 1;
      a.active[atomicAdd(&a.counters[C_ACTIVE], 1u)] = i;
    } else {
      a.state[i] = 0;
    }
  }
  g.sync();
  bool ok = false;
  uint32_t round_base = 0;
  for (int attempt = 0; attempt < SPEC_ATTEMPTS && !ok; ++attempt) {
    if (__ldcg(&a.counters[C_OVERFLOW]) || __ldcg(&a.counters[C_JIGGLE])) break;
    const uint32_t n_active = __ldcg(&a.counters[C_ACTIVE]);
    for (uint32_t round = 0;; ++round) {
      if (round_base + round >= SPEC_MAX_ROUNDS) {
        if (tid == 0) atomicAdd(&a.counters[C_OVERFLOW], 1u);
        break;
      }
      const uint64_t tag = 0xFFFFFFFFull - (round_base + round);
      for (uint32_t k = tid; k < n_active; k += nth) {
        const uint32_t i = rd(&a.active[k]);
        if (rd(&a.state[i]) == 1) spec_mark(a, i, tag);
      }
      g.sync();
      for (uint32_t k = tid; k < n_active; k += nth) {
        const uint32_t i = rd(&a.active[k]);
        if (rd(&a.state[i]) != 1 || !spec_ready(a, i, tag)) continue;
        a.state[i] = 2;  // done (or 3 = failed, set by the turn)
        spec_turn(a, i);
        atomicAdd(&a.counters[C_DONE], 1u);
      }
      g.sync();
      if (__ldcg(&a.counters[C_DONE]) >= n_active) {
        round_base += round + 1;
        break;
      }
    }
    // V: inactive nodes stayed no-ops.
    for (uint32_t i = tid; i < n; i += nth) {
      if (rd(&a.state[i]) != 0) continue;
      // every push on i comes from an earlier node; on a head j > i only the
      // pushes of nodes before i count, bounded by all of them
      const double di = rd(&a.push[i]);
      bool bad = !(di < a.delta);
      const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
      const uint32_t nr = rd(&a.rcount[i]);
      for (uint32_t k = 0; k < nr && !bad; ++k) {
        const uint32_t j = rd(&rl[k]);
        const double dj = rd(&a.min_pusher[j]) < i ? rd(&a.push[j]) : 0.0;
        if (!(di + dj < a.delta)) bad = true;
      }
      if (bad) {
        a.state[i] = 4;  // inactive, moved too far: promote
        atomicAdd(&a.counters[C_FAIL], 1u);
      }
    }
    g.sync();
    if (tid == 0) atomicAdd(&a.counters[C_ATTEMPTS], 1u);
    if (__ldcg(&a.counters[C_FAIL]) == 0 && __ldcg(&a.counters[C_DONE]) >= n_active &&
        __ldcg(&a.counters[C_JIGGLE]) == 0) {
      ok = true;
      break;
    }
    // Retry: restore, promote failed nodes, requeue every active node.
    for (uint32_t i = tid; i < n; i += nth) {
      a.vxs[i] = a.svx[i];
      a.vys[i] = a.svy[i];
      a.push[i] = 0;
      a.min_pusher[i] = NONE;
      const uint8_t st = rd(&a.state[i]);
      if (st == 3 || st == 4) {
        // examined something unguessed, or moved too far: every head within
        // a wider margin may be written
        if (!spec_guess(a, i, 4 * a.delta, true)) atomicAdd(&a.counters[C_OVERFLOW], 1u);
        if (st == 4) a.active[atomicAdd(&a.counters[C_ACTIVE], 1u)] = i;  // was inactive
        a.state[i] = 1;
      } else if (st == 2) {
        a.state[i] = 1;
      }
    }
    g.sync();
    if (tid == 0) {
      a.counters[C_FAIL] = 0;
      a.counters[C_DONE] = 0;
    }
    g.sync();
  }
  if (ok) {
    if (tid == 0) a.counters[C_ROUNDS] = round_base;
    return;
  }
  // Fallback: the serial loop on the restored pass-start state.
  for (uint32_t i = tid; i < n; i += nth) {
    a.vxs[i] = a.svx[i];
    a.vys[i] = a.svy[i];
  }
  g.sync();
  if (tid == 0) {
    a.counters[C_SERIAL] = 1;
    spec_serial(a);
  }
}

static int g_spec_blocks = 0;

int collide_spec_reserve(CollideSpec &s, uint32_t n) {
  if (n <= s.cap && s.cap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  cudaFree(s.rlist); cudaFree(s.rcount); cudaFree(s.wmask); cudaFree(s.state); cudaFree(s.active);
  cudaFree(s.min_acc); cudaFree(s.min_wr); cudaFree(s.push); cudaFree(s.min_pusher);
  if (!s.counters) {
    D3_CUDA_OK(cudaMalloc(&s.counters, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(s.counters, 0, 16 * sizeof(uint32_t)));
  }
  D3_CUDA_OK(cudaMalloc(&s.rlist, (size_t)cap * SPEC_CAP * 4));
  D3_CUDA_OK(cudaMalloc(&s.rcount, cap));
  D3_CUDA_OK(cudaMalloc(&s.wmask, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.state, cap));
  D3_CUDA_OK(cudaMalloc(&s.active, 2ull * cap * 4));
  D3_CUDA_OK(cudaMalloc(&s.min_acc, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.min_wr, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.push, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.min_pusher, cap * 4ull));
  s.cap = cap;
  return 0;
}

void collide_spec_free(CollideSpec &s) {
  cudaFree(s.rlist); cudaFree(s.rcount); cudaFree(s.wmask); cudaFree(s.state); cudaFree(s.active);
  cudaFree(s.min_acc); cudaFree(s.min_wr); cudaFree(s.push); cudaFree(s.min_pusher);
  cudaFree(s.counters);
  s = CollideSpec();
}

int collide_parallel(TreeDev &t, const NodeArrays &a, const double *radii, double strength,
                     double delta, Rng *rng, CollideSpec &s, cudaStream_t st) {
  if (a.n == 0) return 0;
  if (!g_spec_blocks) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_collide_spec, SPEC_THREADS, 0);
    g_spec_blocks = sms * (per > 4 ? 4 : per);
    if (g_spec_blocks <= 0) g_spec_blocks = sms;
  }
  SpecArgs args;
  args.cells = t.cells; args.skip = t.skip; args.perm = t.perm; args.info = t.info;
  args.xs = a.x; args.ys = a.y; args.px = a.px; args.py = a.py; args.radii = radii;
  args.vxs = a.vx; args.vys = a.vy; args.svx = a.snap_vx; args.svy = a.snap_vy;
  args.strength = strength; args.delta = delta; args.n = a.n;
  args.rlist = s.rlist; args.rcount = s.rcount; args.wmask = s.wmask; args.state = s.state;
  args.active = s.active; args.min_acc = s.min_acc; args.min_wr = s.min_wr; args.push = s.push;
  args.min_pusher = s.min_pusher; args.counters = s.counters; args.rng = rng;
  void *params[] = {&args};
  ++g_launches;
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_collide_spec, g_spec_blocks,
                                              SPEC_THREADS, params, 0, st);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace d3
