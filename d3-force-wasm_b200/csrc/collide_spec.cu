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
constexpr int VISIT_CAP = 128;      // recorded margin-visited cells per node
constexpr uint16_t VISIT_NONE = 0xffff;
constexpr int SPEC_ATTEMPTS = 3;
constexpr uint32_t SPEC_MAX_ROUNDS = 4096;
constexpr unsigned SPEC_THREADS = 256;

enum : uint32_t {
  C_ACTIVE = 0, C_DONE, C_FAIL, C_JIGGLE, C_OVERFLOW, C_ROUNDS, C_ATTEMPTS, C_SERIAL,
  C_FAIL_READ, C_FAIL_WRITE, C_FAIL_MOVED, C_FAST_TURNS, C_SLOW_TURNS
};

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
  uint64_t *emask;       // n: heads the exact traversal from the pass start visits
  uint32_t *vlist;       // n * VISIT_CAP: cells the margin traversal entered, preorder
  uint16_t *vcount;      // n (VISIT_NONE: not recorded)
  uint8_t *state;        // n: 0 inactive, 1 pending, 2 done
  uint32_t *active;      // active node list
  uint64_t *min_acc, *min_wr;  // tagged marks per node
  double *push;          // push magnitude received per node
  uint32_t *min_pusher;  // lowest pusher index per node
  uint32_t *max_pusher;  // highest pusher index per node
  uint32_t *counters;    // C_*
  unsigned long long *stamps;  // phase timestamps (ns): G end, then per attempt rounds / V ends
  Rng *rng;
};

// Mutable data is read through L2 (ld.global.cg): other SMs write it between
// the grid-wide barriers and L1 is not coherent across SMs.
__device__ inline double rd(const double *p) { return __ldcg(p); }
__device__ inline uint32_t rd(const uint32_t *p) { return __ldcg(p); }
__device__ inline uint64_t rd(const uint64_t *p) { return __ldcg((const unsigned long long *)p); }
__device__ inline uint8_t rd(const uint8_t *p) { return (uint8_t)__ldcg((const unsigned char *)p); }
__device__ inline uint16_t rd(const uint16_t *p) { return (uint16_t)__ldcg((const unsigned short *)p); }

// G: guessed heads (j > i) with pruning relaxed by `margin`, a mask of the
// heads within r + margin of the pass-start positions, and a mask of the heads
// the exact traversal from the pass-start position visits (those in a subtree
// the exact test prunes are skipped via ex_until, the end of that subtree).
__device__ bool spec_guess(const SpecArgs &a, uint32_t i, double margin, bool all_writes) {
  const uint32_t len = a.info[1];
  const double xi = a.px[i], yi = a.py[i], ri = a.radii[i];
  uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  uint32_t *vl = a.vlist + (size_t)i * VISIT_CAP;
  uint32_t nr = 0, ex_until = 0, nv = 0;
  uint64_t wm = 0, em = 0;
  a.rcount[i] = 0;
  a.wmask[i] = 0;
  a.emask[i] = 0;
  for (uint32_t c = 0; c < len;) {
    const Cell &q = a.cells[c];
    const double r = ri + q.r;
    const bool ex_vis = c >= ex_until;
    if (is_leaf(q)) {
      const uint32_t j = a.perm[q.first + q.count - 1];
      if (nv < VISIT_CAP) vl[nv] = c;
      ++nv;
      if (j > i) {
        if (nr == SPEC_CAP) return false;
        const double dx = xi - a.px[j], dy = yi - a.py[j];
        const double rr = r + margin;
        if (all_writes || dx * dx + dy * dy < rr * rr) wm |= 1ull << nr;
        if (ex_vis) em |= 1ull << nr;
        rl[nr++] = j;
      }
      c = c + 1;
      continue;
    }
    if (q.x0 > xi + r + margin || q.x1 < xi - r - margin || q.y0 > yi + r + margin ||
        q.y1 < yi - r - margin) {
      c = a.skip[c];
      continue;
    }
    if (ex_vis && (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r))
      ex_until = a.skip[c];
    if (nv < VISIT_CAP) vl[nv] = c;
    ++nv;
    c = c + 1;
  }
  a.rcount[i] = (uint8_t)nr;
  a.wmask[i] = wm;
  a.emask[i] = em;
  a.vcount[i] = nv <= VISIT_CAP ? (uint16_t)nv : VISIT_NONE;
  return true;
}

__device__ inline int spec_find(const uint32_t *rl, uint32_t nr, uint32_t j) {
  for (uint32_t k = 0; k < nr; ++k)
    if (rd(&rl[k]) == j) return (int)k;
  return -1;
}

__device__ inline bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}

// The exact traversal of node i from (xi, yi), replayed over the cells its
// margin traversal entered (in preorder): every cell the exact traversal
// enters is among them while i stays within `delta` of the pass start, and a
// subtree the exact test prunes is skipped to its end. `visit(j, k, rj)` is
// called for each examined head j > i (k its index among the guessed heads);
// returns false to stop. Returns -1 when the replay does not apply (no
// record, or i moved too far), 0 when stopped, 1 when done.
template <typename F>
__device__ int spec_replay(const SpecArgs &a, uint32_t i, double xi, double yi, F visit) {
  const uint16_t nv = rd(&a.vcount[i]);
  if (nv == VISIT_NONE) return -1;
  const double slack = a.delta * (1 - 1e-9);
  if (!(fabs(xi - a.px[i]) < slack && fabs(yi - a.py[i]) < slack)) return -1;
  const uint32_t *vl = a.vlist + (size_t)i * VISIT_CAP;
  const double ri = a.radii[i];
  uint32_t ex_until = 0;
  int k = 0;
  for (uint32_t t = 0; t < nv; ++t) {
    const uint32_t c = rd(&vl[t]);
    if (c < ex_until) continue;
    const Cell &q = a.cells[c];
    if (is_leaf(q)) {
      const uint32_t j = a.perm[q.first + q.count - 1];
      if (j > i) {
        if (!visit(j, k, q.r)) return 0;
        ++k;
      }
      continue;
    }
    const double r = ri + q.r;
    if (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r) ex_until = a.skip[c];
  }
  return 1;
}

// E: node i's turn, exactly collide.zig:48-99; writes only if every examined
// head and every overlap was guessed and no zero delta occurs. A node not
// pushed since the pass start sits where the guess traversed from, so it
// examines exactly the heads of its exact-visit mask, in that order, and needs
// no traversal.
__device__ void spec_turn(const SpecArgs &a, uint32_t i) {
  const uint32_t len = a.info[1];
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  const double ri = a.radii[i], ri2 = ri * ri;
  double vi = rd(&a.vxs[i]), wi = rd(&a.vys[i]);
  const double xi = a.xs[i] + vi, yi = a.ys[i] + wi;
  const bool fast = same_bits(vi, rd(&a.svx[i])) && same_bits(wi, rd(&a.svy[i]));
  uint32_t pj[SPEC_CAP];
  double pdx[SPEC_CAP], pdy[SPEC_CAP];
  uint32_t np = 0;
  // One examined head: false = the turn must not write (failure or jiggle).
  auto head = [&](uint32_t j, int k, double rj) -> bool {
    double r = ri + rj;
    double x = xi - a.xs[j] - rd(&a.vxs[j]);
    double y = yi - a.ys[j] - rd(&a.vys[j]);
    double l = x * x + y * y;
    if (!(l < r * r)) return true;
    if (!((wm >> k) & 1)) {
      atomicAdd(&a.counters[C_FAIL], 1u);
      atomicAdd(&a.counters[C_FAIL_WRITE], 1u);
      a.state[i] = 3;
      return false;
    }
    if (x == 0 || y == 0) {
      atomicAdd(&a.counters[C_JIGGLE], 1u);
      return false;
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
    return true;
  };
  if (fast) {
    uint64_t em = rd(&a.emask[i]);
    while (em) {
      const int k = __ffsll((long long)em) - 1;
      em &= em - 1;
      const uint32_t j = rd(&rl[k]);
      if (!head(j, k, a.radii[j])) return;
    }
    atomicAdd(&a.counters[C_FAST_TURNS], 1u);
  } else {
    for (uint32_t c = 0; c < len;) {
      const Cell &q = a.cells[c];
      const double r = ri + q.r;
      if (is_leaf(q)) {
        const uint32_t j = a.perm[q.first + q.count - 1];
        if (j > i) {
          const int k = spec_find(rl, nr, j);
          if (k < 0) {
            atomicAdd(&a.counters[C_FAIL], 1u);
            atomicAdd(&a.counters[C_FAIL_READ], 1u);
            a.state[i] = 3;
            return;
          }
          if (!head(j, k, q.r)) return;
        }
        c = c + 1;
        continue;
      }
      if (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r) c = a.skip[c];
      else c = c + 1;
    }
    atomicAdd(&a.counters[C_SLOW_TURNS], 1u);
  }
  a.vxs[i] = vi;
  a.vys[i] = wi;
  for (uint32_t k = 0; k < np; ++k) {
    const uint32_t j = pj[k];
    a.vxs[j] = rd(&a.vxs[j]) - pdx[k];
    a.vys[j] = rd(&a.vys[j]) - pdy[k];
    atomicAdd(&a.push[j], sqrt(pdx[k] * pdx[k] + pdy[k] * pdy[k]));
    atomicMin(&a.min_pusher[j], i);
    atomicMax(&a.max_pusher[j], i);
  }
}

// V: an inactive node's turn, re-run at its exact turn state. Its own
// velocity is final (every push on i comes from an earlier node); a head's is
// its start value if all its pushers come later, its final value if all came
// earlier, and otherwise only bounded (then a distance margin must hold).
// Returns false when the turn might examine or overlap something unguessed.
__device__ bool spec_inactive_ok(const SpecArgs &a, uint32_t i) {
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const double vi = rd(&a.vxs[i]), wi = rd(&a.vys[i]);
  bool any = !same_bits(vi, rd(&a.svx[i])) || !same_bits(wi, rd(&a.svy[i]));
  for (uint32_t k = 0; k < nr && !any; ++k) any = rd(&a.min_pusher[rd(&rl[k])]) != NONE;
  if (!any) return true;  // nothing it reads moved: the guess holds as computed
  const uint32_t len = a.info[1];
  const double ri = a.radii[i];
  const double xi = a.xs[i] + vi, yi = a.ys[i] + wi;
  // false: the head may overlap at i's turn
  auto clear = [&](uint32_t j, double rj) -> bool {
    const double r = ri + rj;
    const uint32_t lo = rd(&a.min_pusher[j]), hi = rd(&a.max_pusher[j]);
    double vj, wj;
    if (lo == NONE || lo > i) {
      vj = rd(&a.svx[j]);
      wj = rd(&a.svy[j]);
    } else if (hi < i) {
      vj = rd(&a.vxs[j]);
      wj = rd(&a.vys[j]);
    } else {
      // pushed before and after i's turn: bound the move by all pushes
      const double dx = xi - a.xs[j] - rd(&a.svx[j]), dy = yi - a.ys[j] - rd(&a.svy[j]);
      const double gap = sqrt(dx * dx + dy * dy) - r - rd(&a.push[j]);
      return gap > 1e-9 * (r + 1);
    }
    const double x = xi - a.xs[j] - vj, y = yi - a.ys[j] - wj;
    return !(x * x + y * y < r * r);
  };
  bool ok = true;
  const int rp = spec_replay(a, i, xi, yi, [&](uint32_t j, int, double rj) {
    ok = clear(j, rj);
    return ok;
  });
  if (rp >= 0) return ok;
  for (uint32_t c = 0; c < len;) {
    const Cell &q = a.cells[c];
    const double r = ri + q.r;
    if (is_leaf(q)) {
      const uint32_t j = a.perm[q.first + q.count - 1];
      if (j > i && (spec_find(rl, nr, j) < 0 || !clear(j, q.r))) return false;
      c = c + 1;
      continue;
    }
    if (q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r) c = a.skip[c];
    else c = c + 1;
  }
  return true;
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

__device__ inline unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void __launch_bounds__(SPEC_THREADS) k_collide_spec(SpecArgs a) {
  cg::grid_group g = cg::this_grid();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int k = 0; k < 16; ++k) a.stamps[k] = 0;
    a.stamps[0] = now_ns();
  }
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t n = a.n;
  if (tid < 16) a.counters[tid] = 0;
  g.sync();
  // G, plus per-node resets and the pass-start snapshot.
  for (uint32_t i = tid; i < n; i += nth) {
    a.svx[i] = a.vxs[i];
    a.svy[i] = a.vys[i];
    a.min_acc[i] = ~0ull;
    a.min_wr[i] = ~0ull;
    a.push[i] = 0;
    a.min_pusher[i] = NONE;
    a.max_pusher[i] = 0;
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
  if (tid == 0) a.stamps[1] = now_ns();
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
    if (tid == 0 && attempt < 3) a.stamps[2 + 2 * attempt] = now_ns();
    // V: inactive nodes stayed no-ops.
    for (uint32_t i = tid; i < n; i += nth) {
      if (rd(&a.state[i]) != 0) continue;
      if (!spec_inactive_ok(a, i)) {
        a.state[i] = 4;  // inactive, but its turn would write: promote
        atomicAdd(&a.counters[C_FAIL], 1u);
        atomicAdd(&a.counters[C_FAIL_MOVED], 1u);
      }
    }
    g.sync();
    if (tid == 0 && attempt < 3) a.stamps[3 + 2 * attempt] = now_ns();
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
      a.max_pusher[i] = 0;
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
    if (tid == 0) {
      a.counters[C_ROUNDS] = round_base;
      a.stamps[9] = now_ns();
    }
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
    a.stamps[9] = now_ns();
  }
}

static int g_spec_blocks = 0;

int collide_spec_reserve(CollideSpec &s, uint32_t n) {
  if (n <= s.cap && s.cap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  cudaFree(s.rlist); cudaFree(s.rcount); cudaFree(s.wmask); cudaFree(s.state); cudaFree(s.active);
  cudaFree(s.min_acc); cudaFree(s.min_wr); cudaFree(s.push); cudaFree(s.min_pusher);
  cudaFree(s.emask); cudaFree(s.max_pusher); cudaFree(s.vlist); cudaFree(s.vcount);
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
  D3_CUDA_OK(cudaMalloc(&s.emask, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.max_pusher, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.vlist, (size_t)cap * VISIT_CAP * 4));
  D3_CUDA_OK(cudaMalloc(&s.vcount, cap * 2ull));
  if (!s.stamps) D3_CUDA_OK(cudaMalloc(&s.stamps, 16 * sizeof(unsigned long long)));
  s.cap = cap;
  return 0;
}

void collide_spec_free(CollideSpec &s) {
  cudaFree(s.rlist); cudaFree(s.rcount); cudaFree(s.wmask); cudaFree(s.state); cudaFree(s.active);
  cudaFree(s.min_acc); cudaFree(s.min_wr); cudaFree(s.push); cudaFree(s.min_pusher);
  cudaFree(s.emask); cudaFree(s.max_pusher); cudaFree(s.vlist); cudaFree(s.vcount);
  cudaFree(s.counters); cudaFree(s.stamps);
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
    // one block per SM short of full occupancy, so a concurrent one-block
    // kernel (the center sums on the side stream) never delays the launch
    g_spec_blocks = sms * (per > 3 ? 3 : (per > 1 ? per - 1 : 1));
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
  args.emask = s.emask; args.max_pusher = s.max_pusher;
  args.vlist = s.vlist; args.vcount = s.vcount; args.stamps = s.stamps;
  void *params[] = {&args};
  ++g_launches;
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_collide_spec, g_spec_blocks,
                                              SPEC_THREADS, params, 0, st);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace d3
