// collide_spec.cu — exact forceCollide in parallel, bit-identical to the
// ordered node loop of collide.zig:47-100 (d3's collide.js).
//
// In the reference, node i's turn reads its own velocity and the velocity of
// every leaf head j > i it examines, and writes velocities only where it finds
// an overlap; later turns read what earlier turns wrote. Two turns commute
// unless one writes something the other reads or writes. The kernel runs the
// turns as a dependency DAG, in one cooperative launch:
//
//  G. Guess, per node, from the pass-start state and a per-node margin
//     delta_i (larger for nodes the previous pass pushed hard): the heads it may
//     examine (R) and those it may overlap (W, a mask over R), the heads the
//     exact traversal from the start examines (E), and the cells the margin
//     traversal entered, in preorder. Traversals start at the smallest ancestor
//     of the node's leaf whose box holds the whole search box: every cell
//     outside that subtree is pruned anyway. A node with W empty is inactive.
//  E. Rounds over the active nodes, one warp per node: a node runs when no
//     earlier unfinished active node writes what it reads or accesses what it
//     writes (per-node "earliest accessor / writer" marks, 64-bit atomicMin
//     tagged with the round so no reset is needed). A running node evaluates
//     its examined heads in parallel (from E if nothing moved it, else by
//     replaying its recorded cells with the exact pruning test), adds its own
//     pushes in visit order, and writes only if everything it examined or
//     overlapped was guessed.
//  V. Inactive nodes are re-run at their exact turn state (their own velocity
//     is final: every push on a node comes from an earlier node) and must
//     still find no overlap.
//  Any failure promotes the failing nodes (every guessed head may be written,
//  with a wider margin), restores the pass-start velocities and runs E and V
//  again; after 3 attempts, or when a turn would draw from `random` (a zero
//  delta), block 0 runs the serial loop itself on the restored state.
#include <cooperative_groups.h>
#include <cstdlib>

#include "forces.cuh"

namespace cg = cooperative_groups;

namespace d3 {

constexpr int SPEC_CAP = 64;        // guessed heads per node (R)
constexpr int VISIT_CAP = 128;      // recorded margin-entered cells per node (4 per lane)
constexpr uint16_t VISIT_NONE = 0xffff;
constexpr uint32_t LEAF_TAG = 0x80000000u;  // vaux: the recorded cell is a leaf
constexpr int SPEC_ATTEMPTS = 3;
constexpr uint32_t SPEC_MAX_ROUNDS = 4096;
constexpr unsigned SPEC_THREADS = 256;
constexpr unsigned SPEC_WARPS = SPEC_THREADS / 32;

enum : uint32_t {
  C_ACTIVE = 0, C_DONE, C_FAIL, C_JIGGLE, C_OVERFLOW, C_ROUNDS, C_ATTEMPTS, C_SERIAL,
  C_FAIL_READ, C_FAIL_WRITE, C_FAIL_MOVED, C_FAST_TURNS, C_SLOW_TURNS, C_PEND0, C_PEND1, C_PEND2
};

struct SpecArgs {
  const Cell *cells;
  const uint32_t *skip, *perm, *info, *parent, *leaf_of;
  const double *xs, *ys, *px, *py, *radii;
  double *vxs, *vys, *svx, *svy;
  double strength, delta0;
  int force_traverse;    // every moved or unmoved turn takes the exact warp traversal (tests)
  uint32_t n;
  uint32_t *rlist;       // n * SPEC_CAP
  uint8_t *rcount;       // n
  uint64_t *wmask;       // n
  uint64_t *emask;       // n: heads the exact traversal from the pass start visits
  uint32_t *vlist;       // n * VISIT_CAP: cells the margin traversal entered, preorder
  uint32_t *vaux;        // n * VISIT_CAP: per recorded cell, a leaf's head | LEAF_TAG, else its skip
  uint16_t *vcount;      // n (VISIT_NONE: not recorded)
  uint32_t *start;       // n: subtree root the traversals start from
  double *mdelta;        // n: the node's margin
  uint8_t *state;        // n: 0 inactive, 1 pending, 2 done, 3 / 4 failed (active / inactive)
  uint32_t *active;      // active node list
  uint32_t *pend[2];     // nodes still pending, compacted each round (alternating)
  uint64_t *min_acc, *min_wr;  // tagged marks per node, two rounds' worth (round parity)
  double *push;          // push magnitude received per node (this pass)
  double *push_prev;     // ... in the previous pass (margin heuristic)
  uint32_t *min_pusher, *max_pusher;
  uint32_t *counters;    // C_*
  unsigned long long *stamps;  // phase timestamps (ns)
  Rng *rng;
};

// Mutable data is read through L2 (ld.global.cg): other SMs write it between
// the grid-wide barriers and L1 is not coherent across SMs.
__device__ inline double rd(const double *p) { return __ldcg(p); }
__device__ inline uint32_t rd(const uint32_t *p) { return __ldcg(p); }
__device__ inline uint64_t rd(const uint64_t *p) { return __ldcg((const unsigned long long *)p); }
__device__ inline uint8_t rd(const uint8_t *p) { return (uint8_t)__ldcg((const unsigned char *)p); }
__device__ inline uint16_t rd(const uint16_t *p) { return (uint16_t)__ldcg((const unsigned short *)p); }

__device__ inline bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}

__device__ inline bool pruned(const Cell &q, double xi, double yi, double r) {
  return q.x0 > xi + r || q.x1 < xi - r || q.y0 > yi + r || q.y1 < yi - r;
}

// The margin of node j: the base margin plus three times what the previous
// pass pushed it, bounded.
__device__ inline double margin_of(const SpecArgs &a, uint32_t j) {
  const double d = a.delta0 + 3 * a.push_prev[j];
  const double cap = 2 * a.delta0;
  return d < cap ? d : cap;
}

__device__ bool spec_guess(const SpecArgs &a, uint32_t i, double margin, bool all_writes);

// A guess that overflows the lists is retried with half the margin, down to
// the base margin (a smaller margin guesses fewer heads).
__device__ bool spec_guess_fit(const SpecArgs &a, uint32_t i, double margin, bool all_writes) {
  for (;;) {
    if (spec_guess(a, i, margin, all_writes)) return true;
    if (!(margin > a.delta0)) return false;
    margin = margin * 0.5 > a.delta0 ? margin * 0.5 : a.delta0;
  }
}

// The smallest ancestor of i's leaf whose box strictly contains the search
// box of half-width R around (xi, yi), slack included; the root otherwise.
// (With a negative radius an enclosing box no longer implies "not pruned":
// those traversals start at the root.)
__device__ uint32_t start_cell(const SpecArgs &a, uint32_t i, double xi, double yi, double R) {
  uint32_t c = a.leaf_of[i];
  if (c == NONE || !(R > 0) || !(a.radii[i] >= 0)) return 0;
  const double slack = (fabs(xi) + fabs(yi) + R) * 0x1p-40 + 1e-300;
  const double h = R + slack;
  while (c != 0 && c != NONE) {
    const Cell &q = a.cells[c];
    if (q.x0 < xi - h && q.x1 > xi + h && q.y0 < yi - h && q.y1 > yi + h) break;
    c = a.parent[c];
  }
  return c == NONE ? 0 : c;
}

// G for node i with margin `margin` (all_writes: every guessed head may be
// written).
__device__ bool spec_guess(const SpecArgs &a, uint32_t i, double margin, bool all_writes) {
  const uint32_t len = a.info[1];
  const double xi = a.px[i], yi = a.py[i], ri = a.radii[i];
  uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  uint32_t *vl = a.vlist + (size_t)i * VISIT_CAP;
  uint32_t *va = a.vaux + (size_t)i * VISIT_CAP;
  a.rcount[i] = 0;
  a.wmask[i] = 0;
  a.emask[i] = 0;
  a.vcount[i] = 0;
  a.mdelta[i] = margin;
  if (len == 0 || xi != xi || yi != yi) {  // a NaN node never overlaps: a no-op turn
    a.start[i] = 0;
    return true;
  }
  const double rmax = a.cells[0].r;
  const uint32_t c0 = start_cell(a, i, xi, yi, ri + rmax + margin);
  const uint32_t c1 = c0 == 0 ? len : a.skip[c0];
  a.start[i] = c0;
  uint32_t nr = 0, ex_until = 0, nv = 0;
  uint64_t wm = 0, em = 0;
  for (uint32_t c = c0; c < c1;) {
    const Cell &q = a.cells[c];
    const double r = ri + q.r;
    const bool ex_vis = c >= ex_until;
    if (is_leaf(q)) {
      const uint32_t j = a.perm[q.first + q.count - 1];
      if (nv < VISIT_CAP) {
        vl[nv] = c;
        va[nv] = j | LEAF_TAG;
      }
      ++nv;
      if (j > i) {
        if (nr == SPEC_CAP) return false;
        const double dx = xi - a.px[j], dy = yi - a.py[j];
        const double rr = r + margin + margin_of(a, j);
        if (all_writes || dx * dx + dy * dy < rr * rr) wm |= 1ull << nr;
        if (ex_vis) em |= 1ull << nr;
        rl[nr++] = j;
      }
      c = c + 1;
      continue;
    }
    if (pruned(q, xi, yi, r + margin)) {
      c = a.skip[c];
      continue;
    }
    if (ex_vis && pruned(q, xi, yi, r)) ex_until = a.skip[c];
    if (nv < VISIT_CAP) {
      vl[nv] = c;
      va[nv] = a.skip[c];
    }
    ++nv;
    c = c + 1;
  }
  a.rcount[i] = (uint8_t)nr;
  a.wmask[i] = wm;
  a.emask[i] = em;
  a.vcount[i] = nv <= VISIT_CAP ? (uint16_t)nv : VISIT_NONE;
  return true;
}

// Which guessed heads node i examines from (xi, yi), once i has moved: a mask
// over R. The recorded cells (vc, va: entries 4 lane .. 4 lane + 3, loaded by
// the caller) are replayed by the warp in parallel: a recorded cell is skipped
// when it lies in the subtree of an earlier recorded cell the exact test
// prunes (a running maximum of those subtrees' ends). Only the internal
// cells' boxes are loaded here. Returns false when the record does not apply
// (i moved beyond its margin, or no record): lane-uniform.
__device__ bool warp_replay(const SpecArgs &a, uint32_t i, double xi, double yi, uint16_t nv,
                            double md, double pxi, double pyi, const uint32_t *vc,
                            const uint32_t *va, uint64_t &mask) {
  const unsigned lane = threadIdx.x & 31;
  md *= (1 - 1e-9);
  if (nv == VISIT_NONE || !(fabs(xi - pxi) < md && fabs(yi - pyi) < md)) return false;
  const double ri = a.radii[i];
  uint32_t cell[4], upto[4];
  bool head[4];
  uint32_t run = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const uint32_t t = 4 * lane + u;
    cell[u] = NONE;
    head[u] = false;
    upto[u] = 0;
    if (t < nv) {
      const uint32_t c = vc[u], x = va[u];
      cell[u] = c;
      if (x & LEAF_TAG) {
        head[u] = (x & ~LEAF_TAG) > i;
      } else {
        const Cell &q = a.cells[c];
        if (pruned(q, xi, yi, ri + q.r)) upto[u] = x;
      }
    }
    run = max(run, upto[u]);
  }
  // exclusive max over earlier lanes' entries
  uint32_t incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yv = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl = max(incl, yv);
  }
  uint32_t before = __shfl_up_sync(0xffffffffu, incl, 1);
  if (lane == 0) before = 0;
  // heads' indices in R: exclusive count of heads before
  uint32_t nh = 0;
  for (int u = 0; u < 4; ++u) nh += head[u];
  uint32_t hincl = nh;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yv = __shfl_up_sync(0xffffffffu, hincl, o);
    if (lane >= (unsigned)o) hincl += yv;
  }
  uint32_t k = hincl - nh;
  uint64_t m = 0;
  uint32_t ex = before;
  for (int u = 0; u < 4; ++u) {
    if (cell[u] == NONE) continue;
    const bool vis = cell[u] >= ex;
    if (head[u]) {
      if (vis && k < 64) m |= 1ull << k;
      ++k;
    }
    ex = max(ex, upto[u]);
  }
  for (int o = 16; o > 0; o >>= 1) m |= __shfl_xor_sync(0xffffffffu, m, o);
  mask = m;
  return true;
}

// V: an inactive node's turn re-run at its exact turn state. Its own velocity
// is final; a head's is its start value if all its pushers come later, its
// final value if all came earlier, and otherwise only bounded (then a distance
// margin must hold). Returns false when the turn could write.
__device__ bool spec_inactive_ok(const SpecArgs &a, uint32_t i) {
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const double vi = rd(&a.vxs[i]), wi = rd(&a.vys[i]);
  const bool unmoved = same_bits(vi, rd(&a.svx[i])) && same_bits(wi, rd(&a.svy[i]));
  bool any = !unmoved;
  for (uint32_t k = 0; k < nr && !any; ++k) any = rd(&a.min_pusher[rd(&rl[k])]) != NONE;
  if (!any) return true;  // nothing it reads moved: the guess holds as computed
  const double ri = a.radii[i];
  const double xi = a.xs[i] + vi, yi = a.ys[i] + wi;
  if (xi != xi || yi != yi) return true;
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
      const double dx = xi - a.xs[j] - rd(&a.svx[j]), dy = yi - a.ys[j] - rd(&a.svy[j]);
      const double gap = sqrt(dx * dx + dy * dy) - r - rd(&a.push[j]);
      return gap > 1e-9 * (r + 1);
    }
    const double x = xi - a.xs[j] - vj, y = yi - a.ys[j] - wj;
    return !(x * x + y * y < r * r);
  };
  // replay the recorded cells (valid while i stays within its margin)
  const uint16_t nv = rd(&a.vcount[i]);
  const double md = rd(&a.mdelta[i]) * (1 - 1e-9);
  if (nv != VISIT_NONE && fabs(xi - a.px[i]) < md && fabs(yi - a.py[i]) < md) {
    const uint32_t *vl = a.vlist + (size_t)i * VISIT_CAP;
    const uint32_t *va = a.vaux + (size_t)i * VISIT_CAP;
    uint32_t ex_until = 0;
    for (uint32_t t = 0; t < nv; ++t) {
      const uint32_t c = rd(&vl[t]), x = rd(&va[t]);
      const Cell &q = a.cells[c];
      if (x & LEAF_TAG) {
        const uint32_t j = x & ~LEAF_TAG;
        if (j > i && c >= ex_until && !clear(j, q.r)) return false;
        continue;
      }
      if (c >= ex_until && pruned(q, xi, yi, ri + q.r)) ex_until = x;
    }
    return true;
  }
  const uint32_t len = a.info[1];
  for (uint32_t c = 0; c < len;) {
    const Cell &q = a.cells[c];
    const double r = ri + q.r;
    if (is_leaf(q)) {
      const uint32_t j = a.perm[q.first + q.count - 1];
      if (j > i) {
        bool found = false;
        for (uint32_t k = 0; k < nr && !found; ++k) found = rd(&rl[k]) == j;
        if (!found || !clear(j, q.r)) return false;
      }
      c = c + 1;
      continue;
    }
    c = pruned(q, xi, yi, r) ? a.skip[c] : c + 1;
  }
  return true;
}

__device__ void warp_mark(const SpecArgs &a, uint32_t i, uint64_t tag, uint32_t par) {
  const unsigned lane = threadIdx.x & 31;
  uint64_t *min_acc = a.min_acc + (size_t)par * a.n, *min_wr = a.min_wr + (size_t)par * a.n;
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  const unsigned long long t = (tag << 32) | i;
  if (lane == 0) {
    atomicMin((unsigned long long *)&min_acc[i], t);
    atomicMin((unsigned long long *)&min_wr[i], t);
  }
  for (uint32_t k = lane; k < nr; k += 32) {
    const uint32_t j = rd(&rl[k]);
    atomicMin((unsigned long long *)&min_acc[j], t);
    if ((wm >> k) & 1) atomicMin((unsigned long long *)&min_wr[j], t);
  }
}

// The exact traversal of node i from (xi, yi), by the warp: windows of 32
// consecutive cells in preorder; a cell is visited when no earlier cell the
// exact test prunes covers it (a running maximum of the pruned cells' skip
// links), and the next window starts past both the window and that maximum.
// Every leaf head j > i it examines must be among the guessed heads (lane k
// holds heads k and k + 32 in jj[]); mask gets their indices in R. Returns
// false if one is missing (lane-uniform).
__device__ bool warp_traverse(const SpecArgs &a, uint32_t i, double xi, double yi, double ri,
                              const uint32_t *jj, uint64_t &mask) {
  const unsigned lane = threadIdx.x & 31;
  // from the smallest ancestor of i's leaf that holds the whole search box:
  // every cell outside its subtree is pruned anyway
  uint32_t start = 0;
  if (lane == 0) start = start_cell(a, i, xi, yi, ri + a.cells[0].r);
  start = __shfl_sync(0xffffffffu, start, 0);
  const uint32_t len = start == 0 ? a.info[1] : a.skip[start];
  uint32_t carry = 0;  // cells below this index lie in pruned subtrees
  uint64_t m = 0;
  bool missing = false;
  for (uint32_t c0 = start; c0 < len;) {
    const uint32_t c = c0 + lane;
    uint32_t up = 0, head = NONE;
    bool leaf = false;
    if (c < len) {
      const Cell &q = a.cells[c];
      leaf = is_leaf(q);
      if (leaf) head = a.perm[q.first + q.count - 1];
      else if (pruned(q, xi, yi, ri + q.r)) up = a.skip[c];
    }
    uint32_t incl = up;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (unsigned)o) incl = max(incl, y);
    }
    uint32_t before = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) before = 0;
    const bool vis = c < len && c >= max(carry, before);
    const bool want = vis && leaf && head > i;
    // the examined heads' indices in R
    int k = -1;
    if (__any_sync(0xffffffffu, want)) {
      for (int t = 0; t < 32; ++t) {
        const uint32_t r0 = __shfl_sync(0xffffffffu, jj[0], t), r1 = __shfl_sync(0xffffffffu, jj[1], t);
        if (want && r0 == head) k = t;
        if (want && r1 == head) k = t + 32;
      }
    }
    if (want) {
      if (k < 0) missing = true;
      else m |= 1ull << k;
    }
    carry = max(carry, __shfl_sync(0xffffffffu, incl, 31));
    c0 = max(c0 + 32, carry);
  }
  for (int o = 16; o > 0; o >>= 1) m |= __shfl_xor_sync(0xffffffffu, m, o);
  mask = m;
  return !__any_sync(0xffffffffu, missing);
}

// One pending node's step in a round, by one warp, with its loads issued
// together: first the node's own data and its guessed heads (lane k holds
// heads k and k + 32), then the heads' marks together with their positions
// and velocities. If an earlier pending node conflicts, the node marks its
// accesses for the next round and joins the next list; otherwise it runs its
// turn (the head data loaded before the decision is what the turn would read:
// once the node is ready no other node of the round writes those heads).
// Returns nothing; state, velocities and counters are updated in place.
__device__ void warp_step(const SpecArgs &a, uint32_t i, uint64_t tag, uint32_t par,
                          uint32_t *next, uint32_t *next_n, double *cx, double *cy) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  // round trip 1
  const uint8_t state = rd(&a.state[i]);
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  const uint64_t em = rd(&a.emask[i]);
  const double vi = rd(&a.vxs[i]), wi = rd(&a.vys[i]);
  const double svi = rd(&a.svx[i]), swi = rd(&a.svy[i]);
  const uint32_t j0 = lane < nr ? rd(&rl[lane]) : NONE;
  const uint32_t j1 = lane + 32 < nr ? rd(&rl[lane + 32]) : NONE;
  if (state != 1) return;
  // round trip 2: marks, the heads' data for the turn, and (if i moved) its
  // record of the cells the guess entered
  const bool unmoved = same_bits(vi, svi) && same_bits(wi, swi);
  uint32_t vc[4], va[4];
  uint16_t nv = VISIT_NONE;
  double md = 0, pxi = 0, pyi = 0;
  if (!unmoved) {
    const uint32_t *vl = a.vlist + (size_t)i * VISIT_CAP, *vx = a.vaux + (size_t)i * VISIT_CAP;
    nv = rd(&a.vcount[i]);
    md = rd(&a.mdelta[i]);
    pxi = a.px[i];
    pyi = a.py[i];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      vc[u] = rd(&vl[4 * lane + u]);
      va[u] = rd(&vx[4 * lane + u]);
    }
  }
  const uint64_t *min_acc = a.min_acc + (size_t)par * a.n, *min_wr = a.min_wr + (size_t)par * a.n;
  bool ok = true;
  if (lane == 0) {  // self: read and written
    const uint64_t v = rd(&min_acc[i]);
    ok = !((v >> 32) == tag && (uint32_t)v < i);
  }
  // per head: the offset (x, y) = (xi - xs[j] - vxs[j], ...) of the turn,
  // formed as the turn forms it, and the head's radius
  const double xi = a.xs[i] + vi, yi = a.ys[i] + wi;
  double hx[2], hy[2], hr[2];
  const uint32_t jj[2] = {j0, j1};
  for (int h = 0; h < 2; ++h) {
    const uint32_t k = lane + 32 * h, j = jj[h];
    hx[h] = hy[h] = hr[h] = 0;
    if (j == NONE) continue;
    const uint64_t v = ((wm >> k) & 1) ? rd(&min_acc[j]) : rd(&min_wr[j]);
    if ((v >> 32) == tag && (uint32_t)v < i) ok = false;
    hx[h] = xi - a.xs[j] - rd(&a.vxs[j]);
    hy[h] = yi - a.ys[j] - rd(&a.vys[j]);
    hr[h] = a.radii[j];
  }
  if (!__all_sync(0xffffffffu, ok)) {
    // mark for the next round (the other parity's marks) and stay pending
    uint64_t *nacc = a.min_acc + (size_t)(par ^ 1u) * a.n, *nwr = a.min_wr + (size_t)(par ^ 1u) * a.n;
    const unsigned long long t = ((tag - 1) << 32) | i;
    if (lane == 0) {
      atomicMin((unsigned long long *)&nacc[i], t);
      atomicMin((unsigned long long *)&nwr[i], t);
      next[atomicAdd(next_n, 1u)] = i;
    }
    for (int h = 0; h < 2; ++h) {
      const uint32_t k = lane + 32 * h, j = jj[h];
      if (j == NONE) continue;
      atomicMin((unsigned long long *)&nacc[j], t);
      if ((wm >> k) & 1) atomicMin((unsigned long long *)&nwr[j], t);
    }
    return;
  }
  if (lane == 0) a.state[i] = 2;  // done (3 = failed, set below)
  const double ri = a.radii[i], ri2 = ri * ri;
  uint64_t ex = 0;
  if (unmoved && !a.force_traverse) {
    ex = em;
  } else if (a.force_traverse || !warp_replay(a, i, xi, yi, nv, md, pxi, pyi, vc, va, ex)) {
    // i moved beyond its margin: the warp runs the exact traversal; every head
    // it examines must still be among the guessed ones.
    if (!warp_traverse(a, i, xi, yi, ri, jj, ex)) {
      if (lane == 0) {
        atomicAdd(&a.counters[C_FAIL], 1u);
        atomicAdd(&a.counters[C_FAIL_READ], 1u);
        a.state[i] = 3;
        atomicAdd(&a.counters[C_DONE], 1u);
      }
      return;
    }
  }
  // each lane evaluates the examined heads with indices lane and lane + 32
  bool fail = false, jig = false;
  uint64_t over = 0;
  uint32_t pj[2];
  double pdx[2], pdy[2];
  int np = 0;
  for (int h = 0; h < 2; ++h) {
    const uint32_t e = lane + 32 * h;
    if (e >= nr || !((ex >> e) & 1)) continue;
    const uint32_t j = jj[h];
    double rj = hr[h];
    double r = ri + rj;
    double x = hx[h];
    double y = hy[h];
    double l = x * x + y * y;
    if (!(l < r * r)) continue;
    if (!((wm >> e) & 1)) {
      fail = true;
      continue;
    }
    if (x == 0 || y == 0) {
      jig = true;
      continue;
    }
    l = sqrt(l);
    l = (r - l) / l * a.strength;
    x *= l;
    y *= l;
    rj *= rj;
    r = rj / (ri2 + rj);
    cx[e] = x * r;
    cy[e] = y * r;
    over |= 1ull << e;
    r = 1 - r;
    pj[np] = j;
    pdx[np] = x * r;
    pdy[np] = y * r;
    ++np;
  }
  fail = __any_sync(0xffffffffu, fail);
  jig = __any_sync(0xffffffffu, jig);
  for (int o = 16; o > 0; o >>= 1) over |= __shfl_xor_sync(0xffffffffu, over, o);
  __syncwarp();
  if (fail || jig) {
    if (lane == 0) {
      if (jig) atomicAdd(&a.counters[C_JIGGLE], 1u);
      if (fail) {
        atomicAdd(&a.counters[C_FAIL], 1u);
        atomicAdd(&a.counters[C_FAIL_WRITE], 1u);
        a.state[i] = 3;
      }
      atomicAdd(&a.counters[C_DONE], 1u);
    }
    return;
  }
  if (lane == 0) {
    // d3 adds its own share head by head, in visit order (R order)
    double v = vi, w = wi;
    uint64_t o = over;
    while (o) {
      const int e = __ffsll((long long)o) - 1;
      o &= o - 1;
      v += cx[e];
      w += cy[e];
    }
    a.vxs[i] = v;
    a.vys[i] = w;
    atomicAdd(&a.counters[unmoved ? C_FAST_TURNS : C_SLOW_TURNS], 1u);
    atomicAdd(&a.counters[C_DONE], 1u);
  }
  for (int h = 0; h < np; ++h) {
    const uint32_t j = pj[h];
    a.vxs[j] = rd(&a.vxs[j]) - pdx[h];
    a.vys[j] = rd(&a.vys[j]) - pdy[h];
    atomicAdd(&a.push[j], sqrt(pdx[h] * pdx[h] + pdy[h] * pdy[h]));
    atomicMin(&a.min_pusher[j], i);
    atomicMax(&a.max_pusher[j], i);
  }
  __syncwarp();
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
      c = pruned(q, xi, yi, r) ? a.skip[c] : c + 1;
    }
  }
  a.rng->lcg = s;
}

__device__ inline unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void __launch_bounds__(SPEC_THREADS, 3) k_collide_spec(SpecArgs a) {
  __shared__ double contrib[SPEC_WARPS][2][SPEC_CAP];
  cg::grid_group g = cg::this_grid();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t gw = tid >> 5, nwarps = nth >> 5, wl = threadIdx.x >> 5;
  const uint32_t n = a.n;
  if (tid < 16) a.counters[tid] = 0;
  if (tid == 0) {
    for (int k = 0; k < 144; ++k) a.stamps[k] = 0;
    a.stamps[0] = now_ns();
  }
  g.sync();
  // G, plus per-node resets and the pass-start snapshot.
  for (uint32_t i = tid; i < n; i += nth) {
    a.svx[i] = a.vxs[i];
    a.svy[i] = a.vys[i];
    a.min_acc[i] = a.min_acc[n + i] = ~0ull;
    a.min_wr[i] = a.min_wr[n + i] = ~0ull;
    a.push[i] = 0;
    a.min_pusher[i] = NONE;
    a.max_pusher[i] = 0;
    if (!spec_guess_fit(a, i, margin_of(a, i), false)) {
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
    if (rd(&a.counters[C_OVERFLOW]) || rd(&a.counters[C_JIGGLE])) break;
    const uint32_t n_active = rd(&a.counters[C_ACTIVE]);
    // round 0 works on the active list; later rounds on the nodes the
    // previous round left pending (their sizes rotate through C_PEND0..2)
    const uint32_t *list = a.active;
    uint32_t n_list = n_active;
    // The first round's marks; afterwards a node that is not ready marks for
    // the next round at once (the other parity's marks), so each round needs
    // one grid-wide barrier.
    {
      const uint64_t tag0 = 0xFFFFFFFFull - round_base;
      for (uint32_t k = gw; k < n_list; k += nwarps) {
        const uint32_t i = rd(&list[k]);
        if (rd(&a.state[i]) == 1) warp_mark(a, i, tag0, round_base & 1);
      }
      if (tid == 0) a.counters[C_PEND0] = a.counters[C_PEND1] = a.counters[C_PEND2] = 0;
      g.sync();
    }
    for (uint32_t round = 0;; ++round) {
      const uint32_t r = round_base + round;
      if (r + 1 >= SPEC_MAX_ROUNDS) {
        if (tid == 0) atomicAdd(&a.counters[C_OVERFLOW], 1u);
        break;
      }
      const uint64_t tag = 0xFFFFFFFFull - r;
      uint32_t *next = a.pend[round & 1];
      uint32_t *next_n = &a.counters[C_PEND0 + round % 3];
      if (tid == 0 && attempt == 0 && round < 64) a.stamps[80 + round] = n_list;
      for (uint32_t k = gw; k < n_list; k += nwarps)
        warp_step(a, rd(&list[k]), tag, r & 1, next, next_n, contrib[wl][0], contrib[wl][1]);
      g.sync();
      if (tid == 0 && attempt == 0 && round < 64) a.stamps[16 + round] = now_ns();
      // Every thread reads the same count: it changes again only after the
      // next barrier. (C_DONE cannot decide this: the next round's turns may
      // already be adding to it.)
      n_list = rd(next_n);
      if (n_list == 0) {
        round_base += round + 1;
        break;
      }
      list = next;
      // the counter of round + 2 was last read before this round's barrier
      if (tid == 0) a.counters[C_PEND0 + (round + 2) % 3] = 0;
    }
    if (tid == 0 && attempt < 3) a.stamps[2 + 2 * attempt] = now_ns();
    // V: inactive nodes stayed no-ops (Morton order, as G).
    for (uint32_t k = tid; k < n; k += nth) {
      const uint32_t i = a.perm[k];
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
    if (rd(&a.counters[C_FAIL]) == 0 && rd(&a.counters[C_DONE]) >= n_active &&
        rd(&a.counters[C_JIGGLE]) == 0) {
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
        // every head within a four times wider margin may be written
        if (!spec_guess_fit(a, i, 4 * rd(&a.mdelta[i]), true)) atomicAdd(&a.counters[C_OVERFLOW], 1u);
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
    for (uint32_t i = tid; i < n; i += nth) a.push_prev[i] = a.push[i];
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
  cudaFree(s.start); cudaFree(s.mdelta); cudaFree(s.push_prev); cudaFree(s.pend); cudaFree(s.vaux);
  if (!s.counters) {
    D3_CUDA_OK(cudaMalloc(&s.counters, 16 * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(s.counters, 0, 16 * sizeof(uint32_t)));
  }
  // 16 phase stamps, then attempt 1's per-round end times and list sizes (64 each)
  if (!s.stamps) D3_CUDA_OK(cudaMalloc(&s.stamps, 144 * sizeof(unsigned long long)));
  D3_CUDA_OK(cudaMalloc(&s.rlist, (size_t)cap * SPEC_CAP * 4));
  D3_CUDA_OK(cudaMalloc(&s.rcount, cap));
  D3_CUDA_OK(cudaMalloc(&s.wmask, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.state, cap));
  D3_CUDA_OK(cudaMalloc(&s.active, 2ull * cap * 4));
  D3_CUDA_OK(cudaMalloc(&s.min_acc, 2 * cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.min_wr, 2 * cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.push, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.min_pusher, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.emask, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.max_pusher, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.vlist, (size_t)cap * VISIT_CAP * 4));
  D3_CUDA_OK(cudaMalloc(&s.vaux, (size_t)cap * VISIT_CAP * 4));
  D3_CUDA_OK(cudaMalloc(&s.vcount, cap * 2ull));
  D3_CUDA_OK(cudaMalloc(&s.start, cap * 4ull));
  D3_CUDA_OK(cudaMalloc(&s.mdelta, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.push_prev, cap * 8ull));
  D3_CUDA_OK(cudaMemset(s.push_prev, 0, cap * 8ull));
  D3_CUDA_OK(cudaMalloc(&s.pend, 4ull * cap * 4));
  s.cap = cap;
  return 0;
}

void collide_spec_free(CollideSpec &s) {
  cudaFree(s.rlist); cudaFree(s.rcount); cudaFree(s.wmask); cudaFree(s.state); cudaFree(s.active);
  cudaFree(s.min_acc); cudaFree(s.min_wr); cudaFree(s.push); cudaFree(s.min_pusher);
  cudaFree(s.emask); cudaFree(s.max_pusher); cudaFree(s.vlist); cudaFree(s.vcount);
  cudaFree(s.start); cudaFree(s.mdelta); cudaFree(s.push_prev); cudaFree(s.pend); cudaFree(s.vaux);
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
    // blocks per SM: full occupancy (at most 3), or D3_COLLIDE_BLOCKS_PER_SM
    int want = per > 3 ? 3 : per;
    if (const char *e = getenv("D3_COLLIDE_BLOCKS_PER_SM")) {
      const int v = atoi(e);
      if (v >= 1 && v <= want) want = v;
    }
    g_spec_blocks = sms * (want > 0 ? want : 1);
    if (g_spec_blocks <= 0) g_spec_blocks = sms;
  }
  SpecArgs args;
  args.cells = t.cells; args.skip = t.skip; args.perm = t.perm; args.info = t.info;
  args.parent = t.parent; args.leaf_of = t.leaf_of;
  args.xs = a.x; args.ys = a.y; args.px = a.px; args.py = a.py; args.radii = radii;
  args.vxs = a.vx; args.vys = a.vy; args.svx = a.snap_vx; args.svy = a.snap_vy;
  args.strength = strength; args.delta0 = delta; args.n = a.n;
  // D3_COLLIDE_FORCE_TRAVERSE (any value): every turn finds its examined heads
  // by the exact traversal instead of the recorded ones (a test of that path)
  args.force_traverse = getenv("D3_COLLIDE_FORCE_TRAVERSE") != nullptr;
  args.rlist = s.rlist; args.rcount = s.rcount; args.wmask = s.wmask; args.emask = s.emask;
  args.vlist = s.vlist; args.vaux = s.vaux; args.vcount = s.vcount; args.start = s.start; args.mdelta = s.mdelta;
  args.state = s.state; args.active = s.active; args.min_acc = s.min_acc; args.min_wr = s.min_wr;
  args.push = s.push; args.push_prev = s.push_prev; args.min_pusher = s.min_pusher;
  args.max_pusher = s.max_pusher; args.counters = s.counters; args.stamps = s.stamps;
  args.rng = rng;
  args.pend[0] = s.pend;
  args.pend[1] = s.pend + 2ull * s.cap;
  void *params[] = {&args};
  ++g_launches;
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_collide_spec, g_spec_blocks,
                                              SPEC_THREADS, params, 0, st);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace d3
