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
//  E. The active nodes' turns in dependency order, one warp per turn. Every
//     active node accesses its guessed heads (writes those in W, reads the
//     rest) and itself (a write). Per accessed node, the accessors' list is
//     sorted by node: a write waits for every access since the previous
//     write, a read for the previous write; each access records the range of
//     the list it waits on. Waits only point to lower node indices, so warps
//     claim the active nodes in index order: a warp loads everything about
//     its node that cannot change (heads, their positions, the record, the
//     ids of the turns it waits on), waits until those turns are done, then
//     reads the velocities and runs the turn. A running node evaluates its
//     examined heads in parallel (from E if nothing moved it, else by
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
constexpr unsigned SPEC_THREADS = 256;
constexpr unsigned SPEC_WARPS = SPEC_THREADS / 32;
constexpr uint32_t SELF_ENTRY = SPEC_CAP;  // an access list entry of the node itself
// A turn's wait gives up after this long without any turn finishing.
constexpr unsigned long long SPEC_WAIT_NS = 20000000ull;
constexpr unsigned FULL = 0xffffffffu;

// counters[]: 0..13 are reported by the engine (13: waits that gave up); the
// ones every turn touches sit in cache lines of their own.
enum : uint32_t {
  C_ACTIVE = 0, C_FAIL = 2, C_JIGGLE, C_OVERFLOW, C_DEPTH, C_ATTEMPTS, C_SERIAL,
  C_FAIL_READ, C_FAIL_WRITE, C_FAIL_MOVED, C_FAST_TURNS, C_SLOW_TURNS, C_TIMEOUT,
  C_ALLOC = 16, C_BIGFILL, C_BIGLINK, C_VWORK, C_DONE = 32, C_CLAIM = 64, C_COUNTERS = 128
};
constexpr uint32_t PR_SLOTS = SPEC_CAP + 1;  // a node's entries: its heads, then itself

// A cell as the collide traversals read it, in one 64-byte load: its box and
// radius, and for an internal cell its skip link, for a leaf its head (the
// node d3 examines: the last of the leaf's points) with the head's position
// and margin.
struct alignas(64) CRec {
  double x0, y0, x1, y1;
  double r;
  uint32_t link;  // internal: skip link; leaf: head | LEAF_TAG
  float margin;   // leaf: the head's margin (a guess heuristic, rounded)
  double hx, hy;  // leaf: the head's shifted position
};
static_assert(sizeof(CRec) == 64, "record layout");

__device__ inline bool rec_leaf(const CRec &q) { return q.link & LEAF_TAG; }
// The index past c's subtree.
__device__ inline uint32_t rec_skip(const CRec &q, uint32_t c) { return rec_leaf(q) ? c + 1 : q.link; }

struct SpecArgs {
  const Cell *cells;
  CRec *rec;             // cells' records (built at the start of each pass)
  const uint32_t *skip, *perm, *info, *parent, *leaf_of;
  const double *xs, *ys, *px, *py, *radii;
  double *vxs, *vys, *svx, *svy;
  double strength, delta0;
  int force_traverse;    // every moved or unmoved turn takes the exact warp traversal (tests)
  int profile;           // record per-depth finish times and counts (stamps)
  unsigned sleep_ns;     // pause between polls of a wait (after the first four)
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
  uint32_t *cnt;         // n: accesses per node (zero between phases)
  uint32_t *rlen, *roff; // n: each node's access list: length, offset
  uint64_t *ent;         // access entries: node << 32 | index in R << 1 | write
  uint64_t *ents;        // ... each list sorted by node
  uint64_t *pr;          // n * PR_SLOTS: per entry, the sorted entries its access waits
                         // on: first << 32 | count
  uint32_t *lev;         // n: the turn's depth in the dependency order
  uint32_t *aflag, *apos, *sact;  // n each: active flags, their scan, the active in index order
  uint32_t *scan_part;   // grid partials of that scan (a word per block)
  uint32_t *bigfill, *biglink, *vwork;  // n each: the items warps share out (see below)
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

// Appends v to list (size at *count) for the lanes that want to, with one
// atomic per warp. Warp-uniform call.
__device__ inline void warp_append(bool want, uint32_t v, uint32_t *list, uint32_t *count) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(FULL, want);
  if (!m) return;
  const int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(FULL, base, leader);
  if (want) list[base + __popc(m & ((1u << lane) - 1))] = v;
}

__device__ inline bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}

template <class Q>
__device__ inline bool pruned(const Q &q, double xi, double yi, double r) {
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
    const CRec &q = a.rec[c];
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
  const double rmax = a.rec[0].r;
  const uint32_t c0 = start_cell(a, i, xi, yi, ri + rmax + margin);
  const uint32_t c1 = c0 == 0 ? len : rec_skip(a.rec[c0], c0);
  a.start[i] = c0;
  uint32_t nr = 0, ex_until = 0, nv = 0;
  uint64_t wm = 0, em = 0;
  for (uint32_t c = c0; c < c1;) {
    const CRec q = a.rec[c];
    const double r = ri + q.r;
    const bool ex_vis = c >= ex_until;
    if (rec_leaf(q)) {
      const uint32_t j = q.link & ~LEAF_TAG;
      if (nv < VISIT_CAP) {
        vl[nv] = c;
        va[nv] = q.link;
      }
      ++nv;
      if (j > i) {
        if (nr == SPEC_CAP) return false;
        const double dx = xi - q.hx, dy = yi - q.hy;
        const double rr = r + margin + (double)q.margin;
        if (all_writes || dx * dx + dy * dy < rr * rr) wm |= 1ull << nr;
        if (ex_vis) em |= 1ull << nr;
        rl[nr++] = j;
      }
      c = c + 1;
      continue;
    }
    if (pruned(q, xi, yi, r + margin)) {
      c = q.link;
      continue;
    }
    if (ex_vis && pruned(q, xi, yi, r)) ex_until = q.link;
    if (nv < VISIT_CAP) {
      vl[nv] = c;
      va[nv] = q.link;
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
// A recorded internal cell's box and radius, staged in shared memory.
struct Box {
  double x0, y0, x1, y1, r;
};

__device__ bool warp_replay(const SpecArgs &a, uint32_t i, double xi, double yi, uint16_t nv,
                            double md, double pxi, double pyi, const uint32_t *vc,
                            const uint32_t *va, const Box *boxes, uint64_t &mask) {
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
        const Box &q = boxes[t];
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
// margin must hold). head_clear: head j (radius rj) as node i at (xi, yi),
// radius ri, would meet it: true if the turn cannot overlap it.
__device__ inline bool head_clear(const SpecArgs &a, uint32_t i, double xi, double yi, double ri,
                                  uint32_t j, double rj) {
  const uint32_t lo = rd(&a.min_pusher[j]), hi = rd(&a.max_pusher[j]);
  const double sx = rd(&a.svx[j]), sy = rd(&a.svy[j]), fx = rd(&a.vxs[j]), fy = rd(&a.vys[j]);
  const double pu = rd(&a.push[j]);
  const double r = ri + rj;
  double vj, wj;
  if (lo == NONE || lo > i) {
    vj = sx;
    wj = sy;
  } else if (hi < i) {
    vj = fx;
    wj = fy;
  } else {
    const double dx = xi - a.xs[j] - sx, dy = yi - a.ys[j] - sy;
    const double gap = sqrt(dx * dx + dy * dy) - r - pu;
    return gap > 1e-9 * (r + 1);
  }
  const double x = xi - a.xs[j] - vj, y = yi - a.ys[j] - wj;
  return !(x * x + y * y < r * r);
}

enum : int { V_OK = 0, V_WRITES = 1, V_REPLAY = 2, V_TRAVERSE = 3 };

// V's first step, a lane per node: V_OK if nothing the guess read moved (or
// the node is NaN), V_REPLAY if the warp must replay its recorded cells,
// V_TRAVERSE if the record does not apply (the warp runs the traversal).
__device__ int inactive_quick(const SpecArgs &a, uint32_t i) {
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const double vi = rd(&a.vxs[i]), wi = rd(&a.vys[i]);
  const double svi = rd(&a.svx[i]), swi = rd(&a.svy[i]);
  uint32_t r8[8];
#pragma unroll
  for (int h = 0; h < 8; ++h) r8[h] = rd(&rl[h]);  // rows are whole; used up to rcount
  bool any = !(same_bits(vi, svi) && same_bits(wi, swi));
  if (!any) {
    uint32_t mp[8];
#pragma unroll
    for (int h = 0; h < 8; ++h) mp[h] = (uint32_t)h < nr ? rd(&a.min_pusher[r8[h]]) : NONE;
#pragma unroll
    for (int h = 0; h < 8; ++h) any |= mp[h] != NONE;
    for (uint32_t k = 8; k < nr && !any; ++k) any = rd(&a.min_pusher[rd(&rl[k])]) != NONE;
  }
  if (!any) return V_OK;  // nothing it reads moved: the guess holds as computed
  const double xi = a.xs[i] + vi, yi = a.ys[i] + wi;
  if (xi != xi || yi != yi) return V_OK;
  const uint16_t nv = rd(&a.vcount[i]);
  const double md = rd(&a.mdelta[i]) * (1 - 1e-9);
  if (nv != VISIT_NONE && fabs(xi - a.px[i]) < md && fabs(yi - a.py[i]) < md) return V_REPLAY;
  return V_TRAVERSE;
}

// V by the exact traversal of inactive node i, by the warp (windows of 32
// cells from the node's enclosing cell, as warp_traverse): every head j > i it
// examines must be a guessed one and clear. Returns false when the turn could
// write.
__device__ bool warp_inactive_traverse(const SpecArgs &a, uint32_t i) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  const uint32_t j0 = lane < nr ? rd(&rl[lane]) : NONE, j1 = lane + 32 < nr ? rd(&rl[lane + 32]) : NONE;
  const double xi = a.xs[i] + rd(&a.vxs[i]), yi = a.ys[i] + rd(&a.vys[i]);
  const double ri = a.radii[i];
  uint32_t start = 0;
  if (lane == 0) start = start_cell(a, i, xi, yi, ri + a.rec[0].r);
  start = __shfl_sync(FULL, start, 0);
  const uint32_t len = start == 0 ? a.info[1] : rec_skip(a.rec[start], start);
  uint32_t carry = 0;
  bool bad = false;
  for (uint32_t c0 = start; c0 < len;) {
    const uint32_t c = c0 + lane;
    uint32_t up = 0, head = NONE;
    bool leaf = false;
    if (c < len) {
      const CRec &q = a.rec[c];
      leaf = rec_leaf(q);
      if (leaf) head = q.link & ~LEAF_TAG;
      else if (pruned(q, xi, yi, ri + q.r)) up = q.link;
    }
    uint32_t incl = up;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, incl, o);
      if (lane >= (unsigned)o) incl = max(incl, y);
    }
    uint32_t before = __shfl_up_sync(FULL, incl, 1);
    if (lane == 0) before = 0;
    const bool want = c < len && c >= max(carry, before) && leaf && head > i;
    if (__any_sync(FULL, want)) {
      bool found = false;
      for (int t = 0; t < 32; ++t) {
        const uint32_t r0 = __shfl_sync(FULL, j0, t), r1 = __shfl_sync(FULL, j1, t);
        found |= want && (r0 == head || r1 == head);
      }
      if (want && (!found || !head_clear(a, i, xi, yi, ri, head, a.radii[head]))) bad = true;
    }
    carry = max(carry, __shfl_sync(FULL, incl, 31));
    c0 = max(c0 + 32, carry);
  }
  return !__any_sync(FULL, bad);
}

// V's replay of inactive node i's recorded cells, by the warp (entries 4 lane
// .. 4 lane + 3, as warp_replay): a recorded cell is skipped when it lies in
// the subtree of an earlier recorded cell the exact test prunes; every head
// j > i left must be clear. Returns false when the turn could write.
__device__ bool warp_inactive_replay(const SpecArgs &a, uint32_t i) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t *vl = a.vlist + (size_t)i * VISIT_CAP, *vx = a.vaux + (size_t)i * VISIT_CAP;
  const uint16_t nv = rd(&a.vcount[i]);
  const double xi = a.xs[i] + rd(&a.vxs[i]), yi = a.ys[i] + rd(&a.vys[i]);
  const double ri = a.radii[i];
  uint32_t cell[4], upto[4];
  bool bad[4];
  uint32_t run = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const uint32_t t = 4 * lane + u;
    cell[u] = NONE;
    upto[u] = 0;
    bad[u] = false;
    if (t < nv) {
      const uint32_t c = rd(&vl[t]), x = rd(&vx[t]);
      cell[u] = c;
      if (x & LEAF_TAG) {
        const uint32_t j = x & ~LEAF_TAG;
        if (j > i) bad[u] = !head_clear(a, i, xi, yi, ri, j, a.radii[j]);
      } else {
        const CRec &q = a.rec[c];
        if (pruned(q, xi, yi, ri + q.r)) upto[u] = x;
      }
    }
    run = max(run, upto[u]);
  }
  uint32_t incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yv = __shfl_up_sync(FULL, incl, o);
    if (lane >= (unsigned)o) incl = max(incl, yv);
  }
  uint32_t ex = __shfl_up_sync(FULL, incl, 1);
  if (lane == 0) ex = 0;
  bool fail = false;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    if (cell[u] == NONE) continue;
    if (bad[u] && cell[u] >= ex) fail = true;
    ex = max(ex, upto[u]);
  }
  return !__any_sync(FULL, fail);
}

// V for the nodes at Morton positions base .. base + 31, a lane each; the
// nodes whose record must be replayed or traversed go to a list that whole
// warps share out (item: node | 1 << 31 for a traversal).
__device__ inline void promote_inactive(const SpecArgs &a, uint32_t i) {
  a.state[i] = 4;  // inactive, but its turn would write
  atomicAdd(&a.counters[C_FAIL], 1u);
  atomicAdd(&a.counters[C_FAIL_MOVED], 1u);
}

__device__ void warp_check_inactive(const SpecArgs &a, uint32_t base) {
  const uint32_t k = base + (threadIdx.x & 31);
  uint32_t i = NONE;
  int res = V_OK;
  if (k < a.n) {
    i = a.perm[k];
    if (rd(&a.state[i]) == 0) res = inactive_quick(a, i);
  }
  if (res == V_WRITES) promote_inactive(a, i);
  const bool more = res == V_REPLAY || res == V_TRAVERSE;
  warp_append(more, i | (res == V_TRAVERSE ? 0x80000000u : 0u), a.vwork, &a.counters[C_VWORK]);
}

__device__ void warp_check_inactive_item(const SpecArgs &a, uint32_t item) {
  const uint32_t i = item & 0x7fffffffu;
  const bool ok = item >> 31 ? warp_inactive_traverse(a, i) : warp_inactive_replay(a, i);
  if (!ok && (threadIdx.x & 31) == 0) promote_inactive(a, i);
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
  if (lane == 0) start = start_cell(a, i, xi, yi, ri + a.rec[0].r);
  start = __shfl_sync(0xffffffffu, start, 0);
  const uint32_t len = start == 0 ? a.info[1] : rec_skip(a.rec[start], start);
  uint32_t carry = 0;  // cells below this index lie in pruned subtrees
  uint64_t m = 0;
  bool missing = false;
  for (uint32_t c0 = start; c0 < len;) {
    const uint32_t c = c0 + lane;
    uint32_t up = 0, head = NONE;
    bool leaf = false;
    if (c < len) {
      const CRec &q = a.rec[c];
      leaf = rec_leaf(q);
      if (leaf) head = q.link & ~LEAF_TAG;
      else if (pruned(q, xi, yi, ri + q.r)) up = q.link;
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

__device__ inline unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ inline uint32_t ld_relaxed(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The access lists: node i's entries (its guessed heads, then itself).
__device__ void warp_count(const SpecArgs &a, uint32_t i) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint32_t nr = rd(&a.rcount[i]);
  for (uint32_t h = lane; h < nr; h += 32) atomicAdd(&a.cnt[rd(&rl[h])], 1u);
  if (lane == 0) atomicAdd(&a.cnt[i], 1u);
}

// Each list's place: a warp takes 32 nodes' counts and one block of entries.
__device__ void warp_offsets(const SpecArgs &a, uint32_t base) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t j = base + lane;
  const uint32_t c = j < a.n ? rd(&a.cnt[j]) : 0;
  uint32_t incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  uint32_t b = 0;
  if (lane == 31 && incl) b = atomicAdd(&a.counters[C_ALLOC], incl);
  b = __shfl_sync(FULL, b, 31);
  if (j < a.n) {
    a.rlen[j] = c;
    a.roff[j] = b + incl - c;
  }
  warp_append(c > 4, j, a.biglink, &a.counters[C_BIGLINK]);
}

// Active nodes base .. base + 31 with more than four heads go to the list
// of nodes whose entries a whole warp writes.
__device__ void warp_find_bigfill(const SpecArgs &a, uint32_t base, uint32_t n_active) {
  const uint32_t k = base + (threadIdx.x & 31);
  uint32_t i = NONE, nr = 0;
  if (k < n_active) {
    i = rd(&a.active[k]);
    nr = rd(&a.rcount[i]);
  }
  warp_append(nr > 4, i, a.bigfill, &a.counters[C_BIGFILL]);
}

// Node i's entry for head h (or itself) into the list of node j.
__device__ inline void put_entry(const SpecArgs &a, uint32_t j, uint32_t i, uint32_t h, uint32_t w) {
  const uint32_t slot = rd(&a.roff[j]) + atomicSub(&a.cnt[j], 1u) - 1;
  a.ent[slot] = ((uint64_t)i << 32) | (h << 1) | w;
}

// Active nodes base .. base + 31 write their entries into the lists (cnt
// returns to zero): a lane each (the head entries of nodes with more than
// four heads are written by warp_fill_big).
__device__ void warp_fill(const SpecArgs &a, uint32_t base, uint32_t n_active) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t k = base + lane;
  uint32_t i = NONE, nr = 0;
  uint64_t wm = 0;
  if (k < n_active) {
    i = rd(&a.active[k]);
    const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
    // the node, its first four heads (read whole; used up to rcount), then
    // their places, all issued together
    nr = rd(&a.rcount[i]);
    wm = rd(&a.wmask[i]);
    uint32_t j[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) j[h] = rd(&rl[h]);
    const uint32_t nf = nr <= 4 ? nr : 0;
    uint32_t off[5], old[5];
    off[4] = rd(&a.roff[i]);
    old[4] = atomicSub(&a.cnt[i], 1u);
#pragma unroll
    for (int h = 0; h < 4; ++h)
      if ((uint32_t)h < nf) {
        off[h] = rd(&a.roff[j[h]]);
        old[h] = atomicSub(&a.cnt[j[h]], 1u);
      }
    a.ent[off[4] + old[4] - 1] = ((uint64_t)i << 32) | (SELF_ENTRY << 1) | 1;
#pragma unroll
    for (int h = 0; h < 4; ++h)
      if ((uint32_t)h < nf)
        a.ent[off[h] + old[h] - 1] = ((uint64_t)i << 32) | (h << 1) | ((wm >> h) & 1);
    a.lev[i] = 0;
    a.sact[rd(&a.apos[i])] = i;
  }
}

// The head entries of a node with more than four heads, by the warp.
__device__ void warp_fill_big(const SpecArgs &a, uint32_t i) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  for (uint32_t h = lane; h < nr; h += 32) put_entry(a, rd(&rl[h]), i, h, (wm >> h) & 1);
}

// The range an entry at sorted position p (w: a write) waits on, given the
// last write before it (pw < 0: none) and that write's node: a write waits
// for the accesses since that write (all before it if none), a read for that
// write. A single turn to wait on is stored as its node (WAIT_NODE), else
// as first sorted entry << 32 | count.
constexpr uint64_t WAIT_NODE = 0x80000000ull;
__device__ inline uint64_t wait_range(uint32_t off, uint32_t p, int32_t pw, uint32_t pw_node,
                                      bool w) {
  if (pw < 0) return w ? ((uint64_t)off << 32) | p : 0;
  if (!w || p == (uint32_t)pw + 1) return ((uint64_t)pw_node << 32) | WAIT_NODE | 1u;
  return ((uint64_t)(off + pw) << 32) | (p - (uint32_t)pw);
}

// One list of L > 4 entries at `off`, by the warp: sorted by node (the rank of
// each entry among distinct nodes), then each entry's wait range.
__device__ void warp_link_list(const SpecArgs &a, uint32_t off, uint32_t L) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t *src = a.ent + off;
  uint64_t *dst = a.ents + off;
  for (uint32_t c0 = 0; c0 < L; c0 += 32) {
    const uint32_t p = c0 + lane;
    const uint64_t e = p < L ? rd(&src[p]) : ~0ull;
    const uint32_t me = (uint32_t)(e >> 32);
    uint32_t rank = 0;
    for (uint32_t d0 = 0; d0 < L; d0 += 32) {
      const uint32_t f =
          d0 == c0 ? me : (d0 + lane < L ? (uint32_t)(rd(&src[d0 + lane]) >> 32) : NONE);
      for (int t = 0; t < 32; ++t) rank += __shfl_sync(FULL, f, t) < me;
    }
    if (p < L) dst[rank] = e;
  }
  __syncwarp();
  int32_t prev_w = -1;  // the last write before the chunk, and its node
  uint32_t prev_node = NONE;
  for (uint32_t c0 = 0; c0 < L; c0 += 32) {
    const uint32_t p = c0 + lane;
    const uint64_t e = p < L ? rd(&dst[p]) : 0;
    const bool w = p < L && (e & 1);
    const unsigned wb = __ballot_sync(FULL, w);
    const unsigned below = wb & ((1u << lane) - 1);
    const int src = below ? 31 - __clz(below) : 0;
    const uint32_t node_below = __shfl_sync(FULL, (uint32_t)(e >> 32), src);
    const int32_t pw = below ? (int32_t)(c0 + src) : prev_w;
    const uint32_t pw_node = below ? node_below : prev_node;
    if (p < L) {
      const uint32_t h = (uint32_t)(e >> 1) & 127;
      a.pr[(e >> 32) * PR_SLOTS + h] = wait_range(off, p, pw, pw_node, w);
    }
    if (wb) {  // (wb is the same in every lane)
      const int last = 31 - __clz(wb);
      prev_w = (int32_t)(c0 + last);
      prev_node = __shfl_sync(FULL, (uint32_t)(e >> 32), last);
    }
  }
}

// Lists of nodes base .. base + 31 with up to four entries, a lane each
// (longer lists are shared out to whole warps).
__device__ void warp_link(const SpecArgs &a, uint32_t base) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t j = base + lane;
  uint32_t L = 0, off = 0;
  if (j < a.n) {
    L = rd(&a.rlen[j]);
    off = rd(&a.roff[j]);
  }
  if (L >= 1 && L <= 4) {
    // sorted in registers (entries of distinct nodes; padding sorts last)
    uint64_t e[4];
#pragma unroll
    for (uint32_t t = 0; t < 4; ++t) e[t] = t < L ? rd(&a.ent[off + t]) : ~0ull;
    auto cs = [](uint64_t &x, uint64_t &y) {
      const uint64_t lo = x < y ? x : y, hi = x < y ? y : x;
      x = lo;
      y = hi;
    };
    cs(e[0], e[1]);
    cs(e[2], e[3]);
    cs(e[0], e[2]);
    cs(e[1], e[3]);
    cs(e[1], e[2]);
    int32_t pw = -1;
    uint32_t pw_node = NONE;
#pragma unroll
    for (uint32_t t = 0; t < 4; ++t) {
      if (t >= L) break;
      a.ents[off + t] = e[t];
      const bool w = e[t] & 1;
      const uint32_t h = (uint32_t)(e[t] >> 1) & 127;
      a.pr[(e[t] >> 32) * PR_SLOTS + h] = wait_range(off, t, pw, pw_node, w);
      if (w) {
        pw = (int32_t)t;
        pw_node = (uint32_t)(e[t] >> 32);
      }
    }
  }
}

__device__ inline uint8_t ld_acquire_u8(const uint8_t *p) {
  uint16_t v;
  asm volatile("ld.acquire.gpu.global.u8 %0, [%1];" : "=h"(v) : "l"(p) : "memory");
  return (uint8_t)v;
}

// A lane's wait on the turns of one wait range (see wait_range; `first`: the
// first turn's node, already known): until none is pending any more. dmax gets their largest depth. Gives up (false) after
// SPEC_WAIT_NS in which no turn anywhere finished.
__device__ bool wait_on(const SpecArgs &a, uint64_t r, uint32_t first, uint32_t &dmax,
                        unsigned long long &t0, uint32_t &seen) {
  const uint32_t c = (uint32_t)r & 0x7fffffffu;
  for (uint32_t t = 0; t < c; ++t) {
    const uint32_t x = t ? (uint32_t)(rd(&a.ents[(r >> 32) + t]) >> 32) : first;
    for (uint32_t it = 0; ld_acquire_u8(&a.state[x]) == 1; ++it) {
      if (it >= 4 && a.sleep_ns) __nanosleep(a.sleep_ns);
      if ((it & 15) == 15) {
        const uint32_t d = ld_relaxed(&a.counters[C_DONE]);
        const unsigned long long now = now_ns();
        if (!t0 || d != seen) {
          t0 = now;
          seen = d;
        } else if (now - t0 > SPEC_WAIT_NS) {
          return false;
        }
      }
    }
    dmax = max(dmax, ld_relaxed(&a.lev[x]));
  }
  return true;
}

// Per-warp tallies of the turns, added to the counters once per attempt.
struct TurnTally {
  uint32_t fast = 0, slow = 0, depth = 0;
};

// Node i's turn, by one warp: everything about it that cannot change (its
// guessed heads, lane k holding heads k and k + 32, with their positions and
// radii; its record; its masks and pass-start velocity; the first turn each
// of its accesses waits on) is loaded first; then the warp waits until every
// turn its accesses wait on is done; then it reads the velocities and runs
// the turn, and marks the node done (also after a failed turn: the attempt
// then fails as a whole, but every turn still runs).
__device__ void warp_pull(const SpecArgs &a, uint32_t i, bool stamp, TurnTally &tally, double *cx,
                          double *cy, Box *boxes) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
  const uint64_t *prr = a.pr + (size_t)i * PR_SLOTS;
  // what cannot change (rows are read whole; entries past rcount are ignored)
  const uint32_t nr = rd(&a.rcount[i]);
  const uint64_t wm = rd(&a.wmask[i]);
  const uint64_t em = rd(&a.emask[i]);
  const double svi = rd(&a.svx[i]), swi = rd(&a.svy[i]);
  const uint32_t r0 = rd(&rl[lane]), r1 = rd(&rl[lane + 32]);
  const uint64_t q0 = rd(&prr[lane]), q1 = rd(&prr[lane + 32]);
  const uint64_t qs = lane == 0 ? rd(&prr[SELF_ENTRY]) : 0;
  const uint16_t nv = rd(&a.vcount[i]);
  const double md = rd(&a.mdelta[i]);
  const double pxi = a.px[i], pyi = a.py[i];
  uint32_t vc[4], va[4];
  {
    const uint32_t *vl = a.vlist + (size_t)i * VISIT_CAP, *vx = a.vaux + (size_t)i * VISIT_CAP;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      vc[u] = rd(&vl[4 * lane + u]);
      va[u] = rd(&vx[4 * lane + u]);
    }
    // the recorded internal cells' boxes, for a replay (a lane stages its own)
    if (nv != VISIT_NONE) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t t = 4 * lane + u;
        if (t < nv && !(va[u] & LEAF_TAG)) {
          const CRec &q = a.rec[vc[u]];
          boxes[t] = Box{q.x0, q.y0, q.x1, q.y1, q.r};
        }
      }
    }
  }
  const uint32_t j0 = lane < nr ? r0 : NONE, j1 = lane + 32 < nr ? r1 : NONE;
  const uint64_t ww[3] = {lane < nr ? q0 : 0, lane + 32 < nr ? q1 : 0, qs};
  const uint32_t jj[2] = {j0, j1};
  double hxs[2], hys[2], hr[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    hxs[h] = hys[h] = hr[h] = 0;
    if (jj[h] == NONE) continue;
    hxs[h] = a.xs[jj[h]];
    hys[h] = a.ys[jj[h]];
    hr[h] = a.radii[jj[h]];
  }
  uint32_t first[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    first[k] = NONE;
    if (ww[k] & WAIT_NODE) first[k] = (uint32_t)(ww[k] >> 32);
    else if ((uint32_t)ww[k]) first[k] = (uint32_t)(rd(&a.ents[ww[k] >> 32]) >> 32);
  }
  // the wait
  uint32_t dmax = 0, seen = 0;
  unsigned long long t0 = 0;
  bool waited = true;
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (waited) waited = wait_on(a, ww[k], first[k], dmax, t0, seen);
  if (!__all_sync(FULL, waited) && lane == 0) atomicAdd(&a.counters[C_TIMEOUT], 1u);
  for (int o = 16; o > 0; o >>= 1) dmax = max(dmax, __shfl_xor_sync(FULL, dmax, o));
  // the velocities, each read by the lane whose acquiring waits cover it: the
  // node's own by lane 0 (it waited on the node's own accesses), its heads'
  // by their lanes (no other turn writes the heads of a running turn: the
  // values loaded here are what its pushes update)
  double vi = 0, wi = 0;
  if (lane == 0) {
    vi = rd(&a.vxs[i]);
    wi = rd(&a.vys[i]);
  }
  vi = __shfl_sync(FULL, vi, 0);
  wi = __shfl_sync(FULL, wi, 0);
  double hv[2], hw[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    hv[h] = hw[h] = 0;
    if (jj[h] == NONE) continue;
    hv[h] = rd(&a.vxs[jj[h]]);
    hw[h] = rd(&a.vys[jj[h]]);
  }
  const bool unmoved = same_bits(vi, svi) && same_bits(wi, swi);
  // per head: the offset (x, y) = (xi - xs[j] - vxs[j], ...) of the turn,
  // formed as the turn forms it
  const double xi = a.xs[i] + vi, yi = a.ys[i] + wi;
  double hx[2], hy[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    hx[h] = xi - hxs[h] - hv[h];
    hy[h] = yi - hys[h] - hw[h];
  }
  const double ri = a.radii[i], ri2 = ri * ri;
  uint64_t ex = 0;
  bool fail_read = false;
  if (unmoved && !a.force_traverse) {
    ex = em;
  } else if (a.force_traverse ||
             !warp_replay(a, i, xi, yi, unmoved ? VISIT_NONE : nv, md, pxi, pyi, vc, va, boxes, ex)) {
    // i moved beyond its margin: the warp runs the exact traversal; every head
    // it examines must still be among the guessed ones.
    fail_read = !warp_traverse(a, i, xi, yi, ri, jj, ex);
  }
  // each lane evaluates the examined heads with indices lane and lane + 32
  bool fail = false, jig = false;
  uint64_t over = 0;
  // per head slot h: the push on head jj[h] (pushed[h]), written after the
  // warp agrees the turn holds
  bool pushed[2] = {false, false};
  double pdx[2] = {0, 0}, pdy[2] = {0, 0};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t e = lane + 32 * h;
    if (fail_read || e >= nr || !((ex >> e) & 1)) continue;
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
    pushed[h] = true;
    pdx[h] = x * r;
    pdy[h] = y * r;
  }
  fail = __any_sync(FULL, fail);
  jig = __any_sync(FULL, jig);
  for (int o = 16; o > 0; o >>= 1) over |= __shfl_xor_sync(FULL, over, o);
  __syncwarp();
  uint8_t result = 2;
  const bool holds = !(fail_read || fail || jig);
  if (!holds) {
    if (lane == 0) {
      if (jig) atomicAdd(&a.counters[C_JIGGLE], 1u);
      if (fail_read || fail) {
        atomicAdd(&a.counters[C_FAIL], 1u);
        atomicAdd(&a.counters[fail_read ? C_FAIL_READ : C_FAIL_WRITE], 1u);
        result = 3;
      }
    }
  } else {
    if (lane == 0 && over) {
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
    }
    if (unmoved) ++tally.fast;
    else ++tally.slow;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!pushed[h]) continue;
      const uint32_t j = jj[h];
      a.vxs[j] = hv[h] - pdx[h];
      a.vys[j] = hw[h] - pdy[h];
      atomicAdd(&a.push[j], sqrt(pdx[h] * pdx[h] + pdy[h] * pdy[h]));
      atomicMin(&a.min_pusher[j], i);
      atomicMax(&a.max_pusher[j], i);
    }
  }
  // done: after the writes (a turn that wrote nothing has finished its reads)
  if (holds && over) __threadfence();
  __syncwarp();
  const uint32_t lv = dmax + 1;
  tally.depth = max(tally.depth, lv);
  if (lane == 0) {
    a.lev[i] = lv;
    a.state[i] = result;
    atomicAdd(&a.counters[C_DONE], 1u);
    if (stamp) {
      const uint32_t k = lv - 1 < 63 ? lv - 1 : 63;
      atomicMax(&a.stamps[16 + k], now_ns());
      atomicAdd(&a.stamps[80 + k], 1ull);
    }
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
      c = pruned(q, xi, yi, r) ? a.skip[c] : c + 1;
    }
  }
  a.rng->lcg = s;
}

__global__ void __launch_bounds__(SPEC_THREADS, 2) k_collide_spec(SpecArgs a) {
  __shared__ double contrib[SPEC_WARPS][2][SPEC_CAP];
  extern __shared__ Box boxes_all[];  // SPEC_WARPS * VISIT_CAP (dynamic)
  cg::grid_group g = cg::this_grid();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t gw = tid >> 5, nwarps = nth >> 5, wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t n = a.n;
  if (tid < C_COUNTERS) a.counters[tid] = 0;
  if (tid == 0) {
    for (int k = 0; k < 144; ++k) a.stamps[k] = 0;
    a.stamps[0] = now_ns();
  }
  // No tree this pass (cell buffer overflow or a failed build launch, both
  // already reported in the status word): leaf_of and the cells are not this
  // pass's, so nothing is read. Every thread reads the same word, written
  // before this launch, so every block returns here before any grid barrier.
  if (__ldcg(&a.info[5])) return;
  for (uint32_t i = tid; i < n; i += nth) a.cnt[i] = 0;
  {
    const uint32_t len = a.info[1];
    for (uint32_t c = tid; c < len; c += nth) {
      const Cell &q = a.cells[c];
      CRec rc;
      rc.x0 = q.x0;
      rc.y0 = q.y0;
      rc.x1 = q.x1;
      rc.y1 = q.y1;
      rc.r = q.r;
      if (is_leaf(q)) {
        const uint32_t j = a.perm[q.first + q.count - 1];
        rc.link = j | LEAF_TAG;
        rc.margin = (float)margin_of(a, j);
        rc.hx = a.px[j];
        rc.hy = a.py[j];
      } else {
        rc.link = a.skip[c];
        rc.margin = 0;
        rc.hx = rc.hy = 0;
      }
      a.rec[c] = rc;
    }
  }
  g.sync();
  // G, plus per-node resets, the pass-start snapshot and the access counts.
  for (uint32_t i = tid; i < n; i += nth) {
    a.svx[i] = a.vxs[i];
    a.svy[i] = a.vys[i];
    a.push[i] = 0;
    a.min_pusher[i] = NONE;
    a.max_pusher[i] = 0;
    a.aflag[i] = 0;
    if (!spec_guess_fit(a, i, margin_of(a, i), false)) {
      atomicAdd(&a.counters[C_OVERFLOW], 1u);
      a.state[i] = 0;
      continue;
    }
    if (a.wmask[i]) {
      a.state[i] = 1;
      a.active[atomicAdd(&a.counters[C_ACTIVE], 1u)] = i;
      a.aflag[i] = 1;
      const uint32_t *rl = a.rlist + (size_t)i * SPEC_CAP;
      const uint32_t nr = a.rcount[i];
      for (uint32_t h = 0; h < nr; ++h) atomicAdd(&a.cnt[rl[h]], 1u);
      atomicAdd(&a.cnt[i], 1u);
    } else {
      a.state[i] = 0;
    }
  }
  g.sync();
  if (tid == 0) a.stamps[1] = now_ns();
  bool ok = false;
  for (int attempt = 0; attempt < SPEC_ATTEMPTS && !ok; ++attempt) {
    if (rd(&a.counters[C_OVERFLOW]) || rd(&a.counters[C_JIGGLE]) || rd(&a.counters[C_TIMEOUT]))
      break;
    const uint32_t n_active = rd(&a.counters[C_ACTIVE]);
    if (attempt > 0) {
      for (uint32_t k = gw; k < n_active; k += nwarps) warp_count(a, rd(&a.active[k]));
      g.sync();
    }
    // The access lists: places (and the nodes and lists with more than four
    // entries, which whole warps share out), entries, then sorted and linked.
    for (uint32_t base = gw * 32; base < n; base += nwarps * 32) warp_offsets(a, base);
    for (uint32_t base = gw * 32; base < n_active; base += nwarps * 32)
      warp_find_bigfill(a, base, n_active);
    if (tid == 0) a.counters[C_CLAIM] = a.counters[C_VWORK] = 0;
    // the active nodes' places in index order (one grid barrier inside)
    grid_excl_scan(g, a.aflag, a.apos, n, a.scan_part);
    g.sync();
    if (tid == 0 && attempt == 0) a.stamps[13] = now_ns();
    for (uint32_t base = gw * 32; base < n_active; base += nwarps * 32) warp_fill(a, base, n_active);
    {
      const uint32_t nb = rd(&a.counters[C_BIGFILL]);
      for (uint32_t k = gw; k < nb; k += nwarps) warp_fill_big(a, rd(&a.bigfill[k]));
    }
    g.sync();
    if (tid == 0 && attempt == 0) a.stamps[14] = now_ns();
    for (uint32_t base = gw * 32; base < n; base += nwarps * 32) warp_link(a, base);
    {
      const uint32_t nb = rd(&a.counters[C_BIGLINK]);
      for (uint32_t k = gw; k < nb; k += nwarps) {
        const uint32_t j = rd(&a.biglink[k]);
        warp_link_list(a, rd(&a.roff[j]), rd(&a.rlen[j]));
      }
    }
    g.sync();
    if (tid == 0 && attempt < 3) a.stamps[10 + attempt] = now_ns();
    // E: warps claim the active nodes in index order (every turn waits only
    // on turns of lower index) and run them once what they wait on is done.
    {
      TurnTally tally;
      uint32_t k = 0;
      if (lane == 0) k = atomicAdd(&a.counters[C_CLAIM], 1u);
      k = __shfl_sync(FULL, k, 0);
      uint32_t i = k < n_active ? rd(&a.sact[k]) : NONE;
      while (k < n_active) {
        // the next claim and its node, loaded before this turn runs
        uint32_t nk = 0, ni = NONE;
        if (lane == 0) {
          nk = atomicAdd(&a.counters[C_CLAIM], 1u);
          if (nk < n_active) ni = rd(&a.sact[nk]);
        }
        warp_pull(a, __shfl_sync(FULL, i, 0), a.profile && attempt == 0, tally, contrib[wl][0],
                  contrib[wl][1], boxes_all + (size_t)wl * VISIT_CAP);
        k = __shfl_sync(FULL, nk, 0);
        i = __shfl_sync(FULL, ni, 0);
      }
      if (lane == 0) {
        if (tally.fast) atomicAdd(&a.counters[C_FAST_TURNS], tally.fast);
        if (tally.slow) atomicAdd(&a.counters[C_SLOW_TURNS], tally.slow);
        if (tally.depth) atomicMax(&a.counters[C_DEPTH], tally.depth);
      }
    }
    g.sync();
    if (tid == 0 && attempt < 3) a.stamps[2 + 2 * attempt] = now_ns();
    // V: inactive nodes stayed no-ops (Morton order, as G).
    for (uint32_t base = gw * 32; base < n; base += nwarps * 32) warp_check_inactive(a, base);
    g.sync();
    {
      const uint32_t nw = rd(&a.counters[C_VWORK]);
      for (uint32_t k = gw; k < nw; k += nwarps) warp_check_inactive_item(a, rd(&a.vwork[k]));
    }
    g.sync();
    if (tid == 0 && attempt < 3) a.stamps[3 + 2 * attempt] = now_ns();
    if (tid == 0) atomicAdd(&a.counters[C_ATTEMPTS], 1u);
    if (rd(&a.counters[C_FAIL]) == 0 && rd(&a.counters[C_DONE]) >= n_active &&
        rd(&a.counters[C_JIGGLE]) == 0 && rd(&a.counters[C_TIMEOUT]) == 0) {
      ok = true;
      break;
    }
    // Retry: restore, promote failed nodes, make every active node pending again.
    for (uint32_t i = tid; i < n; i += nth) {
      a.vxs[i] = a.svx[i];
      a.vys[i] = a.svy[i];
      a.push[i] = 0;
      a.min_pusher[i] = NONE;
      a.max_pusher[i] = 0;
      a.cnt[i] = 0;
      const uint8_t st = rd(&a.state[i]);
      if (st == 3 || st == 4) {
        // every head within a four times wider margin may be written
        if (!spec_guess_fit(a, i, 4 * rd(&a.mdelta[i]), true)) atomicAdd(&a.counters[C_OVERFLOW], 1u);
        if (st == 4) {  // was inactive
          a.active[atomicAdd(&a.counters[C_ACTIVE], 1u)] = i;
          a.aflag[i] = 1;
        }
        a.state[i] = 1;
      } else if (st == 2) {
        a.state[i] = 1;
      }
    }
    g.sync();
    if (tid == 0) {
      a.counters[C_FAIL] = 0;
      a.counters[C_DONE] = 0;
      a.counters[C_ALLOC] = 0;
      a.counters[C_BIGFILL] = 0;
      a.counters[C_BIGLINK] = 0;
    }
    g.sync();
  }
  if (ok) {
    for (uint32_t i = tid; i < n; i += nth) a.push_prev[i] = a.push[i];
    if (tid == 0) a.stamps[9] = now_ns();
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
// Dynamic shared memory of k_collide_spec: the staged boxes, per warp.
constexpr size_t SPEC_DYN_SMEM = (size_t)SPEC_WARPS * VISIT_CAP * sizeof(Box);

// Every device array of the scratch, with its bytes per node of capacity.
template <class F>
static void spec_arrays(CollideSpec &s, F f) {
  f((void **)&s.rlist, SPEC_CAP * 4ull);
  f((void **)&s.rcount, 1);
  f((void **)&s.wmask, 8);
  f((void **)&s.emask, 8);
  f((void **)&s.state, 1);
  f((void **)&s.active, 8);  // room for promoted nodes
  f((void **)&s.push, 8);
  f((void **)&s.min_pusher, 4);
  f((void **)&s.max_pusher, 4);
  f((void **)&s.vlist, VISIT_CAP * 4ull);
  f((void **)&s.vaux, VISIT_CAP * 4ull);
  f((void **)&s.vcount, 2);
  f((void **)&s.start, 4);
  f((void **)&s.mdelta, 8);
  f((void **)&s.push_prev, 8);
  f((void **)&s.cnt, 4);
  f((void **)&s.rlen, 4);
  f((void **)&s.roff, 4);
  f((void **)&s.ent, (SPEC_CAP + 1) * 8ull);  // at most SPEC_CAP heads and itself per node
  f((void **)&s.ents, (SPEC_CAP + 1) * 8ull);
  f((void **)&s.pr, PR_SLOTS * 8ull);
  f((void **)&s.lev, 4);
  f((void **)&s.aflag, 4);
  f((void **)&s.apos, 4);
  f((void **)&s.sact, 4);
  f((void **)&s.work, 3 * 4ull);  // bigfill, biglink, vwork
}

int collide_spec_reserve(CollideSpec &s, uint32_t n) {
  if (n <= s.cap && s.cap) return 0;
  uint32_t cap = n < 1024 ? 1024 : n;
  spec_arrays(s, [](void **p, size_t) {
    cudaFree(*p);
    *p = nullptr;
  });
  if (!s.counters) {
    D3_CUDA_OK(cudaMalloc(&s.counters, C_COUNTERS * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMemset(s.counters, 0, C_COUNTERS * sizeof(uint32_t)));
    D3_CUDA_OK(cudaMalloc(&s.grid_part, 1024 * sizeof(uint32_t)));
  }
  // 16 phase stamps, then attempt 1's per-depth last finish times and turn
  // counts (64 each)
  if (!s.stamps) D3_CUDA_OK(cudaMalloc(&s.stamps, 144 * sizeof(unsigned long long)));
  bool fail = false;
  spec_arrays(s, [&](void **p, size_t per) {
    if (!fail && cudaMalloc(p, per * cap) != cudaSuccess) fail = true;
  });
  if (fail) {
    spec_arrays(s, [](void **p, size_t) {
      cudaFree(*p);
      *p = nullptr;
    });
    cudaGetLastError();
    return D3_OUT_OF_MEMORY;
  }
  D3_CUDA_OK(cudaMemset(s.push_prev, 0, cap * 8ull));
  s.cap = cap;
  return 0;
}

void collide_spec_free(CollideSpec &s) {
  spec_arrays(s, [](void **p, size_t) { cudaFree(*p); });
  cudaFree(s.counters);
  cudaFree(s.grid_part);
  cudaFree(s.stamps);
  s = CollideSpec();
}

int collide_parallel(TreeDev &t, const NodeArrays &a, const double *radii, double strength,
                     double delta, Rng *rng, CollideSpec &s, cudaStream_t st) {
  if (a.n == 0) return 0;
  if (!g_spec_blocks) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_collide_spec, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)SPEC_DYN_SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_collide_spec, SPEC_THREADS, SPEC_DYN_SMEM);
    // blocks per SM: full occupancy (at most 2), or D3_COLLIDE_BLOCKS_PER_SM
    int want = per > 2 ? 2 : per;
    if (const char *e = getenv("D3_COLLIDE_BLOCKS_PER_SM")) {
      const int v = atoi(e);
      if (v >= 1 && v <= want) want = v;
    }
    g_spec_blocks = sms * (want > 0 ? want : 1);
    if (g_spec_blocks <= 0) g_spec_blocks = sms;
  }
  SpecArgs args;
  args.rec = (CRec *)t.rec;
  args.cells = t.cells; args.skip = t.skip; args.perm = t.perm; args.info = t.info;
  args.parent = t.parent; args.leaf_of = t.leaf_of;
  args.xs = a.x; args.ys = a.y; args.px = a.px; args.py = a.py; args.radii = radii;
  args.vxs = a.vx; args.vys = a.vy; args.svx = a.snap_vx; args.svy = a.snap_vy;
  args.strength = strength; args.delta0 = delta; args.n = a.n;
  // D3_COLLIDE_FORCE_TRAVERSE (any value): every turn finds its examined heads
  // by the exact traversal instead of the recorded ones (a test of that path)
  args.force_traverse = getenv("D3_COLLIDE_FORCE_TRAVERSE") != nullptr;
  args.profile = s.profile;
  args.sleep_ns = wait_sleep_ns();
  args.rlist = s.rlist; args.rcount = s.rcount; args.wmask = s.wmask; args.emask = s.emask;
  args.vlist = s.vlist; args.vaux = s.vaux; args.vcount = s.vcount; args.start = s.start; args.mdelta = s.mdelta;
  args.state = s.state; args.active = s.active;
  args.cnt = s.cnt; args.rlen = s.rlen; args.roff = s.roff; args.ent = s.ent; args.ents = s.ents;
  args.pr = s.pr; args.lev = s.lev; args.aflag = s.aflag; args.apos = s.apos; args.sact = s.sact;
  args.scan_part = s.grid_part;
  args.bigfill = s.work;
  args.biglink = s.work + s.cap;
  args.vwork = s.work + 2ull * s.cap;
  args.push = s.push; args.push_prev = s.push_prev; args.min_pusher = s.min_pusher;
  args.max_pusher = s.max_pusher; args.counters = s.counters; args.stamps = s.stamps;
  args.rng = rng;
  void *params[] = {&args};
  ++g_launches;
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_collide_spec, g_spec_blocks,
                                              SPEC_THREADS, params, SPEC_DYN_SMEM, st);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace d3
