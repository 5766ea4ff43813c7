// fmm_tc.cu — the precision form of the fast many-body force: an FMM whose
// translation operators are the same at every level, with M2L run as batched
// dense BF16x3 contractions on the tensor cores (tcgen05) and the near field
// in FP32 (no reference counterpart: it is judged by its RMS force error
// against an FP64 direct sum, the measure of test/fast/error-test.js:44-70).
//
// The reference FMM (fmm.zig:247-354) centres each cell on its points'
// bounding box (fmm.zig:749-753), so no two cells share a translation vector.
// Here each cell is centred on its square (the key grid of tree.zig:346-364),
// and expansions are stored normalised by the cell side s:
//     M'_k = M_k / s^k,    L'_l = L_l * s^(l+1),
// in the scaled coordinates u = (x - ox) / w of fmm.zig:668-682. Then, for
// two cells of one level with c_A - c_B = s v (v integer),
//     L'_l += (-1)^l sum_k C(k+l, l) M'_k / v^(k+l+1),
// a fixed q x q complex matrix per v, the same at every level; M2M and L2L
// are fixed matrices per child quadrant. With the separation test
// |v|^2 >= 2 kappa^2 (the MAC (2 kappa - 1) r_max + r_min <= d of
// fmm.zig:400-453 for equal squares, r = s / sqrt 2), the cells a cell gets
// M2L from are the children of its parent's near cells that are separated
// from it: 39 vectors per child quadrant at kappa = 1.5 (60 in all).
//
// Passes (one GPU; the main stream in order, two passes on a second stream):
//   prepare  fmm_prepare (fmm.cu): keys, sort, gather, level-order cells.
//   geom     per cell: level, integer coordinates, quadrant, child mask;
//            the leaf list and the M2L target groups (one per quadrant).
//   lists    a launch per level from the root, a warp per cell: near cells
//            (13 at kappa 1.5), the M2L table (source per vector slot), and
//            the adaptive lists: P2P leaves, coarse leaves (P2L), finer
//            cells seen from a leaf (M2P). Then one host read of the counts.
//   upward   FP64, a thread per leaf (on the second stream, beside the
//            lists): P2M, then M2M into each parent by the
//            thread that completes it (arrival counters, no level
//            barriers); M' stored in FP64 and split into bf16 hi + lo
//            (x ~ hi + lo to 2^-17) for the tensor cores.
//   m2l      tcgen05: a CTA per tile of 128 target cells of one quadrant
//            group; per vector slot the 128 gathered source rows (A: 128 x
//            32 bf16, hi and lo) times that vector's operator (B: 32 x 32,
//            hi and lo) accumulate in TMEM as A_hi B_hi + A_hi B_lo +
//            A_lo B_hi (BF16x3), FP32 accumulation; cp.async gathers into a
//            3-stage smem ring with mbarriers, one lane issues the MMAs.
//   p2l      coarse leaves' points into local expansions (FP32 series).
//   down     a thread per leaf: its ancestors' local expansions shifted to
//            the leaf's centre (the L2L chain composed, FP32).
//   near     a warp per leaf, on the second stream beside M2L / P2L /
//            down: the source leaves' points staged in shared memory
//            relative to the leaf's first point (the shift in FP64, the pair
//            sums in FP32: d3's pair formula, distanceMin clamp, hashed
//            jiggle of hash.zig for coincident points) into a per-point
//            buffer.
//   far      a thread per point: L2P and M2P, then v += near + far in FP64.

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fast.cuh"
#include "mlp.cuh"
#include "tc.cuh"


namespace d3 {
namespace {

constexpr uint32_t TC_MAXQ = 16;     // q = p + 1: 2q <= 32, the MMA's K and N
constexpr uint32_t TC_KN = 32;       // padded real length of an expansion
constexpr uint32_t TC_NEAR_MAX = 32;  // near offsets (13 at kappa 1.5)
constexpr uint32_t TC_SLOT_MAX = 96;  // M2L vectors per quadrant (39 at kappa 1.5)
constexpr uint32_t TC_CLASS_MAX = 192;
constexpr uint32_t TC_THREADS = 256;
constexpr uint32_t TC_WARPS = TC_THREADS / 32;
constexpr uint32_t TC_TILE = 128;     // target cells per M2L tile (the MMA's M)
constexpr uint32_t TC_STACK = 64;
constexpr uint32_t TC_NONE = 0xFFFFFFFFu;
constexpr uint32_t TC_NEAR_FLAG = 0x8000u;
// info words
enum : uint32_t { TI_POOL_P2P = 0, TI_POOL_W, TI_POOL_X, TI_POOL_C, TI_OVF, TI_GROUP = 8,
                  TI_LEAVES = 12, TI_ERR = 16, TI_WORDS = 32 };
// The learned correction's output unit: the network predicts
// (L'_0 at order 12 - L'_0 at order 4) / sc * LEARN_TARGET_SCALE.
constexpr float LEARN_TARGET_SCALE = 1000.f;
constexpr uint32_t LEARN_ORDER = 4;
constexpr uint32_t CHECK_THREADS = 256;

// A cell of the geometric tree: the square of level `level` at integer
// coordinates (ix, iy), side 2^-level in scaled coordinates, centre
// -0.5 + (ix + 0.5) 2^-level.
struct TcCell {
  uint32_t first, count, child0, parent;
  uint16_t ix, iy;
  uint8_t level, quad, cmask, nchild;
};

struct TcTables {
  uint32_t q, nnear, nslot[4];
  uint32_t sstride;  // the M2L table's row length: the largest nslot
  int8_t near_dx[TC_NEAR_MAX], near_dy[TC_NEAR_MAX];
  // [target quadrant a][parent near offset o][child quadrant b]: M2L slot,
  // or TC_NEAR_FLAG | near index
  uint16_t map[4][TC_NEAR_MAX][4];
  uint16_t slot_class[4][TC_SLOT_MAX];
  double kappa2x2;   // 2 kappa^2: separation of same-level offsets
  double mac_far;    // 2 kappa - 1
  double m2m_re[4][TC_MAXQ][TC_MAXQ], m2m_im[4][TC_MAXQ][TC_MAXQ];  // [b][n][k]
  float l2l_re[4][TC_MAXQ][TC_MAXQ], l2l_im[4][TC_MAXQ][TC_MAXQ];   // [b][m][l]
};

// The tables of one (order, opening): operators on the device, and their
// host copy.
struct TcTabSet {
  uint32_t p = 0;
  double kappa = 0;
  TcTables *tab = nullptr;
  unsigned char *wops = nullptr;  // [class][hi, lo][32 x 32 bf16, B tile layout]
  TcTables h;
};

struct TcDev {
  uint32_t ccap = 0, pcap = 0, lcap = 0;
  TcTabSet sets[2];  // the last two (order, opening) pairs used
  uint32_t next_set = 0;
  TcCell *cells = nullptr;
  double *mco = nullptr;            // M' (FP64), 2q per cell
  __nv_bfloat16 *mbf = nullptr;     // M' hi (32) then lo (32) per cell
  float *lco = nullptr;             // L' (FP32), 32 per cell
  uint32_t *near = nullptr;         // [cell][nnear]
  uint32_t *m2l = nullptr;          // [cell][nslot of its quadrant]
  uint32_t *groups = nullptr;       // 4 lists of cells, each ccap long
  uint32_t *loff = nullptr;         // per cell: offsets/counts of p2p, w, x, coarse lists
  uint32_t *pool = nullptr;
  size_t pool_cap = 0, last_pool = 0;
  uint32_t *info = nullptr, *h_info = nullptr;
  int sms = 0;
  uint32_t *arrive = nullptr;        // per cell: children finished (upward pass)
  // the learned form
  float *feat = nullptr;             // per cell: 16 floats (k_tc_features)
  uint32_t *leaves = nullptr;        // leaf cells (ccap)
  float *mlp_x = nullptr, *mlp_y = nullptr;  // per leaf: 12 inputs, 2 outputs
  double2 *kick = nullptr;           // per sorted point: the many-body kick
  double *chk = nullptr, *h_chk = nullptr;   // sampled check: sum err^2, sum ref^2
  double2 *chk_part = nullptr;               // the check's partial direct sums
  uint32_t chk_cap = 0;                      // entries chk_part holds
  float2 *nearbuf = nullptr;                 // per sorted point: the learned pass's near field
  uint32_t *leafidx = nullptr;               // per sorted point: its leaf's index in the leaf list
  float *mlp = nullptr;              // installed network parameters (device)
  uint32_t ncells_last = 0;
  uint32_t hold = 0;                 // ticks left on the fallback after a failed check
  // CUDA events of the last run: main stream 0 start, 1 prepared, 2 lists
  // built, 3 upward waited for, 4 M2L, 5 P2L, 6 downward, 11 network, 12 far
  // field; side stream 7, 8 around the near field, 9, 10 around the upward
  // pass
  cudaEvent_t ev[13] = {};
  // the upward pass runs on `side` while the lists are built on the main
  // stream: ev_geom (geometry done) and ev_up (upward done) order them
  cudaStream_t side = nullptr;
  cudaEvent_t ev_geom = nullptr, ev_up = nullptr;
  // the near field runs on `side` after the lists (ev_lists) until ev_near;
  // the feature rows after the downward pass (ev_down) until ev_feat
  cudaEvent_t ev_lists = nullptr, ev_near = nullptr, ev_down = nullptr, ev_feat = nullptr;
  cudaEvent_t ev_side_idle = nullptr;  // all side-stream work queued so far
  uint32_t last_tiles = 0, last_slots = 0;
  void *last_args = nullptr;  // a TcArgs copy of the last pass (for the work counts)
};

struct TcArgs {
  const TcTables *tab;
  const unsigned char *wops;
  const uint64_t *keys;
  const uint32_t *perm;
  const double *px, *py, *ps, *ux, *uy;
  const FCell *fc;
  TcCell *cells;
  double *mco;
  __nv_bfloat16 *mbf;
  float *lco;
  uint32_t *near, *m2l, *groups, *loff, *pool;
  size_t pool_cap;
  float *feat, *mlp_x, *mlp_y;
  uint32_t *leaves;
  uint32_t *leafidx;  // per sorted point: its leaf's index in the leaf list (near pass)
  double2 *kick;  // non-null: the many-body kick goes here instead of into vx, vy
  double *vx, *vy;
  uint32_t *info;
  uint32_t *status;     // the simulation's status word (ST_WAIT_TIMEOUT on a failed wait)
  const uint32_t *lvl;  // device: first cell of each level
  uint32_t ncells, nlev, m, q, ccap;
  double inv_w, dmin2;
  float dmin2f;
  const double *seed;
};

// 2^e for the small exponents of cell levels (|e| < 127), built exactly.
__device__ __forceinline__ double pow2(int e) {
  return __longlong_as_double((long long)(1023 + e) << 52);
}
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }
__device__ __forceinline__ double cell_side(uint32_t level) { return pow2(-(int)level); }
__device__ __forceinline__ void cell_centre(const TcCell &c, double &x, double &y) {
  const double s = cell_side(c.level);
  x = -0.5 + (c.ix + 0.5) * s;
  y = -0.5 + (c.iy + 0.5) * s;
}
__device__ __forceinline__ uint32_t child_at(const TcCell &c, uint32_t b) {
  if (!((c.cmask >> b) & 1)) return TC_NONE;
  return c.child0 + __popc(c.cmask & ((1u << b) - 1));
}

// ---- geom -------------------------------------------------------------------------

__device__ __forceinline__ uint32_t compact16(uint32_t x) {  // even bits -> 16 bits
  x &= 0x55555555u;
  x = (x | (x >> 1)) & 0x33333333u;
  x = (x | (x >> 2)) & 0x0F0F0F0Fu;
  x = (x | (x >> 4)) & 0x00FF00FFu;
  x = (x | (x >> 8)) & 0x0000FFFFu;
  return x;
}

// A thread per cell; the leaf list and the four quadrant groups are filled
// with one atomic per warp and list (their order is free: every later pass
// treats their entries independently).
__global__ void k_tc_geom(TcArgs a) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned lane = threadIdx.x & 31, lt = (1u << lane) - 1;
  const bool valid = c < a.ncells;
  TcCell t{};
  uint32_t depth = 0;
  if (valid) {
    const FCell f = a.fc[c];
    t.first = f.first;
    t.count = f.count;
    t.parent = f.parent;
    t.level = (uint8_t)f.depth;
    depth = f.depth;
    const uint32_t key = (uint32_t)a.keys[f.first];
    const uint32_t pre = f.depth ? key >> (2 * (16 - f.depth)) : 0;
    t.ix = (uint16_t)compact16(pre);
    t.iy = (uint16_t)compact16(pre >> 1);
    t.quad = (uint8_t)(pre & 3);
    // the children: contiguous from child0, one per non-empty quadrant in order
    uint32_t mask = 0;
    const uint32_t nch = f.nchild;
    for (uint32_t j = 0; j < nch; ++j) {
      const FCell ch = a.fc[f.child0 + j];
      const uint32_t ck = (uint32_t)a.keys[ch.first];
      mask |= 1u << ((ck >> (2 * (16 - ch.depth))) & 3);
    }
    t.cmask = (uint8_t)mask;
    t.nchild = (uint8_t)nch;
    t.child0 = nch ? f.child0 : 0;
    a.cells[c] = t;
    if (nch) a.feat[(size_t)c * 16 + 15] = -1.f;  // no feature row: not a leaf
    if (c == 0)  // the root gets no M2L: its local expansion starts at zero
      for (uint32_t k = 0; k < TC_KN; ++k) a.lco[k] = 0;
  }
  // the leaf list
  const unsigned leaves = __ballot_sync(0xffffffffu, valid && t.nchild == 0);
  uint32_t lb = 0;
  if (leaves && lane == __ffs(leaves) - 1) lb = atomicAdd(&a.info[TI_LEAVES], __popc(leaves));
  lb = __shfl_sync(0xffffffffu, lb, leaves ? __ffs(leaves) - 1 : 0);
  if (valid && t.nchild == 0) a.leaves[lb + __popc(leaves & lt)] = c;
  // the quadrant groups (every cell but the root)
  const uint32_t g = valid && depth > 0 ? t.quad : 4u + lane;  // 4+: no group, never matches
  const unsigned peers = __match_any_sync(0xffffffffu, g);
  const uint32_t leader = __ffs(peers) - 1;
  uint32_t gb = 0;
  if (g < 4 && lane == leader) gb = atomicAdd(&a.info[TI_GROUP + g], __popc(peers));
  gb = __shfl_sync(0xffffffffu, gb, leader);
  if (g < 4) a.groups[(size_t)g * a.ccap + gb + __popc(peers & lt)] = c;
}

// ---- upward (FP64): P2M per leaf, M2M by the last child to finish ----------------------------

constexpr uint32_t UP_THREADS = 128;

// M' of cell c (Q = q complex coefficients) into mco and its bf16 split
// (hi row then lo row, 32 reals each, zero padded) into mbf.
template <int Q>
__device__ __forceinline__ void tc_store_m(const TcArgs &a, uint32_t c, const double *mr,
                                           const double *mi) {
  double *mc = a.mco + (size_t)c * 2 * Q;
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    mc[k] = mr[k];
    mc[Q + k] = mi[k];
  }
  uint32_t hi[16], lo[16];  // bf16 pairs
#pragma unroll
  for (int w = 0; w < 16; ++w) {
    __nv_bfloat16 h0, l0, h1, l1;
    const int p0 = 2 * w, p1 = 2 * w + 1;
    const double v0 = p0 < Q ? mr[p0 < Q ? p0 : 0] : p0 < 2 * Q ? mi[p0 < 2 * Q && p0 >= Q ? p0 - Q : 0] : 0.0;
    const double v1 = p1 < Q ? mr[p1 < Q ? p1 : 0] : p1 < 2 * Q ? mi[p1 < 2 * Q && p1 >= Q ? p1 - Q : 0] : 0.0;
    tc::split_bf16(v0, h0, l0);
    tc::split_bf16(v1, h1, l1);
    hi[w] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
    lo[w] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
  }
  uint4 *dst = reinterpret_cast<uint4 *>(a.mbf + (size_t)c * 64);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    dst[v] = make_uint4(hi[4 * v], hi[4 * v + 1], hi[4 * v + 2], hi[4 * v + 3]);
    dst[4 + v] = make_uint4(lo[4 * v], lo[4 * v + 1], lo[4 * v + 2], lo[4 * v + 3]);
  }
}

// A thread per leaf: P2M, M'_k = sum_j s_j ((u_j - c) / s)^k with the points
// added in order (upwardCell, fmm.zig:757-807, on the cell's square); then, while its cell
// is the last of its parent's children to finish (arrival counters, `arrive`
// zeroed before the launch), the same thread builds the parent by M2M,
// M'^P_n = sum_b sum_{k<=n} op_b[n][k] M'^b_k over the children in quadrant
// order (the M2M of upwardCell with the fixed quadrant operators). No level
// barriers: a parent is built once, by the thread that completes it, from
// children read through L2.
template <int Q>
__global__ void __launch_bounds__(UP_THREADS) k_tc_upward(TcArgs a, uint32_t *arrive) {
  __shared__ double opr[4][Q][Q], opi[4][Q][Q];
  for (uint32_t i = threadIdx.x; i < 4 * Q * Q; i += blockDim.x) {
    const uint32_t b = i / (Q * Q), n = (i / Q) % Q, k = i % Q;
    opr[b][n][k] = a.tab->m2m_re[b][n][k];
    opi[b][n][k] = a.tab->m2m_im[b][n][k];
  }
  __syncthreads();
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= __ldcg(&a.info[TI_LEAVES])) return;
  uint32_t c = a.leaves[e];
  TcCell C = a.cells[c];
  double mr[Q], mi[Q];
#pragma unroll
  for (int k = 0; k < Q; ++k) mr[k] = mi[k] = 0.0;
  {
    double cx, cy;
    cell_centre(C, cx, cy);
    const double inv_s = pow2((int)C.level);
    for (uint32_t j = C.first; j < C.first + C.count; ++j) {
      const double sv = __ldg(&a.ps[j]);
      const double zr = (__ldg(&a.ux[j]) - cx) * inv_s, zi = (__ldg(&a.uy[j]) - cy) * inv_s;
      double pr = sv, pi = 0;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        mr[k] += pr;
        mi[k] += pi;
        const double nr = pr * zr - pi * zi;
        pi = pr * zi + pi * zr;
        pr = nr;
      }
    }
  }
  for (uint32_t guard = 0; guard < 32; ++guard) {
    tc_store_m<Q>(a, c, mr, mi);
    __threadfence();
    if (C.parent == TC_NONE) break;
    const uint32_t par = C.parent;
    const TcCell P = a.cells[par];
    if (atomicAdd(&arrive[par], 1u) + 1 != P.nchild) break;
    __threadfence();
#pragma unroll
    for (int k = 0; k < Q; ++k) mr[k] = mi[k] = 0.0;
    for (uint32_t b = 0; b < 4; ++b) {
      const uint32_t ch = child_at(P, b);
      if (ch == TC_NONE) continue;
      const double *cm = a.mco + (size_t)ch * 2 * Q;
      double cr[Q], ci[Q];
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        cr[k] = __ldcg(&cm[k]);
        ci[k] = __ldcg(&cm[Q + k]);
      }
#pragma unroll
      for (int n = 0; n < Q; ++n)
#pragma unroll
        for (int k = 0; k <= n; ++k) {
          const double orr = opr[b][n][k], oi = opi[b][n][k];
          mr[n] += orr * cr[k] - oi * ci[k];
          mi[n] += orr * ci[k] + oi * cr[k];
        }
    }
    c = par;
    C = P;
  }
}

template <int Q>
void launch_up_q(const TcArgs &g, uint32_t *arrive, unsigned blocks, cudaStream_t st) {
  D3_LAUNCH(k_tc_upward<Q>, blocks, UP_THREADS, 0, st)(g, arrive);
}

void launch_up(const TcArgs &g, uint32_t *arrive, uint32_t nleaf, cudaStream_t st) {
  const unsigned blocks = blocks_for(nleaf, UP_THREADS);
  if (!blocks) return;
  switch (g.q) {
    case 2: launch_up_q<2>(g, arrive, blocks, st); break;
    case 3: launch_up_q<3>(g, arrive, blocks, st); break;
    case 4: launch_up_q<4>(g, arrive, blocks, st); break;
    case 5: launch_up_q<5>(g, arrive, blocks, st); break;
    case 6: launch_up_q<6>(g, arrive, blocks, st); break;
    case 7: launch_up_q<7>(g, arrive, blocks, st); break;
    case 8: launch_up_q<8>(g, arrive, blocks, st); break;
    case 9: launch_up_q<9>(g, arrive, blocks, st); break;
    case 10: launch_up_q<10>(g, arrive, blocks, st); break;
    case 11: launch_up_q<11>(g, arrive, blocks, st); break;
    case 12: launch_up_q<12>(g, arrive, blocks, st); break;
    case 13: launch_up_q<13>(g, arrive, blocks, st); break;
    case 14: launch_up_q<14>(g, arrive, blocks, st); break;
    case 15: launch_up_q<15>(g, arrive, blocks, st); break;
    default: launch_up_q<16>(g, arrive, blocks, st); break;
  }
}

// ---- lists ----------------------------------------------------------------------------

// The MAC of fmm.zig:400-453 between squares of different levels (r = s / sqrt 2).
__device__ __forceinline__ bool separated(const TcArgs &a, const TcCell &A, const TcCell &B) {
  double ax, ay, bx, by;
  cell_centre(A, ax, ay);
  cell_centre(B, bx, by);
  const double ra = cell_side(A.level) * 0.7071067811865476;
  const double rb = cell_side(B.level) * 0.7071067811865476;
  const double dx = ax - bx, dy = ay - by;
  const double rmax = ra > rb ? ra : rb, rmin = ra > rb ? rb : ra;
  const double thr = a.tab->mac_far * rmax + rmin;
  return dx * dx + dy * dy >= thr * thr;
}

// Per-lane list events. WRITE false: counts; true: writes from the offsets.
struct Ev {
  uint32_t np, nw, nx, nc;
};

// Leaf A against the subtree of B (not a leaf, near A): M2P for the cells
// separated from A, P2P for the leaves that are not.
template <bool WRITE>
__device__ bool tc_walk(const TcArgs &a, const TcCell &A, uint32_t b, Ev &e, uint32_t op,
                        uint32_t ow) {
  uint32_t stack[TC_STACK];
  uint32_t sp = 0;
  const TcCell B = a.cells[b];
  for (uint32_t j = 0; j < 4; ++j) {
    const uint32_t ch = child_at(B, 3 - j);
    if (ch != TC_NONE) stack[sp++] = ch;
  }
  while (sp) {
    const uint32_t c = stack[--sp];
    const TcCell C = a.cells[c];
    if (separated(a, A, C)) {
      if (WRITE) a.pool[ow + e.nw] = c;
      ++e.nw;
    } else if (C.nchild == 0) {
      if (WRITE) a.pool[op + e.np] = c;
      ++e.np;
    } else {
      if (sp + 4 > TC_STACK) return false;
      for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t ch = child_at(C, 3 - j);
        if (ch != TC_NONE) stack[sp++] = ch;
      }
    }
  }
  return true;
}

// The events of candidate u of cell c (u < 4 nnear: a child of a parent's
// near cell; beyond: the parent's coarse leaf u - 4 nnear).
template <bool WRITE>
__device__ bool tc_candidate(const TcArgs &a, uint32_t c, const TcCell &A, uint32_t u, Ev &e,
                             const uint32_t *o4) {
  const uint32_t nn = a.tab->nnear;
  const bool leaf = A.nchild == 0;
  uint32_t coarse = TC_NONE;
  if (u < 4 * nn) {
    const uint32_t o = u >> 2, b = u & 3;
    const uint32_t pb = __ldcg(&a.near[(size_t)A.parent * nn + o]);
    if (pb == TC_NONE) return true;
    const TcCell PB = a.cells[pb];
    if (PB.nchild == 0) {
      if (b != 0) return true;
      coarse = pb;  // a near leaf of the parent: seen from A as a coarse leaf
    } else {
      const uint32_t B = child_at(PB, b);
      if (B == TC_NONE) return true;
      const uint32_t e16 = a.tab->map[A.quad][o][b];
      if (!(e16 & TC_NEAR_FLAG)) {
        if (WRITE) a.m2l[(size_t)c * a.tab->sstride + e16] = B;
        return true;
      }
      if (WRITE) a.near[(size_t)c * nn + (e16 & 0xFF)] = B;
      if (!leaf) return true;
      const TcCell Bc = a.cells[B];
      if (Bc.nchild == 0) {
        if (WRITE) a.pool[o4[0] + e.np] = B;
        ++e.np;
        return true;
      }
      return tc_walk<WRITE>(a, A, B, e, o4[0], o4[1]);
    }
  } else {
    const uint32_t k = u - 4 * nn;
    coarse = __ldcg(&a.pool[__ldcg(&a.loff[(size_t)A.parent * 8 + 6]) + k]);
  }
  const TcCell L = a.cells[coarse];
  if (separated(a, A, L)) {
    if (WRITE) a.pool[o4[2] + e.nx] = coarse;
    ++e.nx;
  } else if (leaf) {
    if (WRITE) a.pool[o4[0] + e.np] = coarse;
    ++e.np;
  } else {
    if (WRITE) a.pool[o4[3] + e.nc] = coarse;
    ++e.nc;
  }
  return true;
}


__device__ __forceinline__ uint32_t warp_excl_sum(uint32_t v, uint32_t &total) {
  const unsigned lane = threadIdx.x & 31;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  total = __shfl_sync(0xffffffffu, incl, 31);
  return incl - v;
}

// One candidate's pool event: its kind (0 none, 1 P2P leaf, 2 W cell, 3 X
// leaf, 4 coarse leaf passed down, 5 a walk of the subtree of `id`) and cell.
struct Cand {
  uint32_t kind, id;
};

// The events of an evaluated candidate: counted into e, or (WRITE) written
// from the offsets o4 (p2p, w, x, coarse) plus e's counts so far.
template <bool WRITE>
__device__ __forceinline__ bool cand_events(const TcArgs &a, const TcCell &A, Cand cd, Ev &e,
                                            const uint32_t *o4) {
  switch (cd.kind) {
    case 1:
      if (WRITE) a.pool[o4[0] + e.np] = cd.id;
      ++e.np;
      return true;
    case 2:
      if (WRITE) a.pool[o4[1] + e.nw] = cd.id;
      ++e.nw;
      return true;
    case 3:
      if (WRITE) a.pool[o4[2] + e.nx] = cd.id;
      ++e.nx;
      return true;
    case 4:
      if (WRITE) a.pool[o4[3] + e.nc] = cd.id;
      ++e.nc;
      return true;
    case 5:
      return tc_walk<WRITE>(a, A, cd.id, e, o4[0], o4[1]);
    default:
      return true;
  }
}

// A cell's list state between its count and its writes (registers).
// mode 0: the root; 1: candidates kept in registers (at most LIST_KEEP
// rounds of the warp); 2: more candidates, evaluated again to write.
constexpr uint32_t LIST_KEEP = 4;

struct ListState {
  Ev tot;
  bool ok;
  uint32_t mode, ncand;
  Cand kept[LIST_KEEP];
  uint32_t off[LIST_KEEP][4];
};

// The per-kind totals of one round of events: tot += the warp's sums, off[k]
// = this lane's offset among the round's events of kind k (after tot).
__device__ __forceinline__ void round_offsets(const Ev &e, Ev &tot, uint32_t *off) {
  uint32_t t;
  if (__all_sync(0xffffffffu, (e.np | e.nw | e.nx | e.nc) < 2048u)) {
    // two counts per word: 32 lanes x 2047 stays below 2^16
    uint32_t t23;
    const uint32_t x01 = warp_excl_sum(e.np | (e.nw << 16), t);
    const uint32_t x23 = warp_excl_sum(e.nx | (e.nc << 16), t23);
    off[0] = tot.np + (x01 & 0xFFFFu); tot.np += t & 0xFFFFu;
    off[1] = tot.nw + (x01 >> 16);     tot.nw += t >> 16;
    off[2] = tot.nx + (x23 & 0xFFFFu); tot.nx += t23 & 0xFFFFu;
    off[3] = tot.nc + (x23 >> 16);     tot.nc += t23 >> 16;
  } else {
    off[0] = tot.np + warp_excl_sum(e.np, t); tot.np += t;
    off[1] = tot.nw + warp_excl_sum(e.nw, t); tot.nw += t;
    off[2] = tot.nx + warp_excl_sum(e.nx, t); tot.nx += t;
    off[3] = tot.nc + warp_excl_sum(e.nc, t); tot.nc += t;
  }
}

// Count phase of a cell that is not the root, its candidates kept: the
// candidates' loads by dependency level for all rounds at once (the parent's
// near cell or coarse leaf, its cell, then for a leaf the near cell's child);
// the M2L table and near list entries are written here.
__device__ void tc_list_count_kept(const TcArgs &a, uint32_t c, const TcCell &A, ListState &S) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nn = a.tab->nnear, ncand = S.ncand;
  const bool leaf = A.nchild == 0;
  const uint32_t rounds = (ncand + 31) / 32;  // warp-uniform, <= LIST_KEEP
  const uint32_t coff = ncand > 4 * nn ? __ldcg(&a.loff[(size_t)A.parent * 8 + 6]) : 0;
  uint32_t id[LIST_KEEP], child[LIST_KEEP];
#pragma unroll
  for (uint32_t r = 0; r < LIST_KEEP; ++r) {
    const uint32_t u = r * 32 + lane;
    id[r] = child[r] = TC_NONE;
    S.kept[r] = {0, 0};
    if (r < rounds && u < ncand)
      id[r] = u < 4 * nn ? __ldcg(&a.near[(size_t)A.parent * nn + (u >> 2)])
                         : __ldcg(&a.pool[coff + u - 4 * nn]);
  }
  TcCell P[LIST_KEEP];
#pragma unroll
  for (uint32_t r = 0; r < LIST_KEEP; ++r)
    if (r < rounds && id[r] != TC_NONE) P[r] = a.cells[id[r]];
#pragma unroll
  for (uint32_t r = 0; r < LIST_KEEP; ++r) {
    if (r >= rounds) break;
    const uint32_t u = r * 32 + lane;
    if (id[r] == TC_NONE) continue;
    bool coarse = u >= 4 * nn;
    if (!coarse) {
      const uint32_t o = u >> 2, b = u & 3;
      if (P[r].nchild == 0) {
        if (b != 0) continue;
        coarse = true;  // a near leaf of the parent: seen from A as a coarse leaf
      } else {
        const uint32_t B = child_at(P[r], b);
        if (B == TC_NONE) continue;
        const uint32_t e16 = a.tab->map[A.quad][o][b];
        if (!(e16 & TC_NEAR_FLAG)) {
          a.m2l[(size_t)c * a.tab->sstride + e16] = B;
          continue;
        }
        a.near[(size_t)c * nn + (e16 & 0xFF)] = B;
        if (leaf) child[r] = B;
        continue;
      }
    }
    if (coarse) S.kept[r] = {separated(a, A, P[r]) ? 3u : leaf ? 1u : 4u, id[r]};
  }
#pragma unroll
  for (uint32_t r = 0; r < LIST_KEEP; ++r)
    if (r < rounds && child[r] != TC_NONE)
      S.kept[r] = {a.cells[child[r]].nchild == 0 ? 1u : 5u, child[r]};
#pragma unroll
  for (uint32_t r = 0; r < LIST_KEEP; ++r) {
    if (r >= rounds) break;
    Ev e{0, 0, 0, 0};
    const uint32_t z4[4] = {0, 0, 0, 0};
    if (!cand_events<false>(a, A, S.kept[r], e, z4)) S.ok = false;
    round_offsets(e, S.tot, S.off[r]);
  }
}

// Count phase of a cell with more candidates than the lanes keep.
__device__ void tc_list_count_general(const TcArgs &a, uint32_t c, const TcCell &A, ListState &S) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t zero4[4] = {0, 0, 0, 0};
  for (uint32_t u0 = 0; u0 < S.ncand; u0 += 32) {
    const uint32_t u = u0 + lane;
    Ev e{0, 0, 0, 0};
    if (u < S.ncand && !tc_candidate<false>(a, c, A, u, e, zero4)) S.ok = false;
    uint32_t off[4];
    round_offsets(e, S.tot, off);
  }
}

// Write phase of the general case: evaluate again, each lane's events after
// those of the candidates before it.
__device__ void tc_list_write_general(const TcArgs &a, uint32_t c, const TcCell &A,
                                      const ListState &S, uint32_t *o4) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t zero4[4] = {0, 0, 0, 0};
  Ev run{0, 0, 0, 0};
  for (uint32_t u0 = 0; u0 < S.ncand; u0 += 32) {
    const uint32_t u = u0 + lane;
    Ev e{0, 0, 0, 0};
    if (u < S.ncand) tc_candidate<false>(a, c, A, u, e, zero4);
    uint32_t off[4];
    round_offsets(e, run, off);
    if (u < S.ncand) {
      Ev w{0, 0, 0, 0};
      const uint32_t w4[4] = {o4[0] + off[0], o4[1] + off[1], o4[2] + off[2], o4[3] + off[3]};
      tc_candidate<true>(a, c, A, u, w, w4);
    }
  }
}

// loff[c * 8 + ...]: 0 p2p off, 1 p2p cnt, 2 w off, 3 w cnt, 4 x off, 5 x cnt,
// 6 coarse off, 7 coarse cnt.
//
// The cells of one level, a warp per cell; the levels run as consecutive
// launches from the root down (a cell's lists read its parent's). Each warp
// counts its cell's events, the block takes one range of the pool for all of
// its warps (one atomic per block), then each warp writes. Blocks of 4
// warps, 8 an SM: the block waits at that range for its slowest warp's count.
constexpr uint32_t LIST_THREADS = 128, LIST_WARPS = LIST_THREADS / 32;
__global__ void __launch_bounds__(LIST_THREADS, 8) k_tc_lists(TcArgs a, uint32_t c0, uint32_t c1) {
  __shared__ uint32_t wsum[LIST_WARPS + 1];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t c = c0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const bool active = c < c1;  // warp-uniform
  const uint32_t nn = a.tab->nnear;
  ListState S;
  S.tot = {0, 0, 0, 0};
  S.ok = true;
  S.mode = 0;
  S.ncand = 0;
  TcCell A;
  uint32_t all = 0;
  if (active) {
    A = a.cells[c];
    for (uint32_t j = lane; j < a.tab->sstride; j += 32) a.m2l[(size_t)c * a.tab->sstride + j] = TC_NONE;
    for (uint32_t j = lane; j < nn; j += 32) a.near[(size_t)c * nn + j] = TC_NONE;
    __syncwarp();
    if (c == 0) {
      S.tot.np = A.nchild == 0 ? 1 : 0;  // the root: near itself; a P2P entry when a leaf
    } else {
      S.ncand = 4 * nn + __ldcg(&a.loff[(size_t)A.parent * 8 + 7]);
      if (S.ncand <= 32 * LIST_KEEP) {
        S.mode = 1;
        tc_list_count_kept(a, c, A, S);
      } else {
        S.mode = 2;
        tc_list_count_general(a, c, A, S);
      }
      S.ok = __all_sync(0xffffffffu, S.ok);
    }
    all = S.tot.np + S.tot.nw + S.tot.nx + S.tot.nc;
  }
  if (lane == 0) wsum[warp] = all;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (uint32_t w = 0; w < LIST_WARPS; ++w) {
      const uint32_t t = wsum[w];
      wsum[w] = run;
      run += t;
    }
    wsum[LIST_WARPS] = run ? atomicAdd(&a.info[TI_POOL_P2P], run) : 0;
  }
  __syncthreads();
  if (!active) return;
  const uint32_t base = wsum[LIST_WARPS] + wsum[warp];
  const uint32_t o4[4] = {base, base + S.tot.np, base + S.tot.np + S.tot.nw,
                          base + S.tot.np + S.tot.nw + S.tot.nx};
  uint32_t *lo = a.loff + (size_t)c * 8;
  if (!S.ok || (size_t)base + all > a.pool_cap) {
    if (lane == 0) {
      atomicOr(&a.info[TI_OVF], S.ok ? 1u : 2u);
      lo[0] = lo[2] = lo[4] = lo[6] = 0;
      lo[1] = lo[3] = lo[5] = lo[7] = 0;
    }
    return;
  }
  if (lane == 0) {
    lo[0] = o4[0]; lo[1] = S.tot.np;
    lo[2] = o4[1]; lo[3] = S.tot.nw;
    lo[4] = o4[2]; lo[5] = S.tot.nx;
    lo[6] = o4[3]; lo[7] = S.tot.nc;
  }
  if (S.mode == 0) {
    if (lane == 0) {
      uint32_t self = 0;
      for (uint32_t o = 0; o < nn; ++o)
        if (a.tab->near_dx[o] == 0 && a.tab->near_dy[o] == 0) self = o;
      a.near[self] = 0;
      if (S.tot.np) a.pool[base] = 0;
    }
  } else if (S.mode == 1) {
#pragma unroll
    for (uint32_t r = 0; r < LIST_KEEP; ++r) {
      if (S.kept[r].kind) {
        const uint32_t w4[4] = {o4[0] + S.off[r][0], o4[1] + S.off[r][1], o4[2] + S.off[r][2],
                                o4[3] + S.off[r][3]};
        Ev w{0, 0, 0, 0};
        cand_events<true>(a, A, S.kept[r], w, w4);
      }
    }
  } else {
    uint32_t o[4] = {o4[0], o4[1], o4[2], o4[3]};
    tc_list_write_general(a, c, A, S, o);
  }
}

// ---- M2L on the tensor cores -------------------------------------------------------------

// M2L CTA: 256 gathering threads (two per target row: the bf16 hi and the lo
// half of the row) and one warp whose first lane only issues the MMAs.
constexpr uint32_t M2L_STAGES = 3;
constexpr uint32_t M2L_AHEAD = 2;  // slots of copies in flight per gathering thread
static_assert(M2L_AHEAD <= M2L_STAGES, "a stage is landed before it is reused");
constexpr uint32_t M2L_PRODUCERS = 2 * TC_TILE;
constexpr uint32_t M2L_THREADS = M2L_PRODUCERS + 32;

struct M2lSmem {
  unsigned char a[M2L_STAGES][2][TC_TILE * TC_KN * 2];  // [stage][hi, lo] 128 x 32 bf16
  unsigned char b[M2L_STAGES][2][TC_KN * TC_KN * 2];    // [stage][hi, lo] 32 x 32 bf16
  uint64_t full[M2L_STAGES], empty[M2L_STAGES], done;
  uint32_t tmem;
  uint32_t tgt[TC_TILE];
  uint32_t err;
};

// Budget of a wait on a barrier the tile's own threads complete.
constexpr uint64_t TC_WAIT_NS = 50ull * 1000 * 1000;

__global__ void __launch_bounds__(M2L_THREADS) k_tc_m2l(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char tc_m2l_smem[];
  M2lSmem &S = *reinterpret_cast<M2lSmem *>(tc_m2l_smem);
  volatile uint32_t *abort = &S.err;
  const uint32_t t = threadIdx.x, warp = t >> 5;
  // this CTA's tile: group g, rows base .. base + 127
  uint32_t g = 0, tile = blockIdx.x, cnt = 0;
  for (; g < 4; ++g) {
    cnt = __ldcg(&a.info[TI_GROUP + g]);
    const uint32_t nt = (cnt + TC_TILE - 1) / TC_TILE;
    if (tile < nt) break;
    tile -= nt;
  }
  if (g == 4) return;  // no tile: nothing allocated yet, nothing to free
  const uint32_t base = tile * TC_TILE;
  const uint32_t nslot = a.tab->nslot[g], sstride = a.tab->sstride;
  if (t < TC_TILE) S.tgt[t] = base + t < cnt ? a.groups[(size_t)g * a.ccap + base + t] : TC_NONE;
  if (t == 0) {
    for (uint32_t s = 0; s < M2L_STAGES; ++s) {
      tc::mbar_init(&S.full[s], M2L_PRODUCERS);
      tc::mbar_init(&S.empty[s], 1);
    }
    tc::mbar_init(&S.done, 1);
    S.err = 0;
    tc::mbar_init_fence();
  }
  __syncwarp();
  if (warp == 0) {
    tc::tmem_alloc(&S.tmem, 32);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = S.tmem;
  uint32_t issued = 0;  // the MMA lane: MMAs issued
  if (t < M2L_PRODUCERS) {
    // a row's half: 4 chunks of 16 bytes (hi for t < 128, lo otherwise)
    const uint32_t r = t & (TC_TILE - 1), h = t >> 7;
    const uint32_t my = S.tgt[r];
    auto source = [&](uint32_t j) -> uint32_t {
      return (my != TC_NONE && j < nslot) ? __ldcg(&a.m2l[(size_t)my * sstride + j]) : TC_NONE;
    };
    // the copies of slot j into stage s: this thread's 4 chunks of the row
    // (zeros when the slot has no source) and 16 bytes of the operator
    const uint32_t a_dst = tc::smem_addr(S.a[0][h]), b_dst = tc::smem_addr(S.b[0][0]) + t * 16;
    auto copy = [&](uint32_t j, uint32_t s, uint32_t src) {
      const char *m = reinterpret_cast<const char *>(a.mbf) +
                      (src != TC_NONE ? (size_t)src * 128 + h * 64 : 0);
      const uint32_t bytes = src != TC_NONE ? 16u : 0u;
#pragma unroll
      for (uint32_t c = 0; c < 4; ++c)
        tc::cp_async16(a_dst + s * sizeof(S.a[0]) + tc::tile_offset(r, c, TC_TILE), m + c * 16,
                       bytes);
      const char *w = reinterpret_cast<const char *>(a.wops) +
                      (size_t)a.tab->slot_class[g][j] * 4096 + t * 16;
      tc::cp_async16(b_dst + s * sizeof(S.b[0]), w, 16u);
      tc::cp_async_commit();
    };
    // slot j's stage is full once this thread's copies of it have landed:
    // wait for them, make them visible to the tensor core, arrive
    auto land = [&](uint32_t j, bool all) {
      if (all) tc::cp_async_wait<0>();
      else tc::cp_async_wait<M2L_AHEAD - 1>();
      tc::fence_proxy_async();
      tc::mbar_arrive(&S.full[j % M2L_STAGES]);
    };
    uint32_t src = source(0), landed = 0;
    for (uint32_t j = 0; j < nslot; ++j) {
      const uint32_t s = j % M2L_STAGES, use = j / M2L_STAGES;
      const uint32_t next = source(j + 1);
      // the stage is free once the MMAs that read it (slot j - STAGES) are done
      if (use > 0 && !tc::mbar_wait(&S.empty[s], (use - 1) & 1, abort, TC_WAIT_NS)) break;
      copy(j, s, src);
      if (j + 1 >= M2L_AHEAD) land(landed++, false);
      src = next;
    }
    // the slots still in flight (also after a wait that gave up: every copy
    // lands before the CTA can exit)
    tc::cp_async_wait<0>();
    if (!*abort)
      while (landed < nslot) land(landed++, true);
  } else if (t == M2L_PRODUCERS) {
    const uint32_t idesc = tc::idesc_bf16_f32(TC_TILE, TC_KN);
    const uint32_t alb = (TC_TILE / 8) * 128, blb = (TC_KN / 8) * 128;
    for (uint32_t j = 0; j < nslot; ++j) {
      const uint32_t s = j % M2L_STAGES, use = j / M2L_STAGES;
      if (!tc::mbar_wait(&S.full[s], use & 1, abort, TC_WAIT_NS)) break;
      tc::fence_after_sync();
      const uint32_t a_hi = tc::smem_addr(S.a[s][0]), a_lo = tc::smem_addr(S.a[s][1]);
      const uint32_t b_hi = tc::smem_addr(S.b[s][0]), b_lo = tc::smem_addr(S.b[s][1]);
#pragma unroll
      for (uint32_t ks = 0; ks < 2; ++ks) {  // K = 32 as two MMAs of K = 16
        const uint32_t ao = ks * 2 * alb, bo = ks * 2 * blb;
        const uint64_t dah = tc::smem_desc(a_hi + ao, alb, 128);
        const uint64_t dal = tc::smem_desc(a_lo + ao, alb, 128);
        const uint64_t dbh = tc::smem_desc(b_hi + bo, blb, 128);
        const uint64_t dbl = tc::smem_desc(b_lo + bo, blb, 128);
        tc::mma_bf16(tmem, dah, dbh, idesc, (j | ks) ? 1u : 0u);
        tc::mma_bf16(tmem, dah, dbl, idesc, 1u);
        tc::mma_bf16(tmem, dal, dbh, idesc, 1u);
      }
      issued += 6;
      tc::commit(&S.empty[s]);
    }
    // every MMA issued so far completes before the accumulator is read and
    // the TMEM freed (also after a wait that gave up)
    if (issued) tc::commit(&S.done);
  }
  const bool any = __syncthreads_or(issued > 0);
  bool done_ok = true;
  if (any) {
    // a fresh budget: this wait only needs the MMAs already issued
    uint32_t no_abort = 0;
    done_ok = tc::mbar_wait(&S.done, 0, &no_abort, TC_WAIT_NS);
  }
  tc::fence_after_sync();
  const bool all_done = __syncthreads_and(done_ok);
  const bool good = any && S.err == 0 && all_done;
  if (warp < 4) {
    const uint32_t my = S.tgt[t];
    if (good) {
      float v[32];
      tc::tmem_ld32(tmem + ((warp * 32u) << 16), v);
      if (my != TC_NONE) {
        float *L = a.lco + (size_t)my * TC_KN;
#pragma unroll
        for (uint32_t k = 0; k < 32; ++k)
          if (k < 2 * a.q) L[k] = v[k];
      }
    } else if (my != TC_NONE) {
      float *L = a.lco + (size_t)my * TC_KN;
      for (uint32_t k = 0; k < 2 * a.q; ++k) L[k] = 0;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  // (after a done-wait that ran out an MMA may still write the accumulator:
  // the columns are then left allocated rather than freed under it)
  if (warp == 0 && all_done) tc::tmem_dealloc(tmem, 32);
  if (t == 0 && (S.err || !all_done) && nslot) {
    atomicOr(&a.info[TI_ERR], 1u);
    if (a.status) atomicOr(a.status, ST_WAIT_TIMEOUT);
  }
}

// ---- P2L (coarse leaves into local expansions, FP32) ------------------------------------------

// The source leaf and point of batch index idx: the leaves' counts are held
// one per lane (running count `incl`, `before` it, first point `first`, ne
// lanes in use); returns the point.
__device__ __forceinline__ uint32_t batch_point(uint32_t idx, uint32_t ne, uint32_t incl,
                                                uint32_t before, uint32_t first) {
  uint32_t j = 0;
#pragma unroll
  for (uint32_t step = 16; step; step >>= 1) {
    const uint32_t v = __shfl_sync(0xffffffffu, incl, j + step - 1);
    if (j + step - 1 < ne && v <= idx) j += step;
  }
  const uint32_t f = __shfl_sync(0xffffffffu, first, j & 31);
  const uint32_t b0 = __shfl_sync(0xffffffffu, before, j & 31);
  return f + (idx - b0);
}

// A warp per cell with an X list (coarse leaves seen from it): the points of
// the listed leaves spread over the lanes; each lane adds its points' terms
//     L'_l += (-1)^l s_j / z^(l+1),   z = (c_A - u_j) / s_A,
// (z from an FP64 difference, the series in FP32), then the lanes' sums are
// reduced and added to the cell's row. Q = q.
template <int Q>
__global__ void __launch_bounds__(TC_THREADS) k_tc_p2l(TcArgs a) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = gw; c < a.ncells; c += nwarps) {
    const uint32_t nx = a.loff[(size_t)c * 8 + 5];
    if (!nx) continue;
    const uint32_t ox = a.loff[(size_t)c * 8 + 4];
    const TcCell A = a.cells[c];
    double ax, ay;
    cell_centre(A, ax, ay);
    const double inv_s = pow2((int)A.level);
    float sr[Q], si[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) sr[l] = si[l] = 0.f;
    for (uint32_t eb = 0; eb < nx; eb += 32) {
      const uint32_t ne = min(32u, nx - eb);
      uint32_t first = 0, cnt = 0;
      if (lane < ne) {
        const TcCell L = a.cells[a.pool[ox + eb + lane]];
        first = L.first;
        cnt = L.count;
      }
      uint32_t total;
      const uint32_t before = warp_excl_sum(cnt, total);
      const uint32_t incl = before + cnt;
      for (uint32_t i0 = 0; i0 < total; i0 += 32) {
        const uint32_t idx = i0 + lane;
        const uint32_t k = batch_point(idx, ne, incl, before, first);
        if (idx >= total) continue;
        const float sv = (float)__ldg(&a.ps[k]);
        const float zr = (float)((ax - __ldg(&a.ux[k])) * inv_s);
        const float zi = (float)((ay - __ldg(&a.uy[k])) * inv_s);
        const float d2 = zr * zr + zi * zi;
        const float ir = __fdividef(zr, d2), ii = -__fdividef(zi, d2);  // 1 / z
        float pr = sv * ir, pi = sv * ii;
#pragma unroll
        for (int l = 0; l < Q; ++l) {
          if (l & 1) {
            sr[l] -= pr;
            si[l] -= pi;
          } else {
            sr[l] += pr;
            si[l] += pi;
          }
          const float nr = pr * ir - pi * ii;
          pi = pr * ii + pi * ir;
          pr = nr;
        }
      }
    }
#pragma unroll
    for (int l = 0; l < Q; ++l)
      for (int o = 16; o > 0; o >>= 1) {
        sr[l] += __shfl_xor_sync(0xffffffffu, sr[l], o);
        si[l] += __shfl_xor_sync(0xffffffffu, si[l], o);
      }
    float *Lc = a.lco + (size_t)c * TC_KN;
#pragma unroll
    for (int l = 0; l < Q; ++l)
      if (lane == (unsigned)l) {
        Lc[l] += sr[l];
        Lc[Q + l] += si[l];
      }
  }
}

// ---- downward: each leaf gathers its ancestors' local expansions ---------------------------------

__host__ __device__ constexpr float binomf(int n, int k) {
  float r = 1.f;
  for (int i = 1; i <= k; ++i) r = r * (float)(n - k + i) / (float)i;
  return r;
}

// A thread per leaf: L'^leaf += sum over its ancestors P of the ancestor's own
// M2L and P2L part shifted to the leaf's centre,
//     L'^leaf_m += r^(m+1) sum_{l>=m} C(l, m) D^(l-m) L'^P_l,
// D = (c_leaf - c_P) / s_P and r = s_leaf / s_P = 2^-d (the level-by-level
// L2L of fmm.zig:821-850 composed along the path; D from the integer
// coordinates, exact in FP32). The leaf's row is updated in place (no other
// thread reads a leaf's row); Q >= q bounds the unrolled loops.
template <int Q>
__global__ void __launch_bounds__(TC_THREADS) k_tc_down(TcArgs a) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= __ldcg(&a.info[TI_LEAVES])) return;
  const uint32_t q = a.q;
  const uint32_t c = a.leaves[e];
  const TcCell C = a.cells[c];
  float lr[Q], li[Q];
  float *L = a.lco + (size_t)c * TC_KN;
#pragma unroll
  for (int l = 0; l < Q; ++l) {
    lr[l] = l < (int)q ? L[l] : 0.f;
    li[l] = l < (int)q ? L[q + l] : 0.f;
  }
  uint32_t p = C.parent;
  for (uint32_t guard = 0; p != TC_NONE && guard < 32; ++guard) {
    const TcCell P = a.cells[p];
    const float *A = a.lco + (size_t)p * TC_KN;
    float ar[Q], ai[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
      ar[l] = l < (int)q ? __ldcg(&A[l]) : 0.f;
      ai[l] = l < (int)q ? __ldcg(&A[q + l]) : 0.f;
    }
    const int d = (int)C.level - (int)P.level;
    const uint32_t mask = (1u << d) - 1u;
    const float dx = ((float)(C.ix & mask) + 0.5f) * pow2f(-d) - 0.5f;
    const float dy = ((float)(C.iy & mask) + 0.5f) * pow2f(-d) - 0.5f;
    float pr[Q], pi[Q];  // D^j
    pr[0] = 1.f;
    pi[0] = 0.f;
#pragma unroll
    for (int j = 1; j < Q; ++j) {
      pr[j] = pr[j - 1] * dx - pi[j - 1] * dy;
      pi[j] = pr[j - 1] * dy + pi[j - 1] * dx;
    }
#pragma unroll
    for (int m = 0; m < Q; ++m) {
      float sr = 0.f, si = 0.f;
#pragma unroll
      for (int j = 0; m + j < Q; ++j) {
        const float b = binomf(m + j, m);
        const float tr = ar[m + j] * b, ti = ai[m + j] * b;
        sr += tr * pr[j] - ti * pi[j];
        si += tr * pi[j] + ti * pr[j];
      }
      const float sc = (m + 1) * d <= 126 ? pow2f(-(m + 1) * d) : 0.f;
      lr[m] += sr * sc;
      li[m] += si * sc;
    }
    p = P.parent;
  }
#pragma unroll
  for (int l = 0; l < Q; ++l)
    if (l < (int)q) {
      L[l] = lr[l];
      L[q + l] = li[l];
    }
}

template <int Q>
void launch_p2l_q(const TcArgs &g, unsigned blocks, cudaStream_t st) {
  D3_LAUNCH(k_tc_p2l<Q>, blocks, TC_THREADS, 0, st)(g);
}

void launch_p2l(const TcArgs &g, cudaStream_t st) {
  const unsigned blocks = blocks_for((size_t)g.ncells * 32, TC_THREADS);
  if (!blocks) return;
  switch (g.q) {
    case 2: launch_p2l_q<2>(g, blocks, st); break;
    case 3: launch_p2l_q<3>(g, blocks, st); break;
    case 4: launch_p2l_q<4>(g, blocks, st); break;
    case 5: launch_p2l_q<5>(g, blocks, st); break;
    case 6: launch_p2l_q<6>(g, blocks, st); break;
    case 7: launch_p2l_q<7>(g, blocks, st); break;
    case 8: launch_p2l_q<8>(g, blocks, st); break;
    case 9: launch_p2l_q<9>(g, blocks, st); break;
    case 10: launch_p2l_q<10>(g, blocks, st); break;
    case 11: launch_p2l_q<11>(g, blocks, st); break;
    case 12: launch_p2l_q<12>(g, blocks, st); break;
    case 13: launch_p2l_q<13>(g, blocks, st); break;
    case 14: launch_p2l_q<14>(g, blocks, st); break;
    case 15: launch_p2l_q<15>(g, blocks, st); break;
    default: launch_p2l_q<16>(g, blocks, st); break;
  }
}

void launch_down(const TcArgs &g, uint32_t nleaf, cudaStream_t st) {
  const unsigned blocks = blocks_for(nleaf, TC_THREADS);
  if (!blocks) return;
  if (g.q <= 5) D3_LAUNCH(k_tc_down<5>, blocks, TC_THREADS, 0, st)(g);
  else if (g.q <= 9) D3_LAUNCH(k_tc_down<9>, blocks, TC_THREADS, 0, st)(g);
  else if (g.q <= 13) D3_LAUNCH(k_tc_down<13>, blocks, TC_THREADS, 0, st)(g);
  else D3_LAUNCH(k_tc_down<16>, blocks, TC_THREADS, 0, st)(g);
}

// Leaf features of the learned correction, from the leaf's final local
// expansion and its points: L'_1 .. L'_4 over sc = |(L'_0 .. L'_4)| (8
// reals), level / 16, count / 32, and the points' mean offset from the centre
// in cell sides (2). Row of 16 floats per cell: features, L'_0 (2), sc, and
// the cell index (as float bits) for leaves, -1 in column 15 otherwise.
__device__ void feature_row(const TcArgs &a, uint32_t c, const TcCell &C, const float *L, float mx,
                            float my) {
  const uint32_t q = a.q;
  float *row = a.feat + (size_t)c * 16;
  const uint32_t lmax = q - 1 < 4 ? q - 1 : 4;
  float s2 = 0;
  for (uint32_t l = 0; l <= lmax; ++l) s2 += L[l] * L[l] + L[q + l] * L[q + l];
  const float sc = sqrtf(s2) + 1e-30f;
  for (uint32_t l = 1; l <= 4; ++l) {
    row[2 * (l - 1)] = l <= lmax ? L[l] / sc : 0.f;
    row[2 * (l - 1) + 1] = l <= lmax ? L[q + l] / sc : 0.f;
  }
  row[8] = C.level / 16.f;
  row[9] = C.count / 32.f;
  row[10] = mx / C.count;
  row[11] = my / C.count;
  row[12] = L[0];
  row[13] = L[q];
  row[14] = sc;
  row[15] = __uint_as_float(c);
}

__global__ void __launch_bounds__(TC_THREADS) k_tc_features(TcArgs a) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nleaf = __ldcg(&a.info[TI_LEAVES]);
  for (uint32_t e = gw; e < nleaf; e += nwarps) {
    const uint32_t c = a.leaves[e];
    const TcCell C = a.cells[c];
    double cx, cy;
    cell_centre(C, cx, cy);
    const double inv_s = pow2((int)C.level);
    float mx = 0, my = 0;
    for (uint32_t k = C.first + lane; k < C.first + C.count; k += 32) {
      mx += (float)((a.ux[k] - cx) * inv_s);
      my += (float)((a.uy[k] - cy) * inv_s);
    }
    for (int o = 16; o > 0; o >>= 1) {
      mx += __shfl_xor_sync(0xffffffffu, mx, o);
      my += __shfl_xor_sync(0xffffffffu, my, o);
    }
    if (lane == 0) feature_row(a, c, C, a.lco + (size_t)c * TC_KN, mx, my);
  }
}

// The learned form's inputs, packed for the network: x[k] = features of leaf
// leaves[k].
__global__ void k_tc_pack(TcArgs a) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= __ldcg(&a.info[TI_LEAVES])) return;
  const float *row = a.feat + (size_t)a.leaves[k] * 16;
  for (int j = 0; j < 12; ++j) a.mlp_x[(size_t)k * 12 + j] = row[j];
}

// ---- P2P (FP32 with an FP64 origin shift) ----------------------------------------------------------

constexpr uint32_t P2P_STAGE = 256;  // staged source points per warp
// The near field's blocks: 4 warps, 8 blocks an SM (64 registers a thread).
// A warp takes one leaf, and a block frees its slot when its slowest warp
// ends, so small blocks keep more warps busy under uneven leaf sizes.
constexpr uint32_t NEAR_THREADS = 128, NEAR_WARPS = NEAR_THREADS / 32;

// One point pair of the near field (d3's pair formula, the distanceMin clamp
// and the hashed jiggle of hash.zig for exact zero deltas; the self pair adds
// nothing). The careful form, for batches that hold a coincident pair.
__device__ __forceinline__ void tc_pair(const float4 sv, float xi, float yi, uint32_t ti, uint32_t gi,
                                        float dmin2, uint64_t seed, const uint32_t *perm, float &ax,
                                        float &ay) {
  float dx = sv.x - xi, dy = sv.y - yi;
  float l = dx * dx + dy * dy;
  if (dx == 0.f || dy == 0.f) {
    const uint32_t tj = __float_as_uint(sv.w);
    if (tj == ti) return;
    const uint32_t gj = perm[tj];
    if (dx == 0.f) {
      dx = (float)hash_jiggle(seed, gi, gj, 0);
      l += dx * dx;
    }
    if (dy == 0.f) {
      dy = (float)hash_jiggle(seed, gi, gj, 1);
      l += dy * dy;
    }
  }
  if (l < dmin2) l = sqrtf(dmin2 * l);
  const float w = __fdividef(sv.z, l);
  ax += dx * w;
  ay += dy * w;
}

// The same pair without the jiggle, for leaves with no coincident points.
// w = s / l, or s / sqrt(dmin2 l) inside distanceMin, is s * rsqrt(y) with
// y = l max(l, dmin2) (one MUFU op); l is floored at 1e-18 there (distances
// under 1e-9, below FP32's resolution of the leaf-local coordinates) so the
// self pair adds 0 * w with w finite. A single zero delta keeps its zero
// here, where d3 would jiggle it by ~1e-6: the change to the kick is ~1e-6
// of that one pair's term.
// It takes two sources at once in sm_100's packed FP32 pairs (FADD2, FMUL2,
// FFMA2, each half rounded as its scalar op): P = (x_a, x_b, y_a, y_b) and
// S = (s_a, s_b) of sources a and b, (nx, ny) the target's negated
// coordinates in both halves, d2 = dmin2 in both. y = max(l^2, l dmin2, fl)
// with fl = 1e-18 max(1e-18, dmin2) equals lf max(lf, dmin2) with
// lf = max(l, 1e-18) bit for bit (the rounding is monotonic). ax, ay: the a
// and b sources' sums.
__device__ __forceinline__ void tc_pair2(const float4 P, const float2 S, const float2 nx,
                                         const float2 ny, const float2 d2, float fl, float2 &ax,
                                         float2 &ay) {
  const float2 dx = __fadd2_rn(make_float2(P.x, P.y), nx);
  const float2 dy = __fadd2_rn(make_float2(P.z, P.w), ny);
  const float2 l = __ffma2_rn(dx, dx, __fmul2_rn(dy, dy));
  const float2 ll = __fmul2_rn(l, l), ld = __fmul2_rn(l, d2);
  const float2 r = make_float2(rsqrtf(fmaxf(fmaxf(ll.x, ld.x), fl)),
                               rsqrtf(fmaxf(fmaxf(ll.y, ld.y), fl)));
  const float2 w = __fmul2_rn(S, r);
  ax = __ffma2_rn(dx, w, ax);
  ay = __ffma2_rn(dy, w, ay);
}

// Staged source k in the paired layout (slot 2i: x, x', y, y' of sources 2i
// and 2i + 1; slot 2i + 1: s, s', index, index'), as (x, y, s, index).
__device__ __forceinline__ float4 staged_point(const float4 *sg, uint32_t k) {
  const float *p = reinterpret_cast<const float *>(sg + (k & ~1u));
  const uint32_t h = k & 1u;
  return make_float4(p[h], p[2 + h], p[4 + h], p[6 + h]);
}

// The far field at target point k of leaf C: L2P of the leaf's final local
// expansion (Lsh: 2q floats, L'_0 possibly corrected) by Horner in FP32 (the
// L2P of downwardCell, fmm.zig:851-886),
//     phi = (1/s) sum_l L'_l w^l,   w = (u - c) / s,
// and M2P from each cell of the leaf's W list (z from an FP64 shift, the
// series in FP32; the adaptive list has no reference counterpart),
//     phi += (1/s_W) sum_k M'_k / z^(k+1),   z = (u - c_W) / s_W.
// Returns the kick's far part in world units; (wr, wi) = w for the feature row.
__device__ __forceinline__ float2 tc_far(const TcArgs &a, uint32_t k, double cx, double cy,
                                         double inv_s, const float *Lsh, float c0r, float c0i,
                                         uint32_t nw, uint32_t ow, float &wr, float &wi) {
  const uint32_t q = a.q;
  const double ux = a.ux[k], uy = a.uy[k];
  wr = (float)((ux - cx) * inv_s);
  wi = (float)((uy - cy) * inv_s);
  // L'_0 + (c0r, c0i): the learned form's correction (zero otherwise)
  float ar = Lsh[q - 1] + (q == 1 ? c0r : 0.f), ai = Lsh[2 * q - 1] + (q == 1 ? c0i : 0.f);
  for (int l = (int)q - 2; l >= 0; --l) {
    const float nr = ar * wr - ai * wi + Lsh[l] + (l == 0 ? c0r : 0.f);
    ai = ar * wi + ai * wr + Lsh[q + l] + (l == 0 ? c0i : 0.f);
    ar = nr;
  }
  double gr = (double)ar * inv_s, gi = (double)ai * inv_s;
  for (uint32_t e = 0; e < nw; ++e) {
    const uint32_t cc = a.pool[ow + e];
    const TcCell W = a.cells[cc];
    double wx, wy;
    cell_centre(W, wx, wy);
    const double winv = pow2((int)W.level);
    // z in FP64 (the shift), the series in FP32: |1/z| < 1 for a separated cell
    const float zr = (float)((ux - wx) * winv), zi = (float)((uy - wy) * winv);
    const float d2 = zr * zr + zi * zi;
    const float ir = __fdividef(zr, d2), ii = -__fdividef(zi, d2);
    const double *mc = a.mco + (size_t)cc * 2 * q;
    float pr = ir, pi = ii, sr = 0, si = 0;
    for (uint32_t kk = 0; kk < q; ++kk) {
      const float mr = (float)mc[kk], mi = (float)mc[q + kk];
      sr += mr * pr - mi * pi;
      si += mr * pi + mi * pr;
      const float nr = pr * ir - pi * ii;
      pi = pr * ii + pi * ir;
      pr = nr;
    }
    gr += (double)sr * winv;
    gi += (double)si * winv;
  }
  return make_float2((float)(-gr * a.inv_w), (float)(gi * a.inv_w));
}

// A warp per leaf (grid-stride over the leaf list): the near field of its
// points into nearbuf (FP32 sums) and each point's leaf into leafidx. It
// reads only the lists and the points, so it runs beside M2L, P2L and the
// downward pass; k_tc_far adds the far field.
// The leaf's targets take a lane each, two per lane: a leaf of W points
// splits the warp into 32 / ceil(W / 2) lane groups that hold the same
// targets and take alternate sources, their sums added at the end in group
// order. The source leaves' points are staged in shared memory relative to
// the target leaf's first point (the shift in FP64): up to 32 source leaves
// at a time, their points spread over the lanes so every load of a batch is
// in flight at once. They are staged in pairs (staged_point), so that the
// pair loop takes two sources per step in packed FP32 (tc_pair2), each half
// of a target's sums adding every other source; there the lane groups take
// alternate source pairs.
__global__ void __launch_bounds__(NEAR_THREADS, 8) k_tc_near(TcArgs a, float2 *nearbuf) {
  __shared__ float4 stage[NEAR_WARPS][P2P_STAGE];
  __shared__ float4 red[NEAR_WARPS][32];
  const unsigned lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const float2 d2 = make_float2(a.dmin2f, a.dmin2f);
  const float fl = 1e-18f * fmaxf(1e-18f, a.dmin2f);
  const uint32_t nleaf = __ldcg(&a.info[TI_LEAVES]);
  float4 *sg = stage[wl];
  for (uint32_t e0 = gw; e0 < nleaf; e0 += nwarps) {
    const uint32_t c = a.leaves[e0];
    const TcCell A = a.cells[c];
    const uint32_t np = a.loff[(size_t)c * 8 + 1], op = a.loff[(size_t)c * 8];
    // lane groups: a lane holds two targets (slots gl and W + gl of the
    // round), W = ceil(count / 2) lanes a group, G = 32 / W groups (lanes
    // past G W idle); a leaf of more than 64 points takes several rounds
    const uint32_t W = A.count <= 64 ? (A.count + 1) / 2 : 32u, G = 32u / W;
    const uint32_t grp = lane / W, gl = lane % W;
    const bool in = grp < G;
    const double ox = a.px[A.first], oy = a.py[A.first];
    // Points at one position share a (sorted, 16-level) key, so they sit in
    // one leaf next to each other: a leaf with two equal neighbouring keys,
    // or that spans several rounds of targets, takes the careful pair. (Two
    // points closer than FP32 resolves in the leaf's local coordinates but
    // with different keys add nothing to each other here.)
    bool careful = A.count > 32;
    if (!careful) {
      const bool dup = lane + 1 < A.count &&
                       (uint32_t)a.keys[A.first + lane] == (uint32_t)a.keys[A.first + lane + 1];
      careful = __any_sync(0xffffffffu, dup);
    }
    const uint32_t end = A.first + A.count;
    for (uint32_t tb = A.first; tb < end; tb += 2 * W) {
      const uint32_t t0 = tb + gl, t1 = tb + W + gl;
      const bool act0 = in && t0 < end, act1 = in && t1 < end;
      const float x0 = act0 ? (float)(a.px[t0] - ox) : 0.f, y0 = act0 ? (float)(a.py[t0] - oy) : 0.f;
      const float x1 = act1 ? (float)(a.px[t1] - ox) : 0.f, y1 = act1 ? (float)(a.py[t1] - oy) : 0.f;
      const float2 nx0 = make_float2(-x0, -x0), ny0 = make_float2(-y0, -y0);
      const float2 nx1 = make_float2(-x1, -x1), ny1 = make_float2(-y1, -y1);
      // targets 0 and 1; the halves sum the even and the odd sources
      float2 ax0 = make_float2(0.f, 0.f), ay0 = ax0, ax1 = ax0, ay1 = ax0;
      for (uint32_t eb = 0; eb < np; eb += 32) {
        // this batch's source leaves: lane j holds leaf j's first point and
        // the running count before it
        const uint32_t ne = min(32u, np - eb);
        uint32_t first = 0, cnt = 0;
        if (lane < ne) {
          const TcCell B = a.cells[a.pool[op + eb + lane]];
          first = B.first;
          cnt = B.count;
        }
        uint32_t total;
        const uint32_t before = warp_excl_sum(cnt, total);
        const uint32_t incl = before + cnt;
        for (uint32_t base = 0; base < total; base += P2P_STAGE) {
          const uint32_t kn = min(P2P_STAGE, total - base);
          __syncwarp();
          // the paired layout (staged_point): lanes 2i and 2i + 1 swap halves
          // and write slots 2i and 2i + 1; a source past kn is a zero (x, y,
          // s all 0) so an odd last pair adds nothing
          const uint32_t rounds = (kn + 31) / 32;
          const bool odd = lane & 1u;
#pragma unroll 4
          for (uint32_t r = 0; r < rounds; ++r) {
            const uint32_t idx = base + r * 32 + lane;
            const uint32_t sj = batch_point(idx, ne, incl, before, first);
            float px = 0.f, py = 0.f, ps = 0.f;
            if (idx < base + kn) {
              px = (float)(__ldg(&a.px[sj]) - ox);
              py = (float)(__ldg(&a.py[sj]) - oy);
              ps = (float)__ldg(&a.ps[sj]);
            }
            const float u = __shfl_xor_sync(0xffffffffu, odd ? px : ps, 1);
            const float v = __shfl_xor_sync(0xffffffffu, odd ? py : __uint_as_float(sj), 1);
            sg[r * 32 + lane] = odd ? make_float4(u, ps, v, __uint_as_float(sj))
                                    : make_float4(px, u, py, v);
          }
          __syncwarp();
          if (!careful) {
            const uint32_t kp_end = (kn + 1) / 2;
#pragma unroll 4
            for (uint32_t kp = in ? grp : kp_end; kp < kp_end; kp += G) {
              const float4 P = sg[2 * kp];
              const float2 S = *reinterpret_cast<const float2 *>(&sg[2 * kp + 1]);
              tc_pair2(P, S, nx0, ny0, d2, fl, ax0, ay0);
              tc_pair2(P, S, nx1, ny1, d2, fl, ax1, ay1);
            }
          } else {
            const uint64_t seed = (uint64_t)__double_as_longlong(*a.seed);
            const uint32_t g0 = act0 ? a.perm[t0] : 0, g1 = act1 ? a.perm[t1] : 0;
            for (uint32_t k = in ? grp : kn; k < kn; k += G) {
              const float4 sv = staged_point(sg, k);
              tc_pair(sv, -nx0.x, -ny0.x, t0, g0, d2.x, seed, a.perm, ax0.x, ay0.x);
              tc_pair(sv, -nx1.x, -ny1.x, t1, g1, d2.x, seed, a.perm, ax1.x, ay1.x);
            }
          }
        }
      }
      // the groups' sums, in group order
      __syncwarp();
      red[wl][lane] = make_float4(ax0.x + ax0.y, ay0.x + ay0.y, ax1.x + ax1.y, ay1.x + ay1.y);
      __syncwarp();
      if (grp == 0) {
        float v0x = 0, v0y = 0, v1x = 0, v1y = 0;
        for (uint32_t g2 = 0; g2 < G; ++g2) {
          const float4 v = red[wl][g2 * W + gl];
          v0x += v.x;
          v0y += v.y;
          v1x += v.z;
          v1y += v.w;
        }
        if (act0) {
          nearbuf[t0] = make_float2(v0x, v0y);
          a.leafidx[t0] = e0;
        }
        if (act1) {
          nearbuf[t1] = make_float2(v1x, v1y);
          a.leafidx[t1] = e0;
        }
      }
    }
  }
}

// A thread per point: the far field of its leaf (tc_far: L2P of the leaf's
// final local expansion, M2P of its W list) plus its near field from
// nearbuf, v += near + far in FP64, or the kick to `kick`. `corrected`: the
// learned form's network output is added to the leaf's L'_0 (sc * y /
// LEARN_TARGET_SCALE). The learned form's fallback reuses the near field of
// its order-4 pass here (it does not depend on the order).
__global__ void __launch_bounds__(TC_THREADS) k_tc_far(TcArgs a, const float2 *nearbuf,
                                                       int corrected) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.m) return;
  const uint32_t e = a.leafidx[k];
  const uint32_t c = a.leaves[e];
  const TcCell C = a.cells[c];
  double cx, cy;
  cell_centre(C, cx, cy);
  const double inv_s = pow2((int)C.level);
  const uint32_t nw = a.loff[(size_t)c * 8 + 3], ow = a.loff[(size_t)c * 8 + 2];
  float c0r = 0.f, c0i = 0.f;
  if (corrected) {
    const float sc = a.feat[(size_t)c * 16 + 14] * (1.f / LEARN_TARGET_SCALE);
    c0r = sc * a.mlp_y[(size_t)e * 2];
    c0i = sc * a.mlp_y[(size_t)e * 2 + 1];
  }
  float wr, wi;
  const float2 f =
      tc_far(a, k, cx, cy, inv_s, a.lco + (size_t)c * TC_KN, c0r, c0i, nw, ow, wr, wi);
  const float2 nv = nearbuf[k];
  const double kx = (double)nv.x + (double)f.x, ky = (double)nv.y + (double)f.y;
  if (a.kick) {
    a.kick[k] = make_double2(kx, ky);
  } else {
    const uint32_t gi = a.perm[k];
    a.vx[gi] = a.vx[gi] + kx;
    a.vy[gi] = a.vy[gi] + ky;
  }
}

// ---- the learned form's sampled check -----------------------------------------------------------

// The sampled check's direct sums, spread over the GPU: block `part` holds
// CHECK_THREADS x CHECK_PTS consecutive points in registers (each thread
// CHECK_PTS of them) and, for every sampled point j (sorted order, spread
// evenly), sums d3's pair formula in FP64 over them (coincident pairs and
// the point itself add nothing; distanceMin's clamp) into
// part_out[j * parts + part]. Each point is read once.
constexpr uint32_t CHECK_PTS = 16;
constexpr uint32_t CHECK_MAX_SAMPLES = 4096;  // sim_set_learned's limit

__device__ __forceinline__ uint32_t check_point(uint32_t j, uint32_t m, uint32_t samples) {
  return (uint32_t)(((2ull * j + 1) * m) / (2ull * samples));
}

__global__ void __launch_bounds__(CHECK_THREADS) k_tc_check(TcArgs a, uint32_t samples,
                                                            double dmin2, double2 *part_out) {
  __shared__ double2 red[CHECK_THREADS / 32];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t base = (size_t)blockIdx.x * CHECK_THREADS * CHECK_PTS;
  double px[CHECK_PTS], py[CHECK_PTS], ps[CHECK_PTS];
#pragma unroll
  for (uint32_t r = 0; r < CHECK_PTS; ++r) {
    const size_t i = base + (size_t)r * CHECK_THREADS + threadIdx.x;
    const bool ok = i < a.m;
    px[r] = ok ? a.px[i] : 0.0;
    py[r] = ok ? a.py[i] : 0.0;
    ps[r] = ok ? a.ps[i] : 0.0;  // a missing point adds 0 (and l = 0 is skipped)
  }
  for (uint32_t j = 0; j < samples; ++j) {
    const uint32_t k = check_point(j, a.m, samples);
    const double xi = a.px[k], yi = a.py[k];
    double vx = 0, vy = 0;
#pragma unroll
    for (uint32_t r = 0; r < CHECK_PTS; ++r) {
      const double dx = px[r] - xi, dy = py[r] - yi;
      double l = dx * dx + dy * dy;
      if (!(l > 0)) continue;
      if (l < dmin2) l = sqrt(dmin2 * l);
      const double w = ps[r] / l;
      vx += dx * w;
      vy += dy * w;
    }
    for (int o = 16; o > 0; o >>= 1) {
      vx += __shfl_xor_sync(0xffffffffu, vx, o);
      vy += __shfl_xor_sync(0xffffffffu, vy, o);
    }
    if (lane == 0) red[warp] = make_double2(vx, vy);
    __syncthreads();
    if (threadIdx.x == 0) {
      double rx = 0, ry = 0;
      for (uint32_t w = 0; w < CHECK_THREADS / 32; ++w) {
        rx += red[w].x;
        ry += red[w].y;
      }
      part_out[(size_t)j * gridDim.x + blockIdx.x] = make_double2(rx, ry);
    }
    __syncthreads();
  }
}

// One block: per sample the reference kick (its parts in order) against the
// kick the pass put in kick[k]; chk[0] = sum |kick - ref|^2, chk[1] =
// sum |ref|^2, in sample order (deterministic).
__global__ void __launch_bounds__(CHECK_THREADS) k_tc_check_fold(TcArgs a, uint32_t samples,
                                                                 uint32_t parts,
                                                                 const double2 *part_in,
                                                                 double *chk) {
  __shared__ double se[CHECK_THREADS], sr[CHECK_THREADS];
  double e2 = 0, r2 = 0;
  for (uint32_t j = threadIdx.x; j < samples; j += blockDim.x) {
    double rx = 0, ry = 0;
    for (uint32_t p = 0; p < parts; ++p) {
      const double2 v = part_in[(size_t)j * parts + p];
      rx += v.x;
      ry += v.y;
    }
    const double2 kk = a.kick[check_point(j, a.m, samples)];
    const double ex = kk.x - rx, ey = kk.y - ry;
    e2 += ex * ex + ey * ey;
    r2 += rx * rx + ry * ry;
  }
  se[threadIdx.x] = e2;
  sr[threadIdx.x] = r2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double te = 0, tr = 0;
    for (uint32_t t = 0; t < blockDim.x; ++t) {
      te += se[t];
      tr += sr[t];
    }
    chk[0] = te;
    chk[1] = tr;
  }
}

__global__ void k_tc_apply(TcArgs a) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.m) return;
  const uint32_t i = a.perm[k];
  const double2 kk = a.kick[k];
  a.vx[i] = a.vx[i] + kk.x;
  a.vy[i] = a.vy[i] + kk.y;
}

// ---- work counts of the last pass (for the roofline) ------------------------------------------------

// out[0] M2L source-target pairs (table entries), out[1] P2P point pairs
// (targets x sources over each leaf's P2P list, self pairs included),
// out[2] M2P point-cell pairs, out[3] P2L point-cell pairs.
__global__ void k_tc_count(TcArgs a, unsigned long long *out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncells) return;
  const TcCell C = a.cells[c];
  unsigned long long m2l = 0, pp = 0, mp = 0, pl = 0;
  if (C.level > 0) {
    const uint32_t ns = a.tab->nslot[C.quad];
    for (uint32_t j = 0; j < ns; ++j) m2l += a.m2l[(size_t)c * a.tab->sstride + j] != TC_NONE;
  }
  const uint32_t *lo = a.loff + (size_t)c * 8;
  if (C.nchild == 0) {
    for (uint32_t e = 0; e < lo[1]; ++e) pp += (unsigned long long)C.count * a.cells[a.pool[lo[0] + e]].count;
    mp = (unsigned long long)C.count * lo[3];
  }
  for (uint32_t e = 0; e < lo[5]; ++e) pl += a.cells[a.pool[lo[4] + e]].count;
  if (m2l) atomicAdd(&out[0], m2l);
  if (pp) atomicAdd(&out[1], pp);
  if (mp) atomicAdd(&out[2], mp);
  if (pl) atomicAdd(&out[3], pl);
}

// ---- tables (host) --------------------------------------------------------------------------------

struct Cplx {
  double re, im;
};
Cplx cmul(Cplx a, Cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

double binom(int n, int k) {
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

// Rounds to bf16 (nearest even) from a float.
uint16_t to_bf16(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  const uint32_t lsb = (u >> 16) & 1;
  u += 0x7FFF + lsb;
  return (uint16_t)(u >> 16);
}
float from_bf16(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// Builds the vector sets, the slot maps, the quadrant operators and the M2L
// operators for order p and opening kappa.
int build_tables(TcTabSet &d, uint32_t p, double kappa, cudaStream_t st) {
  TcTables &T = d.h;
  memset(&T, 0, sizeof T);
  const uint32_t q = p + 1;
  T.q = q;
  T.kappa2x2 = 2 * kappa * kappa;
  T.mac_far = 2 * kappa - 1;
  auto sep = [&](int x, int y) { return (double)(x * x + y * y) >= T.kappa2x2; };
  // near offsets
  uint32_t nn = 0;
  for (int y = -4; y <= 4; ++y)
    for (int x = -4; x <= 4; ++x)
      if (!sep(x, y)) {
        if (nn >= TC_NEAR_MAX) return -3;
        T.near_dx[nn] = (int8_t)x;
        T.near_dy[nn] = (int8_t)y;
        ++nn;
      }
  T.nnear = nn;
  std::vector<std::pair<int, int>> classes;
  for (uint32_t aq = 0; aq < 4; ++aq) {
    const int ax = aq & 1, ay = aq >> 1;
    uint32_t ns = 0;
    for (uint32_t o = 0; o < nn; ++o)
      for (uint32_t b = 0; b < 4; ++b) {
        const int bx = b & 1, by = b >> 1;
        const int vx = 2 * T.near_dx[o] + bx - ax, vy = 2 * T.near_dy[o] + by - ay;
        if (!sep(vx, vy)) {
          uint32_t ci = nn;
          for (uint32_t k = 0; k < nn; ++k)
            if (T.near_dx[k] == vx && T.near_dy[k] == vy) ci = k;
          if (ci == nn) return -3;  // cannot happen: a near child is a near offset
          T.map[aq][o][b] = (uint16_t)(TC_NEAR_FLAG | ci);
          continue;
        }
        size_t cls = 0;
        while (cls < classes.size() && !(classes[cls].first == vx && classes[cls].second == vy)) ++cls;
        if (cls == classes.size()) classes.push_back({vx, vy});
        if (ns >= TC_SLOT_MAX || classes.size() > TC_CLASS_MAX) return -3;
        T.map[aq][o][b] = (uint16_t)ns;
        T.slot_class[aq][ns] = (uint16_t)cls;
        ++ns;
      }
    T.nslot[aq] = ns;
    if (ns > T.sstride) T.sstride = ns;
  }
  // quadrant operators: child centre - parent centre = (s/4) delta_b
  for (uint32_t b = 0; b < 4; ++b) {
    const Cplx delta{(double)(2 * (int)(b & 1) - 1), (double)(2 * (int)(b >> 1) - 1)};
    for (uint32_t n = 0; n < q; ++n)
      for (uint32_t k = 0; k <= n; ++k) {
        // M2M: C(n,k) 2^-k 4^-(n-k) delta^(n-k)
        Cplx pw{1, 0};
        for (uint32_t e = 0; e < n - k; ++e) pw = cmul(pw, delta);
        const double f = binom(n, k) * std::ldexp(1.0, -(int)k) * std::ldexp(1.0, -2 * (int)(n - k));
        T.m2m_re[b][n][k] = f * pw.re;
        T.m2m_im[b][n][k] = f * pw.im;
      }
    for (uint32_t mm = 0; mm < q; ++mm)
      for (uint32_t l = mm; l < q; ++l) {
        // L2L: C(l,m) delta^(l-m) 4^-(l-m) 2^-(m+1)
        Cplx pw{1, 0};
        for (uint32_t e = 0; e < l - mm; ++e) pw = cmul(pw, delta);
        const double f = binom(l, mm) * std::ldexp(1.0, -2 * (int)(l - mm)) * std::ldexp(1.0, -(int)(mm + 1));
        T.l2l_re[b][mm][l] = (float)(f * pw.re);
        T.l2l_im[b][mm][l] = (float)(f * pw.im);
      }
  }
  // M2L operators in real form, W[k][n] (y = x W), stored as the B tile (row
  // n holds W[.][n]), bf16 hi then lo
  std::vector<uint16_t> w(classes.size() * 2 * TC_KN * TC_KN, 0);
  for (size_t cls = 0; cls < classes.size(); ++cls) {
    // classes hold the source's offset from the target, B - A; the
    // translation is z0 = c_A - c_B = -(B - A)
    const Cplx v{-(double)classes[cls].first, -(double)classes[cls].second};
    const double d2 = v.re * v.re + v.im * v.im;
    const Cplx inv{v.re / d2, -v.im / d2};
    std::vector<Cplx> ipw(2 * q + 1);
    ipw[0] = {1, 0};
    for (uint32_t e = 1; e <= 2 * q; ++e) ipw[e] = cmul(ipw[e - 1], inv);
    double W[TC_KN][TC_KN] = {};
    for (uint32_t l = 0; l < q; ++l)
      for (uint32_t k = 0; k < q; ++k) {
        // K[l][k] = (-1)^l C(k+l, l) / v^(k+l+1)
        const double f = ((l & 1) ? -1.0 : 1.0) * binom(k + l, l);
        const double kr = f * ipw[k + l + 1].re, ki = f * ipw[k + l + 1].im;
        W[k][l] = kr;
        W[q + k][l] = -ki;
        W[k][q + l] = ki;
        W[q + k][q + l] = kr;
      }
    for (uint32_t nidx = 0; nidx < TC_KN; ++nidx)
      for (uint32_t k = 0; k < TC_KN; ++k) {
        const double x = W[k][nidx];
        const uint16_t hi = to_bf16((float)x);
        const uint16_t lo = to_bf16((float)(x - (double)from_bf16(hi)));
        const uint32_t off = tc::tile_offset(nidx, k / 8, TC_KN) / 2 + k % 8;
        w[(cls * 2 + 0) * TC_KN * TC_KN + off] = hi;
        w[(cls * 2 + 1) * TC_KN * TC_KN + off] = lo;
      }
  }
  if (!d.tab) D3_CUDA_OK(cudaMalloc(&d.tab, sizeof(TcTables)));
  d.p = 0;
  cudaFree(d.wops);
  D3_CUDA_OK(cudaMalloc(&d.wops, w.size() * 2));
  if (cudaMemcpyAsync(d.tab, &T, sizeof T, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d.wops, w.data(), w.size() * 2, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -1;
  d.p = p;
  d.kappa = kappa;
  return 0;
}

int reserve(TcDev &d, uint32_t ncells, uint32_t m) {
  if (ncells > d.ccap) {
    const uint32_t cap = ncells + ncells / 4 + 64;
    cudaFree(d.cells); cudaFree(d.mco); cudaFree(d.mbf); cudaFree(d.lco); cudaFree(d.near);
    cudaFree(d.m2l); cudaFree(d.groups); cudaFree(d.loff);
    D3_CUDA_OK(cudaMalloc(&d.cells, cap * sizeof(TcCell)));
    D3_CUDA_OK(cudaMalloc(&d.mco, (size_t)cap * 2 * TC_MAXQ * 8));
    D3_CUDA_OK(cudaMalloc(&d.mbf, (size_t)cap * 64 * 2));
    D3_CUDA_OK(cudaMalloc(&d.lco, (size_t)cap * TC_KN * 4));
    D3_CUDA_OK(cudaMalloc(&d.near, (size_t)cap * TC_NEAR_MAX * 4));
    D3_CUDA_OK(cudaMalloc(&d.m2l, (size_t)cap * TC_SLOT_MAX * 4));
    D3_CUDA_OK(cudaMalloc(&d.groups, (size_t)cap * 4 * 4));
    D3_CUDA_OK(cudaMalloc(&d.loff, (size_t)cap * 8 * 4));
    cudaFree(d.arrive);
    D3_CUDA_OK(cudaMalloc(&d.arrive, (size_t)cap * 4));
    d.ccap = cap;
  }
  if (m > d.pcap) {
    const uint32_t cap = m + m / 4 + 1024;
    cudaFree(d.kick);
    cudaFree(d.nearbuf);
    D3_CUDA_OK(cudaMalloc(&d.kick, (size_t)cap * sizeof(double2)));
    D3_CUDA_OK(cudaMalloc(&d.nearbuf, (size_t)cap * sizeof(float2)));
    cudaFree(d.leafidx);
    D3_CUDA_OK(cudaMalloc(&d.leafidx, (size_t)cap * sizeof(uint32_t)));
    d.pcap = cap;
  }
  if (d.ccap > d.lcap) {
    cudaFree(d.feat); cudaFree(d.leaves); cudaFree(d.mlp_x); cudaFree(d.mlp_y);
    D3_CUDA_OK(cudaMalloc(&d.feat, (size_t)d.ccap * 16 * 4));
    D3_CUDA_OK(cudaMalloc(&d.leaves, (size_t)d.ccap * 4));
    D3_CUDA_OK(cudaMalloc(&d.mlp_x, (size_t)d.ccap * 12 * 4));
    D3_CUDA_OK(cudaMalloc(&d.mlp_y, (size_t)d.ccap * 2 * 4));
    d.lcap = d.ccap;
  }
  return 0;
}

// The table set for (p, kappa): an existing one, else built in the older slot.
TcTabSet *tables_for(TcDev &d, uint32_t p, double kappa, cudaStream_t st) {
  for (TcTabSet &t : d.sets)
    if (t.tab && t.p == p && t.kappa == kappa) return &t;
  TcTabSet &t = d.sets[d.next_set];
  d.next_set ^= 1;
  if (build_tables(t, p, kappa, st)) return nullptr;
  return &t;
}


}  // namespace

namespace {

TcDev *tc_dev(FastScratch &s) {
  if (s.fmm_tc) return static_cast<TcDev *>(s.fmm_tc);
  TcDev *d = new TcDev();
  if (cudaMalloc(&d->info, TI_WORDS * 4) != cudaSuccess ||
      cudaHostAlloc(&d->h_info, TI_WORDS * 4, cudaHostAllocDefault) != cudaSuccess ||
      cudaMalloc(&d->chk, 2 * sizeof(double)) != cudaSuccess ||
      cudaHostAlloc(&d->h_chk, 2 * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
    cudaFree(d->info);
    cudaFreeHost(d->h_info);
    cudaFree(d->chk);
    delete d;
    return nullptr;
  }
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(k_tc_m2l, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(M2lSmem));
  d->sms = sms;
  bool ok = cudaStreamCreateWithFlags(&d->side, cudaStreamNonBlocking) == cudaSuccess;
  for (cudaEvent_t *e : {&d->ev_geom, &d->ev_up, &d->ev_lists, &d->ev_near, &d->ev_down,
                         &d->ev_feat, &d->ev_side_idle})
    ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    if (d->side) cudaStreamDestroy(d->side);
    for (cudaEvent_t e : {d->ev_geom, d->ev_up, d->ev_lists, d->ev_near, d->ev_down, d->ev_feat,
                          d->ev_side_idle})
      if (e) cudaEventDestroy(e);
    cudaFree(d->info);
    cudaFreeHost(d->h_info);
    cudaFree(d->chk);
    cudaFreeHost(d->h_chk);
    delete d;
    return nullptr;
  }
  s.fmm_tc = d;
  return d;
}

// The passes of one expansion order over a built tree and lists: upward,
// M2L, P2L, L2L, leaf features, (the network, when `learned`), L2P / M2P and
// the near field.
// The upward pass at the table set's order: on the side stream, to overlap
// the list build (`overlap`), else on st. Its grid covers `ncells` leaves at
// most (the kernel reads the leaf count on the device).
void tc_upward(TcDev &d, TcArgs &g, const TcTabSet &ts, bool overlap, cudaStream_t st) {
  g.tab = ts.tab;
  g.wops = ts.wops;
  g.q = ts.p + 1;
  cudaStream_t us = st;
  if (overlap) {
    cudaEventRecord(d.ev_geom, st);
    cudaStreamWaitEvent(d.side, d.ev_geom, 0);
    us = d.side;
  }
  cudaEventRecord(d.ev[9], us);
  cudaMemsetAsync(d.arrive, 0, (size_t)g.ncells * 4, us);
  launch_up(g, d.arrive, g.ncells, us);
  cudaEventRecord(d.ev[10], us);
  if (overlap) cudaEventRecord(d.ev_up, us);
}

int tc_order_pass(TcDev &d, TcArgs &g, const TcTabSet &ts, uint32_t tiles, bool learned,
                  bool far_only, bool upward_done, cudaStream_t st) {
  g.tab = ts.tab;
  g.wops = ts.wops;
  g.q = ts.p + 1;
  const uint32_t nleaf = d.h_info[TI_LEAVES];
  const unsigned lw = blocks_for((size_t)nleaf * 32, TC_THREADS);
  // the near field on the side stream, beside M2L, P2L and the downward pass
  // (it reads only the lists and the points); `far_only` reuses the stored one
  if (!far_only) {
    cudaEventRecord(d.ev_lists, st);
    cudaStreamWaitEvent(d.side, d.ev_lists, 0);
    cudaEventRecord(d.ev[7], d.side);
    D3_LAUNCH(k_tc_near, blocks_for((size_t)nleaf * 32, NEAR_THREADS), NEAR_THREADS, 0, d.side)(
        g, d.nearbuf);
    cudaEventRecord(d.ev[8], d.side);
    cudaEventRecord(d.ev_near, d.side);
  }
  if (upward_done) cudaStreamWaitEvent(st, d.ev_up, 0);
  else tc_upward(d, g, ts, false, st);
  cudaEventRecord(d.ev[3], st);
  if (tiles) D3_LAUNCH(k_tc_m2l, tiles, M2L_THREADS, sizeof(M2lSmem), st)(g);
  cudaEventRecord(d.ev[4], st);
  d.last_tiles = tiles;
  if (!d.last_args) d.last_args = new TcArgs;
  *static_cast<TcArgs *>(d.last_args) = g;
  launch_p2l(g, st);
  cudaEventRecord(d.ev[5], st);
  launch_down(g, nleaf, st);
  cudaEventRecord(d.ev[6], st);
  if (learned) {
    D3_LAUNCH(k_tc_features, lw, TC_THREADS, 0, st)(g);
    D3_LAUNCH(k_tc_pack, blocks_for(nleaf, 256), 256, 0, st)(g);
    if (mlp_infer_tc(d.mlp_x, nleaf, d.mlp, d.mlp_y, g.status, st)) return -1;
  } else {
    // the leaves' feature rows (sim_fmm_leaves) on the side stream, beside
    // the far field; joined before the pass returns
    cudaEventRecord(d.ev_down, st);
    cudaStreamWaitEvent(d.side, d.ev_down, 0);
    D3_LAUNCH(k_tc_features, lw, TC_THREADS, 0, d.side)(g);
    cudaEventRecord(d.ev_feat, d.side);
  }
  cudaEventRecord(d.ev[11], st);
  if (!far_only) cudaStreamWaitEvent(st, d.ev_near, 0);
  D3_LAUNCH(k_tc_far, blocks_for(g.m, TC_THREADS), TC_THREADS, 0, st)(g, d.nearbuf, learned ? 1 : 0);
  cudaEventRecord(d.ev[12], st);
  if (!learned) cudaStreamWaitEvent(st, d.ev_feat, 0);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

void fmm_tc_free(FastScratch &s) {
  TcDev *d = static_cast<TcDev *>(s.fmm_tc);
  if (!d) return;
  for (TcTabSet &t : d->sets) {
    cudaFree(t.tab);
    cudaFree(t.wops);
  }
  cudaFree(d->cells); cudaFree(d->mco); cudaFree(d->mbf);
  cudaFree(d->lco); cudaFree(d->near); cudaFree(d->m2l); cudaFree(d->groups); cudaFree(d->loff);
  cudaFree(d->arrive);
  cudaFree(d->pool); cudaFree(d->info); cudaFreeHost(d->h_info);
  cudaFree(d->feat); cudaFree(d->leaves); cudaFree(d->mlp_x); cudaFree(d->mlp_y);
  cudaFree(d->kick); cudaFree(d->chk); cudaFreeHost(d->h_chk); cudaFree(d->mlp);
  cudaFree(d->chk_part); cudaFree(d->nearbuf); cudaFree(d->leafidx);
  for (cudaEvent_t e : d->ev)
    if (e) cudaEventDestroy(e);
  if (d->side) {
    cudaStreamSynchronize(d->side);
    cudaStreamDestroy(d->side);
  }
  for (cudaEvent_t e : {d->ev_geom, d->ev_up, d->ev_lists, d->ev_near, d->ev_down, d->ev_feat,
                        d->ev_side_idle})
    if (e) cudaEventDestroy(e);
  delete static_cast<TcArgs *>(d->last_args);
  delete d;
  s.fmm_tc = nullptr;
}

int fmm_tc_set_learned(FastScratch &s, const float *params, uint32_t len) {
  if (len != (uint32_t)MLP_PARAMS || !params) return -3;
  TcDev *d = tc_dev(s);
  if (!d) return -1;
  if (!d->mlp) D3_CUDA_OK(cudaMalloc(&d->mlp, MLP_PARAMS * 4));
  return cudaMemcpy(d->mlp, params, MLP_PARAMS * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}

int fmm_tc_leaves(FastScratch &s, float *out, uint32_t cap) {
  TcDev *d = static_cast<TcDev *>(s.fmm_tc);
  if (!d || !d->feat) return 0;
  const uint32_t n = d->ncells_last;
  if (out && cap >= n && n)
    if (cudaMemcpy(out, d->feat, (size_t)n * 16 * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return (int)n;
}

void fmm_tc_stats(FastScratch &s, double *out) {
  TcDev *d = static_cast<TcDev *>(s.fmm_tc);
  for (int k = 0; k < TC_STATS; ++k) out[k] = 0;
  if (!d) return;
  out[0] = s.learn_checks;
  out[1] = s.learn_fallbacks;
  out[2] = s.learn_last_rms;
  out[3] = d->ncells_last;
  if (!d->ev[0] || !d->last_args) return;
  auto span = [&](int a, int b) -> double {
    float ms = 0;
    return cudaEventElapsedTime(&ms, d->ev[a], d->ev[b]) == cudaSuccess ? ms : 0.0;
  };
  out[4] = span(3, 4);
  out[5] = span(7, 8);
  out[12] = span(0, 1);
  out[13] = span(1, 2);
  out[14] = span(9, 10);
  out[15] = span(4, 5);
  out[16] = span(5, 6);
  out[17] = span(6, 11);
  out[18] = span(0, 12);
  out[19] = span(11, 12);
  const TcArgs &g = *static_cast<const TcArgs *>(d->last_args);
  out[6] = d->last_tiles;
  unsigned long long *cnt = nullptr;
  if (cudaMalloc(&cnt, 4 * sizeof(unsigned long long)) != cudaSuccess) return;
  unsigned long long h[4] = {0, 0, 0, 0};
  cudaMemset(cnt, 0, sizeof h);
  k_tc_count<<<blocks_for(g.ncells, 256), 256>>>(g, cnt);
  if (cudaMemcpy(h, cnt, sizeof h, cudaMemcpyDeviceToHost) == cudaSuccess)
    for (int k = 0; k < 4; ++k) out[7 + k] = (double)h[k];
  cudaFree(cnt);
  out[11] = g.q;
}

namespace {

int tc_run(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
           const FmmParams &prm, int form, const double *seed, uint32_t *status,
           cudaStream_t st);

}  // namespace

int fmm_tc_run(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
               const FmmParams &prm, int form, const double *seed, uint32_t *status,
               cudaStream_t st) {
  if (prm.dmax2 < INFINITY) return fmm_run(s, t, a, strengths, prm, seed, status, st);
  const int r = tc_run(s, t, a, strengths, prm, form, seed, status, st);
  // whatever path the run ended on, later work on st follows all of its
  // side-stream work
  if (TcDev *d = static_cast<TcDev *>(s.fmm_tc)) {
    cudaEventRecord(d->ev_side_idle, d->side);
    cudaStreamWaitEvent(st, d->ev_side_idle, 0);
  }
  return r;
}

namespace {

int tc_run(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
           const FmmParams &prm, int form, const double *seed, uint32_t *status,
           cudaStream_t st) {
  TcDev *dp = tc_dev(s);
  if (!dp) return -1;
  TcDev &d = *dp;
  if (!d.ev[0])
    for (cudaEvent_t &e : d.ev) cudaEventCreate(&e);
  cudaEventRecord(d.ev[0], st);
  FmmPrep pr;
  const int pre = fmm_prepare(s, t, a, strengths, prm.alpha, pr, st);
  if (pre == 2) return 1;
  if (pre <= 0) return pre;
  cudaEventRecord(d.ev[1], st);
  uint32_t p = 8;
  if (prm.order >= 1 && prm.order <= (double)(TC_MAXQ - 1)) p = (uint32_t)prm.order;
  double kappa = prm.opening;
  if (!(kappa >= 1 && kappa <= 2)) kappa = 1.5;
  // the learned form: order 4 plus the network, checked on sampled points;
  // the plain form at the requested order (8 unless it asks for more) when
  // the check fails or no network is installed
  bool learned = form == 3 && d.mlp;
  if (learned && d.hold) {
    --d.hold;
    learned = false;
  }
  if (form == 3 && p < 5) p = 8;
  TcTabSet *main = tables_for(d, learned ? LEARN_ORDER : p, kappa, st);
  if (!main) return -1;
  if (reserve(d, pr.ncells, pr.m)) return -1;
  TcArgs g;
  memset(&g, 0, sizeof g);
  g.tab = main->tab;
  g.wops = main->wops;
  g.keys = pr.keys;
  g.perm = pr.perm;
  g.px = pr.px; g.py = pr.py; g.ps = pr.ps; g.ux = pr.ux; g.uy = pr.uy;
  g.fc = pr.cells;
  g.cells = d.cells;
  g.mco = d.mco; g.mbf = d.mbf; g.lco = d.lco;
  g.near = d.near; g.m2l = d.m2l; g.groups = d.groups; g.loff = d.loff;
  g.feat = d.feat; g.leaves = d.leaves; g.mlp_x = d.mlp_x; g.mlp_y = d.mlp_y;
  g.leafidx = d.leafidx;
  g.kick = learned ? d.kick : nullptr;
  g.vx = a.vx; g.vy = a.vy;
  g.info = d.info;
  g.status = status;
  g.lvl = pr.info + 8;  // FI_LVL
  g.ncells = pr.ncells; g.nlev = pr.nlev; g.m = pr.m; g.q = main->p + 1; g.ccap = d.ccap;
  g.inv_w = pr.inv_w;
  g.dmin2 = prm.dmin2 * pr.inv_w * pr.inv_w;
  g.dmin2f = (float)prm.dmin2;
  g.seed = seed;
  d.ncells_last = pr.ncells;
  if (cudaMemsetAsync(d.info, 0, TI_WORDS * 4, st) != cudaSuccess) return -1;
  D3_LAUNCH(k_tc_geom, blocks_for(pr.ncells, 256), 256, 0, st)(g);
  // the upward pass does not read the lists: it runs beside them
  tc_upward(d, g, *main, true, st);
  // lists (geometry and opening only); grow the pool and redo on overflow
  size_t need = d.last_pool ? d.last_pool + d.last_pool / 4 + 4096 : (size_t)pr.ncells * 24 + 4096;
  for (int attempt = 0;; ++attempt) {
    if (need > d.pool_cap) {
      cudaFree(d.pool);
      d.pool = nullptr;
      d.pool_cap = need;
      D3_CUDA_OK(cudaMalloc(&d.pool, d.pool_cap * 4));
    }
    g.pool = d.pool;
    g.pool_cap = d.pool_cap;
    if (cudaMemsetAsync(d.info, 0, 8 * 4, st) != cudaSuccess) return -1;
    for (uint32_t lev = 0; lev < pr.nlev; ++lev) {
      const uint32_t c0 = pr.lvl[lev], c1 = pr.lvl[lev + 1];
      if (c1 > c0)
        D3_LAUNCH(k_tc_lists, blocks_for((size_t)(c1 - c0) * 32, LIST_THREADS), LIST_THREADS, 0, st)(
            g, c0, c1);
    }
    if (cudaMemcpyAsync(d.h_info, d.info, TI_WORDS * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return -1;
    const uint32_t used = d.h_info[TI_POOL_P2P];
    if (!d.h_info[TI_OVF]) {
      d.last_pool = used;
      break;
    }
    if ((d.h_info[TI_OVF] & 2) || attempt > 6) return -1;  // a walk's stack overflowed
    need = 2 * (size_t)(used > need ? used : need);
  }
  cudaEventRecord(d.ev[2], st);
  uint32_t tiles = 0;
  for (uint32_t q4 = 0; q4 < 4; ++q4) tiles += (d.h_info[TI_GROUP + q4] + TC_TILE - 1) / TC_TILE;
  if (tc_order_pass(d, g, *main, tiles, learned, false, true, st)) return -1;
  if (!learned) return 1;
  // the sampled check against the FP64 direct sum
  uint32_t samples = s.learn_samples ? s.learn_samples : 64;
  if (samples > CHECK_MAX_SAMPLES) samples = CHECK_MAX_SAMPLES;
  const uint32_t parts = blocks_for(pr.m, CHECK_THREADS * CHECK_PTS);
  if ((size_t)samples * parts > d.chk_cap) {
    cudaFree(d.chk_part);
    d.chk_part = nullptr;
    D3_CUDA_OK(cudaMalloc(&d.chk_part, (size_t)samples * parts * sizeof(double2)));
    d.chk_cap = samples * parts;
  }
  D3_LAUNCH(k_tc_check, parts, CHECK_THREADS, 0, st)(g, samples, prm.dmin2, d.chk_part);
  D3_LAUNCH(k_tc_check_fold, 1, CHECK_THREADS, 0, st)(g, samples, parts, d.chk_part, d.chk);
  if (cudaMemcpyAsync(d.h_chk, d.chk, 2 * sizeof(double), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -1;
  const double rms = d.h_chk[1] > 0 ? sqrt(d.h_chk[0] / d.h_chk[1]) : 0;
  s.learn_checks += 1;
  s.learn_last_rms = rms;
  if (rms <= s.learn_tol) {
    D3_LAUNCH(k_tc_apply, blocks_for(pr.m, 256), 256, 0, st)(g);
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
  }
  // the fallback: the plain form at order p, straight into the velocities
  s.learn_fallbacks += 1;
  d.hold = s.learn_hold;
  TcTabSet *fb = tables_for(d, p, kappa, st);
  if (!fb) return -1;
  g.kick = nullptr;
  if (tc_order_pass(d, g, *fb, tiles, false, true, false, st)) return -1;
  return 1;
}

}  // namespace

}  // namespace d3
