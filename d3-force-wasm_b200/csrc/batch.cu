// batch.cu — batched fast mode (no reference counterpart): thousands of
// independent graphs of uneven sizes tick in ONE persistent launch per tick,
// a run of ticks is captured in one CUDA graph, and the launch shape is
// picked by an autotuner.
//
// Each graph is a d3 simulation of its own with forceManyBody (FMM order 8,
// opening 1.5, distanceMin 1, strength -30), forceLink (distance 30, d3's
// default strength 1 / min(degree) and bias, one iteration) and forceCollide
// (radius 3, strength 1, one iteration), in FP32, with d3's alpha schedule
// and velocity decay 0.4. The fast forms follow the reference's fast mode:
// the link and the collide are Jacobi passes over a snapshot x + vx
// (link_fast.zig, grid.zig: each node adds only its own side), the
// many-body force an FMM (fmm.zig's expansions) — here on a complete
// quadtree over the graph's square box, with the level-free lattice
// operators of fmm_tc.cu (geometric centres, expansions normalised by the
// cell side), so every cell's interaction list is a fixed set of offsets.
//
// Persistent kernel, one launch per tick: the CTAs take graphs from the
// tick's queue counter, largest first, and run the graph's whole tick in the
// CTA (shared memory and a per-CTA scratch region in global memory):
//   FMM   box; leaf of each node at level L (chosen per graph from the
//         autotuned leaf size); a bitonic sort of (leaf, node) keys (unique,
//         so the order - and every sum - is the same in any run and on any
//         schedule); P2M; M2M, M2L (39 offsets per quadrant), L2L by level;
//         L2P; P2P over the 13 near leaves; v += kick.
//   link  snapshot px = x + vx; each node sums its links' own sides.
//   collide snapshot; the (grid cell, node) keys sorted; each node scans
//         the 3 x 3 cells around it.
//   integrate v *= 0.6, x += v.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace d3 {
namespace {

constexpr int BQ = 9;           // order 8: q = p + 1
constexpr int BNEAR = 13;       // same-level near offsets at opening 1.5
constexpr int BSLOT = 39;       // M2L offsets per quadrant at opening 1.5
constexpr int BCLASS_MAX = 64;  // distinct M2L offsets (60)
constexpr uint32_t BMAX_N = 16384;
constexpr int BMAX_L = 6;
constexpr uint32_t BSORT = BMAX_N;                         // bitonic array (power of two)
constexpr uint32_t BCELLS = (((1u << (2 * (BMAX_L + 1))) - 1) / 3);  // levels 0..6
constexpr float BDMIN2 = 1.f, BSTRENGTH = -30.f, BDIST = 30.f, BRADIUS = 3.f;

struct BTables {
  int8_t near_dx[BNEAR], near_dy[BNEAR];
  int8_t slot_dx[4][BSLOT], slot_dy[4][BSLOT];
  uint8_t slot_class[4][BSLOT];
  float2 k[BCLASS_MAX][BQ][BQ];  // M2L [class][l][k]
  float2 m2m[4][BQ][BQ];         // [b][n][k]
  float2 l2l[4][BQ][BQ];         // [b][m][l]
};

static_assert(sizeof(BTables) % 16 == 0, "the tables are copied to shared memory in 16-byte units");

struct BArgs {
  const BTables *tab;
  uint32_t graphs;
  const uint32_t *order;     // graphs, largest first
  const uint32_t *node_off;  // [graphs + 1]
  const uint8_t *level;      // FMM leaf level per graph
  const uint32_t *adj_off;   // [N + 1] per node (global index)
  const uint32_t *adj_j;     // local index of the other node
  const float4 *adj_w;       // strength, distance, own-side share, sign (+1 source / -1 target)
  float *x, *y, *vx, *vy;
  float *scratch;            // per CTA
  size_t scratch_stride;     // floats per CTA
  uint32_t *queue;           // this tick's counter
  float alpha;
  uint32_t tick;
  float2 *kick_out;          // non-null: many-body kick only (per global node), no other force
};

// Per-CTA scratch layout (floats): see scratch_layout().
struct BScratch {
  float *sx, *sy, *ss, *px, *py;
  uint32_t *sidx, *leaf_start, *keys2;
  float2 *kick, *M, *L;
};

__device__ __forceinline__ uint32_t cells_before(int level) {  // cells at levels < level
  return ((1u << (2 * level)) - 1) / 3;
}

__device__ __forceinline__ BScratch scratch_of(const BArgs &a) {
  float *base = a.scratch + (size_t)blockIdx.x * a.scratch_stride;
  BScratch s;
  s.sx = base;
  s.sy = s.sx + BMAX_N;
  s.ss = s.sy + BMAX_N;
  s.px = s.ss + BMAX_N;
  s.py = s.px + BMAX_N;
  s.sidx = reinterpret_cast<uint32_t *>(s.py + BMAX_N);
  s.leaf_start = s.sidx + BMAX_N;                                   // 4^6 + 1
  s.keys2 = s.leaf_start + (1u << (2 * BMAX_L)) + 16;              // BMAX_N
  s.kick = reinterpret_cast<float2 *>(s.keys2 + BMAX_N);           // BMAX_N
  s.M = s.kick + BMAX_N;                                            // BCELLS * BQ
  s.L = s.M + (size_t)BCELLS * BQ;                                  // BCELLS * BQ
  return s;
}

__host__ __device__ constexpr size_t scratch_floats() {
  return 5 * (size_t)BMAX_N + BMAX_N + ((1u << (2 * BMAX_L)) + 16) + BMAX_N + 2 * (size_t)BMAX_N +
         4 * (size_t)BCELLS * BQ + 64;
}

__device__ __forceinline__ uint32_t interleave(uint32_t x, uint32_t y) {
  uint32_t r = 0;
  for (int b = 0; b < 16; ++b) r |= ((x >> b) & 1u) << (2 * b) | ((y >> b) & 1u) << (2 * b + 1);
  return r;
}
__device__ __forceinline__ void deinterleave(uint32_t m, uint32_t &x, uint32_t &y) {
  x = y = 0;
  for (int b = 0; b < 16; ++b) {
    x |= ((m >> (2 * b)) & 1u) << b;
    y |= ((m >> (2 * b + 1)) & 1u) << b;
  }
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Bitonic sort of keys[0 .. P) in shared memory (P a power of two, padding
// keys 0xFFFFFFFF sort last).
__device__ void bitonic(uint32_t *keys, uint32_t P) {
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const uint32_t a = keys[i], b = keys[l];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            keys[i] = b;
            keys[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
}

// First index in keys[0 .. n) with keys[i] >= t (keys sorted).
__device__ __forceinline__ uint32_t lower(const uint32_t *keys, uint32_t n, uint32_t t) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (keys[mid] < t) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ float block_reduce(float v, bool is_max, float *sh) {
  for (int o = 16; o > 0; o >>= 1) {
    const float w = __shfl_xor_sync(0xffffffffu, v, o);
    v = is_max ? fmaxf(v, w) : fminf(v, w);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = sh[0];
  for (uint32_t w = 1; w < blockDim.x / 32; ++w) r = is_max ? fmaxf(r, sh[w]) : fminf(r, sh[w]);
  return r;
}

// The many-body force of one graph: kick of every node into S.kick (sorted
// order) and then into the velocities (or kick_out).
__device__ void graph_many_body(const BArgs &a, const BTables &T, uint32_t g, uint32_t n0,
                                uint32_t n, const BScratch &S, uint32_t *skeys, float *red) {
  const uint32_t t = threadIdx.x, nt = blockDim.x;
  const int L = a.level[g];
  const uint32_t side = 1u << L;
  // box
  float mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
  for (uint32_t i = t; i < n; i += nt) {
    const float x = a.x[n0 + i], y = a.y[n0 + i];
    mnx = fminf(mnx, x);
    mxx = fmaxf(mxx, x);
    mny = fminf(mny, y);
    mxy = fmaxf(mxy, y);
  }
  mnx = block_reduce(mnx, false, red);
  mxx = block_reduce(mxx, true, red);
  mny = block_reduce(mny, false, red);
  mxy = block_reduce(mxy, true, red);
  float w = fmaxf(mxx - mnx, mxy - mny);
  if (!(w > 0)) w = 1;
  w *= 1.0001f;  // the largest coordinate stays inside the last cell
  const float inv_w = 1.f / w;
  // keys: (leaf << 14) | node, sorted
  uint32_t P = 64;
  while (P < n) P <<= 1;
  for (uint32_t i = t; i < P; i += nt) {
    uint32_t key = 0xFFFFFFFFu;
    if (i < n) {
      const uint32_t qx = min(side - 1, (uint32_t)((a.x[n0 + i] - mnx) * inv_w * side));
      const uint32_t qy = min(side - 1, (uint32_t)((a.y[n0 + i] - mny) * inv_w * side));
      key = (interleave(qx, qy) << 14) | i;
    }
    skeys[i] = key;
  }
  __syncthreads();
  bitonic(skeys, P);
  const uint32_t nleaf = side * side;
  for (uint32_t c = t; c <= nleaf; c += nt) S.leaf_start[c] = lower(skeys, n, c << 14);
  // sorted points in scaled coordinates: u in [0, 1) x [0, 1)
  for (uint32_t k = t; k < n; k += nt) {
    const uint32_t i = skeys[k] & 0x3FFFu;
    S.sidx[k] = i;
    S.sx[k] = (a.x[n0 + i] - mnx) * inv_w;
    S.sy[k] = (a.y[n0 + i] - mny) * inv_w;
    S.ss[k] = BSTRENGTH * a.alpha;
  }
  __syncthreads();
  // P2M at the leaves: M'_k = sum s ((u - c) / s_L)^k
  const float sL = 1.f / side;
  const uint32_t leaf0 = cells_before(L);
  for (uint32_t c = t; c < nleaf; c += nt) {
    uint32_t ix, iy;
    deinterleave(c, ix, iy);
    const float cx = (ix + 0.5f) * sL, cy = (iy + 0.5f) * sL;
    float2 m[BQ];
    for (int k = 0; k < BQ; ++k) m[k] = make_float2(0, 0);
    for (uint32_t k = S.leaf_start[c]; k < S.leaf_start[c + 1]; ++k) {
      const float2 z = make_float2((S.sx[k] - cx) * side, (S.sy[k] - cy) * side);
      float2 p = make_float2(S.ss[k], 0);
      for (int o = 0; o < BQ; ++o) {
        m[o].x += p.x;
        m[o].y += p.y;
        p = cmul(p, z);
      }
    }
    for (int k = 0; k < BQ; ++k) S.M[(leaf0 + c) * BQ + k] = m[k];
  }
  __syncthreads();
  // M2M up to level 2
  for (int l = L - 1; l >= 2; --l) {
    const uint32_t nc = 1u << (2 * l), base = cells_before(l), cbase = cells_before(l + 1);
    for (uint32_t e = t; e < nc * BQ; e += nt) {
      const uint32_t c = e / BQ, nn = e % BQ;
      float2 acc = make_float2(0, 0);
      for (uint32_t b = 0; b < 4; ++b) {
        const float2 *cm = S.M + (size_t)(cbase + (c << 2 | b)) * BQ;
        for (uint32_t k = 0; k <= nn; ++k) {
          const float2 v = cmul(T.m2m[b][nn][k], cm[k]);
          acc.x += v.x;
          acc.y += v.y;
        }
      }
      S.M[(size_t)(base + c) * BQ + nn] = acc;
    }
    __syncthreads();
  }
  // M2L at every level >= 2 (the lattice offsets of the cell's quadrant)
  for (int l = 2; l <= L; ++l) {
    const uint32_t nc = 1u << (2 * l), base = cells_before(l), sl = 1u << l;
    for (uint32_t e = t; e < nc * BQ; e += nt) {
      const uint32_t c = e / BQ, ll = e % BQ, qd = c & 3;
      uint32_t ix, iy;
      deinterleave(c, ix, iy);
      float2 acc = make_float2(0, 0);
      for (int j = 0; j < BSLOT; ++j) {
        const int bx = (int)ix + T.slot_dx[qd][j], by = (int)iy + T.slot_dy[qd][j];
        if (bx < 0 || by < 0 || bx >= (int)sl || by >= (int)sl) continue;
        const float2 *mb = S.M + (size_t)(base + interleave(bx, by)) * BQ;
        const float2 *kk = T.k[T.slot_class[qd][j]][ll];
        for (int k = 0; k < BQ; ++k) {
          const float2 v = cmul(kk[k], mb[k]);
          acc.x += v.x;
          acc.y += v.y;
        }
      }
      S.L[(size_t)(base + c) * BQ + ll] = acc;
    }
    __syncthreads();
  }
  // L2L down
  for (int l = 2; l < L; ++l) {
    const uint32_t nc = 1u << (2 * (l + 1)), pbase = cells_before(l), cbase = cells_before(l + 1);
    for (uint32_t e = t; e < nc * BQ; e += nt) {
      const uint32_t c = e / BQ, mm = e % BQ, b = c & 3;
      const float2 *pl = S.L + (size_t)(pbase + (c >> 2)) * BQ;
      float2 acc = S.L[(size_t)(cbase + c) * BQ + mm];
      for (uint32_t l2 = mm; l2 < BQ; ++l2) {
        const float2 v = cmul(T.l2l[b][mm][l2], pl[l2]);
        acc.x += v.x;
        acc.y += v.y;
      }
      S.L[(size_t)(cbase + c) * BQ + mm] = acc;
    }
    __syncthreads();
  }
  // L2P and P2P per sorted point
  const float w2 = w * w;
  for (uint32_t k = t; k < n; k += nt) {
    const uint32_t leaf = skeys[k] >> 14;
    uint32_t ix, iy;
    deinterleave(leaf, ix, iy);
    const float cx = (ix + 0.5f) * sL, cy = (iy + 0.5f) * sL;
    const float2 z = make_float2((S.sx[k] - cx) * side, (S.sy[k] - cy) * side);
    const float2 *Lc = S.L + (size_t)(leaf0 + leaf) * BQ;
    float2 phi = Lc[BQ - 1];
    for (int l = BQ - 2; l >= 0; --l) {
      phi = cmul(phi, z);
      phi.x += Lc[l].x;
      phi.y += Lc[l].y;
    }
    // phi / s_L in scaled units; the world kick divides by w
    float kx = -phi.x * side * (1.f / w), ky = phi.y * side * (1.f / w);
    const float xi = S.sx[k], yi = S.sy[k];
    for (int o = 0; o < BNEAR; ++o) {
      const int bx = (int)ix + T.near_dx[o], by = (int)iy + T.near_dy[o];
      if (bx < 0 || by < 0 || bx >= (int)side || by >= (int)side) continue;
      const uint32_t cb = interleave(bx, by);
      for (uint32_t j = S.leaf_start[cb]; j < S.leaf_start[cb + 1]; ++j) {
        if (j == k) continue;
        float dx = (S.sx[j] - xi) * w, dy = (S.sy[j] - yi) * w;
        float l = dx * dx + dy * dy;
        if (dx == 0.f || dy == 0.f) {
          const uint64_t seed = 0x5DEECE66Dull * (a.tick + 1);
          if (dx == 0.f) {
            dx = (float)hash_jiggle(seed, S.sidx[k], S.sidx[j], 0);
            l += dx * dx;
          }
          if (dy == 0.f) {
            dy = (float)hash_jiggle(seed, S.sidx[k], S.sidx[j], 1);
            l += dy * dy;
          }
        }
        if (l < BDMIN2) l = sqrtf(BDMIN2 * l);
        const float s = S.ss[j] / l;
        kx += dx * s;
        ky += dy * s;
      }
    }
    (void)w2;
    const uint32_t i = S.sidx[k];
    if (a.kick_out) {
      a.kick_out[n0 + i] = make_float2(kx, ky);
    } else {
      a.vx[n0 + i] += kx;
      a.vy[n0 + i] += ky;
    }
  }
  __syncthreads();
}

// link_fast.zig: each node adds its own side of each of its links, from the
// snapshot x + vx.
__device__ void graph_link(const BArgs &a, uint32_t n0, uint32_t n, const BScratch &S) {
  const uint32_t t = threadIdx.x, nt = blockDim.x;
  for (uint32_t i = t; i < n; i += nt) {
    S.px[i] = a.x[n0 + i] + a.vx[n0 + i];
    S.py[i] = a.y[n0 + i] + a.vy[n0 + i];
  }
  __syncthreads();
  for (uint32_t i = t; i < n; i += nt) {
    float dvx = 0, dvy = 0;
    for (uint32_t e = a.adj_off[n0 + i]; e < a.adj_off[n0 + i + 1]; ++e) {
      const uint32_t j = a.adj_j[e];
      const float4 wv = a.adj_w[e];  // strength, distance, own share, sign
      // the link's vector target - source
      float dx = (S.px[j] - S.px[i]) * wv.w, dy = (S.py[j] - S.py[i]) * wv.w;
      if (dx == 0.f) dx = (float)hash_jiggle(0x9E37ull * (a.tick + 1), min(i, j), max(i, j), 2);
      if (dy == 0.f) dy = (float)hash_jiggle(0x9E37ull * (a.tick + 1), min(i, j), max(i, j), 3);
      const float l = sqrtf(dx * dx + dy * dy);
      const float f = (l - wv.y) / l * a.alpha * wv.x;
      // target: v -= d f b; source: v += d f (1 - b)  (the sign picks the side)
      dvx += wv.w * dx * f * wv.z;
      dvy += wv.w * dy * f * wv.z;
    }
    a.vx[n0 + i] += dvx;
    a.vy[n0 + i] += dvy;
  }
  __syncthreads();
}

// grid.zig: radius 3 for every node, strength 1; Jacobi from the snapshot.
__device__ void graph_collide(const BArgs &a, uint32_t n0, uint32_t n, const BScratch &S,
                              uint32_t *skeys, float *red) {
  const uint32_t t = threadIdx.x, nt = blockDim.x;
  float mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
  for (uint32_t i = t; i < n; i += nt) {
    const float x = a.x[n0 + i] + a.vx[n0 + i], y = a.y[n0 + i] + a.vy[n0 + i];
    S.px[i] = x;
    S.py[i] = y;
    mnx = fminf(mnx, x);
    mxx = fmaxf(mxx, x);
    mny = fminf(mny, y);
    mxy = fmaxf(mxy, y);
  }
  mnx = block_reduce(mnx, false, red);
  mxx = block_reduce(mxx, true, red);
  mny = block_reduce(mny, false, red);
  mxy = block_reduce(mxy, true, red);
  const float r = BRADIUS, r2 = 2 * r;
  // cell side 2r, coarsened until the grid has at most 4n + 16 cells
  float h = r2;
  uint32_t gx = 1, gy = 1;
  for (int it = 0; it < 64; ++it) {
    gx = (uint32_t)fminf((mxx - mnx) / h, 1e6f) + 1;
    gy = (uint32_t)fminf((mxy - mny) / h, 1e6f) + 1;
    if ((uint64_t)gx * gy <= 4ull * n + 16 && (uint64_t)gx * gy < (1u << 18)) break;
    h *= 2;
  }
  const float inv_h = 1.f / h;
  uint32_t P = 64;
  while (P < n) P <<= 1;
  for (uint32_t i = t; i < P; i += nt) {
    uint32_t key = 0xFFFFFFFFu;
    if (i < n) {
      const uint32_t cx = min(gx - 1, (uint32_t)((S.px[i] - mnx) * inv_h));
      const uint32_t cy = min(gy - 1, (uint32_t)((S.py[i] - mny) * inv_h));
      key = ((cy * gx + cx) << 14) | i;
    }
    skeys[i] = key;
  }
  __syncthreads();
  bitonic(skeys, P);
  const float rr = r2 * r2;
  for (uint32_t i = t; i < n; i += nt) {
    const float xi = S.px[i], yi = S.py[i];
    const int cx = (int)min(gx - 1, (uint32_t)((xi - mnx) * inv_h));
    const int cy = (int)min(gy - 1, (uint32_t)((yi - mny) * inv_h));
    float dvx = 0, dvy = 0;
    for (int oy = -1; oy <= 1; ++oy)
      for (int ox = -1; ox <= 1; ++ox) {
        const int bx = cx + ox, by = cy + oy;
        if (bx < 0 || by < 0 || bx >= (int)gx || by >= (int)gy) continue;
        const uint32_t cell = (uint32_t)by * gx + (uint32_t)bx;
        for (uint32_t k = lower(skeys, n, cell << 14); k < n && (skeys[k] >> 14) == cell; ++k) {
          const uint32_t j = skeys[k] & 0x3FFFu;
          if (j == i) continue;
          float dx = xi - S.px[j], dy = yi - S.py[j];
          float l = dx * dx + dy * dy;
          if (!(l < rr)) continue;
          if (dx == 0.f || dy == 0.f) {
            const uint64_t seed = 0xC2B2AE35ull * (a.tick + 1);
            const float sg = i < j ? 1.f : -1.f;  // the pair's two sides push apart
            if (dx == 0.f) {
              dx = sg * (float)hash_jiggle(seed, min(i, j), max(i, j), 4);
              l += dx * dx;
            }
            if (dy == 0.f) {
              dy = sg * (float)hash_jiggle(seed, min(i, j), max(i, j), 5);
              l += dy * dy;
            }
          }
          l = sqrtf(l);
          const float push = (r2 - l) / l * 0.5f;  // equal radii: an even share
          dvx += dx * push;
          dvy += dy * push;
        }
      }
    a.vx[n0 + i] += dvx;
    a.vy[n0 + i] += dvy;
  }
  __syncthreads();
}

__global__ void k_batch_tick(BArgs a) {
  extern __shared__ unsigned char b_smem[];
  BTables &T = *reinterpret_cast<BTables *>(b_smem);
  uint32_t *skeys = reinterpret_cast<uint32_t *>(b_smem + ((sizeof(BTables) + 15) / 16) * 16);
  __shared__ float red[32];
  __shared__ uint32_t next;
  // the tables into shared memory
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(a.tab);
    uint4 *dst = reinterpret_cast<uint4 *>(b_smem);
    for (uint32_t k = threadIdx.x; k < sizeof(BTables) / 16; k += blockDim.x) dst[k] = src[k];
  }
  const BScratch S = scratch_of(a);
  __syncthreads();
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(a.queue, 1u);
    __syncthreads();
    const uint32_t pos = next;
    __syncthreads();
    if (pos >= a.graphs) break;
    const uint32_t g = a.order[pos];
    const uint32_t n0 = a.node_off[g], n = a.node_off[g + 1] - n0;
    if (n == 0) continue;
    graph_many_body(a, T, g, n0, n, S, skeys, red);
    if (a.kick_out) continue;
    graph_link(a, n0, n, S);
    graph_collide(a, n0, n, S, skeys, red);
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      const float vx = a.vx[n0 + i] * 0.6f, vy = a.vy[n0 + i] * 0.6f;
      a.vx[n0 + i] = vx;
      a.vy[n0 + i] = vy;
      a.x[n0 + i] += vx;
      a.y[n0 + i] += vy;
    }
    __syncthreads();
  }
}

// ---- host ------------------------------------------------------------------------------------

double binom_h(int n, int k) {
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

struct Cx {
  double re, im;
};
Cx cx_mul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

void build_btables(BTables &T) {
  memset(&T, 0, sizeof T);
  const double k2 = 2 * 1.5 * 1.5;
  auto sep = [&](int x, int y) { return (double)(x * x + y * y) >= k2; };
  int nn = 0;
  for (int y = -2; y <= 2; ++y)
    for (int x = -2; x <= 2; ++x)
      if (!sep(x, y)) {
        T.near_dx[nn] = (int8_t)x;
        T.near_dy[nn] = (int8_t)y;
        ++nn;
      }
  std::vector<std::pair<int, int>> classes;
  for (int aq = 0; aq < 4; ++aq) {
    const int ax = aq & 1, ay = aq >> 1;
    int ns = 0;
    for (int o = 0; o < nn; ++o)
      for (int b = 0; b < 4; ++b) {
        const int vx = 2 * T.near_dx[o] + (b & 1) - ax, vy = 2 * T.near_dy[o] + (b >> 1) - ay;
        if (!sep(vx, vy)) continue;
        size_t c = 0;
        while (c < classes.size() && !(classes[c].first == vx && classes[c].second == vy)) ++c;
        if (c == classes.size()) classes.push_back({vx, vy});
        T.slot_dx[aq][ns] = (int8_t)vx;
        T.slot_dy[aq][ns] = (int8_t)vy;
        T.slot_class[aq][ns] = (uint8_t)c;
        ++ns;
      }
  }
  for (size_t c = 0; c < classes.size(); ++c) {
    // z0 = c_A - c_B = -(B - A)
    const Cx v{-(double)classes[c].first, -(double)classes[c].second};
    const double d2 = v.re * v.re + v.im * v.im;
    const Cx inv{v.re / d2, -v.im / d2};
    Cx pw[2 * BQ + 2];
    pw[0] = {1, 0};
    for (int e = 1; e < 2 * BQ + 2; ++e) pw[e] = cx_mul(pw[e - 1], inv);
    for (int l = 0; l < BQ; ++l)
      for (int k = 0; k < BQ; ++k) {
        const double f = ((l & 1) ? -1.0 : 1.0) * binom_h(k + l, l);
        T.k[c][l][k] = make_float2((float)(f * pw[k + l + 1].re), (float)(f * pw[k + l + 1].im));
      }
  }
  for (int b = 0; b < 4; ++b) {
    const Cx delta{(double)(2 * (b & 1) - 1), (double)(2 * (b >> 1) - 1)};
    for (int nn2 = 0; nn2 < BQ; ++nn2)
      for (int k = 0; k <= nn2; ++k) {
        Cx p{1, 0};
        for (int e = 0; e < nn2 - k; ++e) p = cx_mul(p, delta);
        const double f = binom_h(nn2, k) * std::ldexp(1.0, -k) * std::ldexp(1.0, -2 * (nn2 - k));
        T.m2m[b][nn2][k] = make_float2((float)(f * p.re), (float)(f * p.im));
      }
    for (int mm = 0; mm < BQ; ++mm)
      for (int l = mm; l < BQ; ++l) {
        Cx p{1, 0};
        for (int e = 0; e < l - mm; ++e) p = cx_mul(p, delta);
        const double f = binom_h(l, mm) * std::ldexp(1.0, -2 * (l - mm)) * std::ldexp(1.0, -(mm + 1));
        T.l2l[b][mm][l] = make_float2((float)(f * p.re), (float)(f * p.im));
      }
  }
}

struct Batch {
  uint32_t graphs = 0, nodes = 0;
  std::vector<uint32_t> h_off, h_order;
  std::vector<uint8_t> h_level;
  std::vector<uint32_t> h_counts;
  BTables *tab = nullptr;
  uint32_t *order = nullptr, *node_off = nullptr, *adj_off = nullptr, *adj_j = nullptr;
  uint8_t *level = nullptr;
  float4 *adj_w = nullptr;
  float *x = nullptr, *y = nullptr, *vx = nullptr, *vy = nullptr, *scratch = nullptr;
  uint32_t *queues = nullptr;
  uint32_t queue_cap = 0;
  float2 *kick = nullptr;
  double alpha = 1, alpha_decay = 0;
  uint32_t tick = 0;
  int threads = 512, per_sm = 1, sms = 148;
  uint32_t leaf_size = 16;
  size_t scratch_ctas = 0;
  cudaStream_t st = nullptr;
  cudaGraphExec_t graph = nullptr;
  uint32_t graph_ticks = 0;
};

std::vector<Batch *> g_batches;

Batch *get_batch(uint32_t h) {
  return h >= 1 && h <= g_batches.size() ? g_batches[h - 1] : nullptr;
}

size_t smem_bytes() { return ((sizeof(BTables) + 15) / 16) * 16 + BSORT * 4; }

void set_levels(Batch &b) {
  b.h_level.resize(b.graphs);
  for (uint32_t g = 0; g < b.graphs; ++g) {
    int L = 2;
    while (L < BMAX_L && (double)b.h_counts[g] / (double)(1u << (2 * L)) > b.leaf_size) ++L;
    b.h_level[g] = (uint8_t)L;
  }
  cudaMemcpy(b.level, b.h_level.data(), b.graphs, cudaMemcpyHostToDevice);
}

int ensure_scratch(Batch &b) {
  const size_t ctas = (size_t)b.sms * b.per_sm;
  if (ctas <= b.scratch_ctas) return 0;
  cudaFree(b.scratch);
  b.scratch = nullptr;
  if (cudaMalloc(&b.scratch, ctas * scratch_floats() * 4) != cudaSuccess) return -1;
  b.scratch_ctas = ctas;
  return 0;
}

BArgs args_of(Batch &b, float alpha, uint32_t tick, uint32_t *queue, float2 *kick) {
  BArgs a;
  a.tab = b.tab;
  a.graphs = b.graphs;
  a.order = b.order;
  a.node_off = b.node_off;
  a.level = b.level;
  a.adj_off = b.adj_off;
  a.adj_j = b.adj_j;
  a.adj_w = b.adj_w;
  a.x = b.x; a.y = b.y; a.vx = b.vx; a.vy = b.vy;
  a.scratch = b.scratch;
  a.scratch_stride = scratch_floats();
  a.queue = queue;
  a.alpha = alpha;
  a.tick = tick;
  a.kick_out = kick;
  return a;
}

int launch_tick(Batch &b, float alpha, uint32_t tick, uint32_t *queue, float2 *kick) {
  BArgs a = args_of(b, alpha, tick, queue, kick);
  D3_LAUNCH(k_batch_tick, b.sms * b.per_sm, b.threads, smem_bytes(), b.st)(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int ensure_queues(Batch &b, uint32_t n) {
  if (n <= b.queue_cap) return 0;
  cudaFree(b.queues);
  b.queues = nullptr;
  if (cudaMalloc(&b.queues, (size_t)n * 4) != cudaSuccess) return -1;
  b.queue_cap = n;
  return 0;
}

}  // namespace
}  // namespace d3

using namespace d3;

extern "C" {

uint32_t batch_create(uint32_t graphs, const uint32_t *node_counts, const uint32_t *link_counts,
                      const uint32_t *src, const uint32_t *tgt, const float *x, const float *y) {
  if (graphs == 0 || !node_counts || !link_counts || !x || !y) return 0;
  Batch *b = new Batch();
  b->graphs = graphs;
  b->h_counts.assign(node_counts, node_counts + graphs);
  b->h_off.resize(graphs + 1, 0);
  size_t links = 0;
  for (uint32_t g = 0; g < graphs; ++g) {
    if (node_counts[g] > BMAX_N) {
      delete b;
      return 0;
    }
    b->h_off[g + 1] = b->h_off[g] + node_counts[g];
    links += link_counts[g];
  }
  const uint32_t N = b->h_off[graphs];
  b->nodes = N;
  // per-node adjacency: d3's default link strength 1 / min(degree) and bias
  // degree(source) / (degree(source) + degree(target)) (link.js:30-67)
  std::vector<uint32_t> deg(N, 0), adj_off(N + 1, 0), adj_j(2 * links);
  std::vector<float4> adj_w(2 * links);
  size_t e0 = 0;
  for (uint32_t g = 0; g < graphs; ++g) {
    for (uint32_t e = 0; e < link_counts[g]; ++e) {
      const uint32_t s = src[e0 + e], t = tgt[e0 + e];
      if (s >= node_counts[g] || t >= node_counts[g]) {
        delete b;
        return 0;
      }
      ++deg[b->h_off[g] + s];
      ++deg[b->h_off[g] + t];
    }
    e0 += link_counts[g];
  }
  for (uint32_t i = 0; i < N; ++i) adj_off[i + 1] = adj_off[i] + deg[i];
  std::vector<uint32_t> fill(adj_off.begin(), adj_off.end() - 1);
  e0 = 0;
  for (uint32_t g = 0; g < graphs; ++g) {
    const uint32_t o = b->h_off[g];
    for (uint32_t e = 0; e < link_counts[g]; ++e) {
      const uint32_t s = src[e0 + e], t = tgt[e0 + e];
      const float ds = (float)deg[o + s], dt = (float)deg[o + t];
      const float k = 1.f / fminf(ds, dt), bias = ds / (ds + dt);
      // an entry's sign turns (other - self) into d = target - source and
      // gives its side's direction: the target gets -d f bias, the source
      // +d f (1 - bias)
      adj_j[fill[o + t]] = s;
      adj_w[fill[o + t]++] = make_float4(k, BDIST, bias, -1.f);
      adj_j[fill[o + s]] = t;
      adj_w[fill[o + s]++] = make_float4(k, BDIST, 1.f - bias, 1.f);
    }
    e0 += link_counts[g];
  }
  // largest graphs first
  b->h_order.resize(graphs);
  for (uint32_t g = 0; g < graphs; ++g) b->h_order[g] = g;
  std::stable_sort(b->h_order.begin(), b->h_order.end(),
                   [&](uint32_t p, uint32_t q) { return node_counts[p] > node_counts[q]; });
  BTables T;
  build_btables(T);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  bool ok = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&b->tab, sizeof(BTables)) == cudaSuccess &&
            cudaMalloc(&b->order, graphs * 4) == cudaSuccess &&
            cudaMalloc(&b->node_off, (graphs + 1) * 4) == cudaSuccess &&
            cudaMalloc(&b->level, graphs) == cudaSuccess &&
            cudaMalloc(&b->adj_off, (N + 1) * 4ull) == cudaSuccess &&
            cudaMalloc(&b->adj_j, (2 * links + 1) * 4) == cudaSuccess &&
            cudaMalloc(&b->adj_w, (2 * links + 1) * sizeof(float4)) == cudaSuccess &&
            cudaMalloc(&b->x, N * 4ull) == cudaSuccess && cudaMalloc(&b->y, N * 4ull) == cudaSuccess &&
            cudaMalloc(&b->vx, N * 4ull) == cudaSuccess && cudaMalloc(&b->vy, N * 4ull) == cudaSuccess &&
            cudaMalloc(&b->kick, N * sizeof(float2)) == cudaSuccess;
  ok = ok && cudaMemcpy(b->tab, &T, sizeof T, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(b->order, b->h_order.data(), graphs * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(b->node_off, b->h_off.data(), (graphs + 1) * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(b->adj_off, adj_off.data(), (N + 1) * 4ull, cudaMemcpyHostToDevice) == cudaSuccess &&
       (links == 0 ||
        (cudaMemcpy(b->adj_j, adj_j.data(), 2 * links * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(b->adj_w, adj_w.data(), 2 * links * sizeof(float4), cudaMemcpyHostToDevice) ==
             cudaSuccess)) &&
       cudaMemcpy(b->x, x, N * 4ull, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(b->y, y, N * 4ull, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemset(b->vx, 0, N * 4ull) == cudaSuccess && cudaMemset(b->vy, 0, N * 4ull) == cudaSuccess;
  cudaFuncSetAttribute(k_batch_tick, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes());
  b->alpha_decay = 1 - std::pow(0.001, 1.0 / 300);
  if (ok) {
    set_levels(*b);
    ok = ensure_scratch(*b) == 0;
  }
  if (!ok) {
    delete b;
    return 0;
  }
  g_batches.push_back(b);
  return (uint32_t)g_batches.size();
}

int32_t batch_destroy(uint32_t h) {
  Batch *b = get_batch(h);
  if (!b) return D3_BAD_HANDLE;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->tab); cudaFree(b->order); cudaFree(b->node_off); cudaFree(b->level);
  cudaFree(b->adj_off); cudaFree(b->adj_j); cudaFree(b->adj_w); cudaFree(b->x); cudaFree(b->y);
  cudaFree(b->vx); cudaFree(b->vy); cudaFree(b->scratch); cudaFree(b->queues); cudaFree(b->kick);
  cudaStreamDestroy(b->st);
  delete b;
  g_batches[h - 1] = nullptr;
  return D3_OK;
}

// Launch shape: threads per CTA, CTAs per SM, target points per FMM leaf.
int32_t batch_set_shape(uint32_t h, uint32_t threads, uint32_t per_sm, uint32_t leaf_size) {
  Batch *b = get_batch(h);
  if (!b) return D3_BAD_HANDLE;
  if ((threads != 256 && threads != 512 && threads != 1024) || per_sm < 1 || per_sm > 2 ||
      leaf_size < 2 || leaf_size > 256)
    return D3_BAD_ARGUMENT;
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_tick, (int)threads, smem_bytes());
  if ((int)per_sm > per) return D3_BAD_ARGUMENT;
  b->threads = (int)threads;
  b->per_sm = (int)per_sm;
  b->leaf_size = leaf_size;
  set_levels(*b);
  if (ensure_scratch(*b)) return D3_OUT_OF_MEMORY;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_ticks = 0;
  }
  return D3_OK;
}

// Runs `ticks` ticks (d3's alpha schedule continues from the batch's
// state). graph != 0: the ticks are captured once into a CUDA graph (one
// kernel node per tick) and replayed. *ms: device time (CUDA events).
int32_t batch_run(uint32_t h, uint32_t ticks, uint32_t graph, double *ms) {
  Batch *b = get_batch(h);
  if (!b) return D3_BAD_HANDLE;
  if (ticks == 0) return D3_OK;
  if (ensure_queues(*b, ticks)) return D3_OUT_OF_MEMORY;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int32_t rc = D3_OK;
  // alphas of these ticks (simulation.js:64 per tick)
  std::vector<float> alphas(ticks);
  double al = b->alpha;
  for (uint32_t k = 0; k < ticks; ++k) {
    al += (0 - al) * b->alpha_decay;
    alphas[k] = (float)al;
  }
  if (cudaMemsetAsync(b->queues, 0, (size_t)ticks * 4, b->st) != cudaSuccess) rc = D3_WORKER_FAILED;
  if (graph && rc == D3_OK) {
    // a captured run is tied to its alphas and tick numbers: capture anew
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    cudaGraph_t gr = nullptr;
    if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      rc = D3_WORKER_FAILED;
    } else {
      for (uint32_t k = 0; k < ticks; ++k)
        if (launch_tick(*b, alphas[k], b->tick + k, b->queues + k, nullptr)) rc = D3_WORKER_FAILED;
      if (cudaStreamEndCapture(b->st, &gr) != cudaSuccess) rc = D3_WORKER_FAILED;
    }
    if (rc == D3_OK && cudaGraphInstantiate(&b->graph, gr, 0) != cudaSuccess) rc = D3_WORKER_FAILED;
    if (gr) cudaGraphDestroy(gr);
    if (rc == D3_OK) {
      cudaEventRecord(e0, b->st);
      if (cudaGraphLaunch(b->graph, b->st) != cudaSuccess) rc = D3_WORKER_FAILED;
      cudaEventRecord(e1, b->st);
    }
  } else if (rc == D3_OK) {
    cudaEventRecord(e0, b->st);
    for (uint32_t k = 0; k < ticks; ++k)
      if (launch_tick(*b, alphas[k], b->tick + k, b->queues + k, nullptr)) rc = D3_WORKER_FAILED;
    cudaEventRecord(e1, b->st);
  }
  if (cudaStreamSynchronize(b->st) != cudaSuccess) rc = D3_WORKER_FAILED;
  float f = 0;
  cudaEventElapsedTime(&f, e0, e1);
  if (ms) *ms = f;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == D3_OK) {
    b->alpha = al;
    b->tick += ticks;
  }
  return rc;
}

// The many-body kick alone (FMM, the batch's next alpha) at the current
// positions, per node (x, y pairs), into host `out` (2 x nodes floats).
int32_t batch_kick(uint32_t h, float *out, double *alpha_used) {
  Batch *b = get_batch(h);
  if (!b || !out) return b ? D3_BAD_ARGUMENT : D3_BAD_HANDLE;
  if (ensure_queues(*b, 1)) return D3_OUT_OF_MEMORY;
  const double al = b->alpha + (0 - b->alpha) * b->alpha_decay;
  if (alpha_used) *alpha_used = (float)al;
  if (cudaMemsetAsync(b->queues, 0, 4, b->st) != cudaSuccess ||
      launch_tick(*b, (float)al, b->tick, b->queues, b->kick) ||
      cudaMemcpyAsync(out, b->kick, b->nodes * sizeof(float2), cudaMemcpyDeviceToHost, b->st) !=
          cudaSuccess ||
      cudaStreamSynchronize(b->st) != cudaSuccess)
    return D3_WORKER_FAILED;
  return D3_OK;
}

int32_t batch_read(uint32_t h, float *x, float *y, float *vx, float *vy) {
  Batch *b = get_batch(h);
  if (!b) return D3_BAD_HANDLE;
  const size_t bytes = b->nodes * 4ull;
  if ((x && cudaMemcpy(x, b->x, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (y && cudaMemcpy(y, b->y, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (vx && cudaMemcpy(vx, b->vx, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (vy && cudaMemcpy(vy, b->vy, bytes, cudaMemcpyDeviceToHost) != cudaSuccess))
    return D3_WORKER_FAILED;
  return D3_OK;
}

// Autotuner: times `ticks` ticks (from a copy of the current state, which is
// restored) for every launch shape - threads 256 / 512 / 1024, 1 or 2 CTAs
// per SM where they fit, leaf sizes 8 / 16 / 32 - and keeps the fastest.
// out[0..3]: threads, CTAs per SM, leaf size, ms per tick of the choice.
int32_t batch_autotune(uint32_t h, uint32_t ticks, double *out) {
  Batch *b = get_batch(h);
  if (!b) return D3_BAD_HANDLE;
  const size_t bytes = b->nodes * 4ull;
  float *save = nullptr;
  if (cudaMalloc(&save, 4 * bytes) != cudaSuccess) return D3_OUT_OF_MEMORY;
  float *arr[4] = {b->x, b->y, b->vx, b->vy};
  for (int k = 0; k < 4; ++k) cudaMemcpy(save + k * b->nodes, arr[k], bytes, cudaMemcpyDeviceToDevice);
  const double alpha0 = b->alpha;
  const uint32_t tick0 = b->tick;
  double best = 1e30;
  uint32_t bt = 512, bp = 1, bl = 16;
  int32_t rc = D3_OK;
  for (uint32_t th : {256u, 512u, 1024u})
    for (uint32_t ps : {1u, 2u})
      for (uint32_t ls : {8u, 16u, 32u}) {
        if (batch_set_shape(h, th, ps, ls) != D3_OK) continue;
        double ms = 0;
        if (batch_run(h, 1, 0, &ms) != D3_OK || batch_run(h, ticks, 0, &ms) != D3_OK) {
          rc = D3_WORKER_FAILED;
          break;
        }
        ms /= ticks;
        if (ms < best) {
          best = ms;
          bt = th;
          bp = ps;
          bl = ls;
        }
        for (int k = 0; k < 4; ++k)
          cudaMemcpy(arr[k], save + k * b->nodes, bytes, cudaMemcpyDeviceToDevice);
        b->alpha = alpha0;
        b->tick = tick0;
      }
  cudaFree(save);
  if (rc != D3_OK) return rc;
  batch_set_shape(h, bt, bp, bl);
  if (out) {
    out[0] = bt;
    out[1] = bp;
    out[2] = bl;
    out[3] = best;
  }
  return D3_OK;
}

}  // extern "C"
