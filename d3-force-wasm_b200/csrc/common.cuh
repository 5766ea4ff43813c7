// common.cuh — shared types and helpers of the B200 d3-force engine.
//
// Every translation unit is compiled with -fmad=false -prec-div=true
// -prec-sqrt=true -ftz=false: exact mode must reproduce d3-force's f64
// arithmetic bit for bit (no contraction into FMA, IEEE division and square
// root, subnormals kept), as the reference's `@setFloatMode(.strict)` and
// wasm's lack of a fused multiply-add do.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#include "../../include/d3force_b200.h"

namespace d3 {

constexpr uint32_t NONE = 0xffffffffu;
constexpr int KEY_LEVELS = 32;     // tree.zig:30
constexpr uint32_t MAX_DEPTH = 2200;  // tree.zig:33
constexpr int SM_COUNT_B200 = 148;

// Device status word bits (per simulation): set by kernels, read by the host.
enum : uint32_t {
  ST_LINK_JIGGLE = 1u << 0,      // a DAG link pass met a zero / NaN delta
  ST_COLLIDE_SPEC_FAIL = 1u << 1,  // a speculative collide pass failed validation
  ST_COLLIDE_JIGGLE = 1u << 2,   // a speculative collide pass met a zero delta
  ST_DEEP_STACK = 1u << 3,       // a traversal stack would overflow its buffer
  ST_WAIT_TIMEOUT = 1u << 4,     // a bounded device wait expired
  ST_RNG_NEED = 1u << 5,         // a serial kernel needs more host draws
  ST_COLLIDE_OVERFLOW = 1u << 6, // a guessed set exceeded its capacity
  ST_CENTER_RECORDS = 1u << 7,   // a center-sum launch failed or its records disagreed
  ST_LAUNCH_FAILED = 1u << 8,    // a kernel launch the pass depends on did not happen
};

// Device-side failures (a bounded wait that ran out, a tree or record buffer
// too small, a launch that did not happen): the results are not to be trusted.
constexpr uint32_t ST_FATAL = ST_WAIT_TIMEOUT | ST_DEEP_STACK | ST_CENTER_RECORDS | ST_LAUNCH_FAILED;

// One quadtree cell, the reference's 88-byte record (tree.zig:46-62):
// child[4], first, count, d3's x0 y0 x1 y1, per-force x, y, value, r.
struct Cell {
  uint32_t child[4];
  uint32_t first, count;
  double x0, y0, x1, y1;
  double x, y, value, r;
};
static_assert(sizeof(Cell) == 88, "cell layout");

__host__ __device__ inline bool is_leaf(const Cell &c) {
  return c.child[0] == NONE && c.child[1] == NONE && c.child[2] == NONE && c.child[3] == NONE;
}

// d3's LCG (src/lcg.js:1-9): s' = (a s + c) mod 2^32, value s' / 2^32.
__host__ __device__ inline double lcg_value(uint32_t s) { return (double)s / 4294967296.0; }
__host__ __device__ inline uint32_t lcg_step(uint32_t s) { return 1664525u * s + 1013904223u; }
// The state after k steps: s_k = A_k s + C_k (mod 2^32), by squaring.
__host__ __device__ inline uint32_t lcg_skip(uint32_t s, uint64_t k) {
  uint32_t a = 1664525u, c = 1013904223u;  // one step
  uint32_t A = 1u, Cc = 0u;                // accumulated
  while (k) {
    if (k & 1) {
      A = a * A;
      Cc = a * Cc + c;
    }
    c = a * c + c;
    a = a * a;
    k >>= 1;
  }
  return A * s + Cc;
}

// hash.zig:10-25 (splitmix64 finaliser) for fast-mode jiggle.
__host__ __device__ inline uint64_t hash_mix(uint64_t seed, uint32_t i, uint32_t j, uint32_t salt) {
  uint64_t h = seed ^ (((uint64_t)i << 32) | j) ^ ((uint64_t)salt * 0x9E3779B97F4A7C15ull);
  h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
  h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
  return h ^ (h >> 31);
}
__host__ __device__ inline double hash_jiggle(uint64_t seed, uint32_t i, uint32_t j, uint32_t salt) {
  return ((double)(hash_mix(seed, i, j, salt) >> 11) * 0x1.0p-53 - 0.5) * 1e-6;
}

// Random stream state on the device: d3's LCG, or a buffer of draws the host
// pulled from the caller's random function in d3's order.
struct Rng {
  uint32_t lcg;        // LCG state (LCG mode)
  uint32_t mode;       // 0 LCG, 1 host buffer
  uint64_t pos;        // draws consumed from the buffer (host mode)
  uint64_t avail;      // draws in the buffer (host mode)
  const double *buf;   // host-pulled draws (device memory)
};

// The value of draw number `k` from `state`'s stream position.
__device__ inline double rng_draw_at(const Rng &r, uint64_t k) {
  if (r.mode == 0) return lcg_value(lcg_step(lcg_skip(r.lcg, k)));
  return r.buf[r.pos + k];
}

#define D3_CUDA_OK(expr)                                                             \
  do {                                                                              \
    cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      fprintf(stderr, "d3force_b200: %s at %s:%d: %s\n", #expr, __FILE__, __LINE__, \
              cudaGetErrorString(e_));                                              \
      return D3_OUT_OF_MEMORY;                                                      \
    }                                                                               \
  } while (0)

// Kernels this library has launched (every launch site goes through
// D3_LAUNCH); the benchmark reports how many ran in its timed region.
extern unsigned long long g_launches;
#define D3_LAUNCH(kernel, ...) \
  for (int d3_launch_once_ = (++::d3::g_launches, 0); d3_launch_once_ < 1; ++d3_launch_once_) \
  kernel<<<__VA_ARGS__>>>

inline unsigned blocks_for(size_t n, unsigned threads) {
  size_t b = (n + threads - 1) / threads;
  return b ? (unsigned)b : 1u;
}

// The pause between polls of a device wait after its first few polls, in
// nanoseconds: 64, or D3_WAIT_SLEEP_NS (0 .. 1000; 0 = poll without pausing).
inline unsigned wait_sleep_ns() {
  static const unsigned v = [] {
    const char *e = getenv("D3_WAIT_SLEEP_NS");
    const int x = e ? atoi(e) : 64;
    return (unsigned)(x < 0 ? 0 : x > 1000 ? 1000 : x);
  }();
  return v;
}

}  // namespace d3
