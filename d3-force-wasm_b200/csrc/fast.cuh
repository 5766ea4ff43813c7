// fast.cuh — fast mode (precision 'fast', n >= 2000): FMM many-body, uniform
// grid collide, Jacobi link (fmm.zig, grid.zig, link_fast.zig).
#pragma once

#include "common.cuh"
#include "forces.cuh"
#include "tree.cuh"

namespace d3 {

constexpr uint32_t FAST_MIN_N = 2000;  // fmm.zig:43

struct FastScratch {
  uint32_t cap = 0;
  double *seed = nullptr;  // the running force's SEED (f64 bits = hash seed)
  // grid collide
  uint64_t *g_keys = nullptr, *g_keys_tmp = nullptr;
  uint32_t *g_items = nullptr, *g_items_tmp = nullptr, *g_cell_of = nullptr, *g_start = nullptr;
  uint32_t *g_hist = nullptr, *g_part = nullptr;
  double *g_box = nullptr;      // per-block partial bounds
  uint32_t *g_info = nullptr;   // grid geometry: gx, gy, cells, m, active, ticket
  double *g_geom = nullptr;     // x0, y0, inv_h
  // FMM
  void *fmm = nullptr;
  void *fmm_tc = nullptr;  // the precision forms' state
  // the learned form's sampled check: tolerance on the RMS of the sampled
  // kicks, sample count, ticks on the fallback after a failed check; counters
  double learn_tol = 1e-5;
  uint32_t learn_samples = 64, learn_hold = 0;
  double learn_checks = 0, learn_fallbacks = 0, learn_last_rms = 0;
};

int fast_reserve(FastScratch &s, uint32_t n);
void fast_free(FastScratch &s);

// The per-run SEED: one draw from the device LCG (src/core.js:221), or a
// value the host drew from the caller's random function.
void draw_seed(Rng *rng, double *seed, cudaStream_t st);
void set_seed(double *seed, double value, cudaStream_t st);

// link_fast.zig: CSR adjacency (edge id, TARGET_BIT on the target's entry),
// rows filled from the back so each row lists its edges in descending order.
// The fast link's adjacency (CSR over nodes, link_fast.zig:105-130) and, in
// the same adjacency order, each entry's other endpoint and its link's
// distance, strength and bias (copied from the link arrays once per
// rebuild), so a node's links are read contiguously.
struct FastLink {
  uint32_t n = 0, m = 0;
  uint32_t *row = nullptr, *adj = nullptr;
  uint32_t *other = nullptr;   // per adjacency entry
  double *scal = nullptr;      // per adjacency entry: distance, strength, bias planes
  bool gathered = false;       // scal holds the current link arrays
};
int fast_link_build(FastLink &c, const uint32_t *src, const uint32_t *tgt, uint32_t m, uint32_t n);
void fast_link_free(FastLink &c);
void fast_link(const NodeArrays &a, const LinkArrays &l, FastLink &c, double alpha,
               double iterations, const double *seed, cudaStream_t st);

// grid.zig:198-286
void fast_collide(FastScratch &s, const NodeArrays &a, const double *radii, double strength,
                  double iterations, const double *seed, cudaStream_t st);

struct FmmParams {
  double order, opening, dmin2, dmax2, alpha;
};

// fmm.zig:68-78 (a cell of the fast tree, level order, children contiguous),
// with the parent index in the spare word.
struct FCell {
  double cx, cy, r;
  uint32_t first, count, child0, nchild, depth, parent;
};

// What fmm_prepare leaves on the device for the passes of a fast many-body
// run: the points in key order (fmm.zig:668-682: positions, strength x alpha,
// scaled positions (x - ox) / w), the level-order cells and their levels.
struct FmmPrep {
  uint32_t m = 0, ncells = 0, nlev = 0;
  uint32_t lvl[20] = {};  // first cell of each level (host copy)
  double w = 0, inv_w = 0, ox = 0, oy = 0;
  const uint64_t *keys = nullptr;
  const uint32_t *perm = nullptr;
  const double *px = nullptr, *py = nullptr, *ps = nullptr, *ux = nullptr, *uy = nullptr;
  FCell *cells = nullptr;
  uint32_t *info = nullptr;  // device: FI_LVL + d = first cell of level d
  int coop_blocks = 0;
};

// The fast tree of fmm.zig:247-330 up to the cells: square extent, 16-bit
// Morton keys, stable sort, gather, level-order cells (fmm.zig:685-717).
// 1: ready; 2: no point to act on; 0: non-finite extent (the exact kernel
// runs instead); < 0: failure.
int fmm_prepare(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
                double alpha, FmmPrep &out, cudaStream_t st);

// The precision forms of the fast many-body force (no reference
// counterpart; judged by RMS against an FP64 direct sum): geometric cells,
// M2L as batched dense BF16x3 contractions on the tensor cores, FP32 near
// field with a per-leaf FP64 origin shift. form 2: order `order`; form 3:
// order 4 plus the learned per-leaf correction. Returns as fmm_run.
int fmm_tc_run(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
               const FmmParams &p, int form, const double *seed, uint32_t *status,
               cudaStream_t st);
void fmm_tc_free(FastScratch &s);
// Installs the learned form's network (MLP_PARAMS floats, host): 0, or < 0.
int fmm_tc_set_learned(FastScratch &s, const float *params, uint32_t len);
// The last precision-form run's per-cell rows (16 floats: features, L'_0, sc,
// the cell index for leaves or -1) into out when cap >= the cell count;
// returns the cell count.
int fmm_tc_leaves(FastScratch &s, float *out, uint32_t cap);
// out[12]: checks, fallbacks, last sampled RMS, cells of the last run; the
// last pass's M2L and P2P milliseconds (CUDA events), its M2L tiles, its work
// counts (M2L pairs, P2P point pairs, M2P and P2L point-cell pairs) and q.
// The precision forms' counters (TC_STATS doubles): 0 learned-form checks,
// 1 fallbacks, 2 the last check's RMS, 3 cells; the last pass: 4 M2L ms,
// 5 near-field (P2P) ms, 6 M2L tiles, 7 M2L pairs, 8 P2P point pairs, 9 M2P
// and 10 P2L point-cell pairs, 11 q; the last run's ms: 12 prepare,
// 13 geometry and lists, 14 upward, 15 P2L, 16 downward, 17 the learned
// form's network, 18 the whole run, 19 the far field (L2P, M2P, the kick).
constexpr int TC_STATS = 20;
void fmm_tc_stats(FastScratch &s, double *out);
// fmm.zig:247-354. Returns 1 when applied, 0 when the exact kernel must run
// instead (non-finite extent), < 0 on failure.
int fmm_run(FastScratch &s, TreeDev &t, const NodeArrays &a, const double *strengths,
            const FmmParams &p, const double *seed, uint32_t *status, cudaStream_t st);

}  // namespace d3
