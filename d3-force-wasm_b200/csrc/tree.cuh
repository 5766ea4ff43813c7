// tree.cuh — the d3-quadtree-identical tree, built on the device.
#pragma once

#include "common.cuh"
#include "scan_sort.cuh"

namespace d3 {

// A frame of the below-key-resolution split (tree.zig:64-76).
struct Frame {
  uint32_t lo, hi, depth, parent, slot, pad;
  double x0, y0, x1, y1;
};

// Tree scratch and result, all device memory. Cells are in d3's `visit`
// (pre)order, children 0..3; skip[c] is the index just past c's subtree, so a
// traversal that does not descend into c continues at skip[c].
struct TreeDev {
  uint32_t cap = 0;        // points
  uint32_t cells_cap = 0;  // cells
  uint64_t *keys = nullptr, *keys_tmp = nullptr;
  uint32_t *sv = nullptr, *sv_tmp = nullptr;  // sort values (node | invalid bit)
  uint32_t *perm = nullptr, *perm_tmp = nullptr;
  int8_t *lcpx = nullptr;      // per sorted position: levels shared with the previous key
  uint32_t *cnt = nullptr;     // cells starting at each sorted position
  uint32_t *base = nullptr;    // exclusive scan of cnt
  uint32_t *run_end = nullptr; // per start: end of its equal-position run / deep group
  uint8_t *leafd = nullptr;    // per start: depth of its leaf (33 = below key resolution)
  Frame *frames = nullptr;     // 4 frames per point for the deep splits
  Cell *cells = nullptr;
  uint32_t *skip = nullptr, *parent = nullptr, *counter = nullptr;
  uint8_t *pnch = nullptr;       // per cell: how many children its parent has
  void *rec = nullptr;           // per cell: the current traversal's 64-byte record
  uint32_t *leaf_of = nullptr;   // per node: the leaf cell holding it (NONE: NaN coordinate)
  uint32_t *box_part = nullptr;  // per-block bbox partials
  uint32_t *scan_part = nullptr;
  uint32_t *hist = nullptr;
  double *extent = nullptr;      // 4
  uint32_t *info = nullptr;      // 0 m, 1 cells, 2 depth, 3 root, 4 ticket, 5 overflow
  unsigned long long *stamps = nullptr;  // the last build's phase ends (globaltimer ns)
};

// Grid blocks of the build's cooperative launch (at most).
constexpr uint32_t TREE_GRID_MAX = 592;

// Words of t.hist: the build's per-tile digit counts (256 keys a tile) for
// two passes, digit totals and grid partials; also enough for
// radix_sort_u64's histograms.
inline size_t tree_hist_words(uint32_t n) {
  const size_t tiles = (n + 255) / 256 + 1;
  const size_t a = 2 * tiles * 256 + 256 + TREE_GRID_MAX;
  const size_t b = sort_hist_words(n);
  return a > b ? a : b;
}

int tree_reserve(TreeDev &t, uint32_t n);
void tree_free(TreeDev &t);

// Builds the tree over (xs, ys)[0..n) on stream st. Leaves the result in t
// (info[] on the device). No host synchronisation.
void tree_build(TreeDev &t, const double *xs, const double *ys, uint32_t n, uint32_t *status,
                cudaStream_t st);
// The same over the points (xs + vxs, ys + vys), which it also writes to
// (pxs, pys).
void tree_build_shifted(TreeDev &t, const double *xs, const double *ys, const double *vxs,
                        const double *vys, double *pxs, double *pys, uint32_t n, uint32_t *status,
                        cudaStream_t st);

// Fast mode's square extent (tree.zig:287-309): t.extent, t.info[0] = points
// without a NaN coordinate, and square[0..2] = box x0, y0, side.
void fast_box(TreeDev &t, const double *xs, const double *ys, uint32_t n, double *square,
              cudaStream_t st);

}  // namespace d3
