// noalloc.cu — exact many-body force on caller-owned device buffers, with
// every scratch array taken from one static device array: the call itself
// allocates no memory.
//
// Some callers cannot let a library allocate device memory: an engine that
// owns and budgets all GPU memory itself, a frame or control loop where
// cudaMalloc / cudaFree would add synchronisation and unbounded latency, or a
// process that must not grow its footprint after start-up. For them
// d3_many_body_exact_noalloc runs the same kernels as force_run of an exact
// many-body force (the tree build, the accumulation, the traversal and the
// jiggle rerun), but carves the tree and traversal scratch out of
// `g_noalloc_scratch`, a file-scope __device__ array sized for
// D3_NOALLOC_MAX_NODES nodes. Every GPU that loads the library holds that
// array until the process exits.
#include <mutex>

#include "forces.cuh"
#include "scan_sort.cuh"
#include "tree.cuh"

namespace d3 {
namespace {

constexpr uint32_t NA_CAP = D3_NOALLOC_MAX_NODES;
constexpr uint32_t NA_CELLS = 4 * NA_CAP + 1024;  // as tree_reserve
constexpr size_t NA_ALIGN = 256;
constexpr size_t na_round(size_t b) { return (b + NA_ALIGN - 1) / NA_ALIGN * NA_ALIGN; }
// the tree build's per-tile digit counts, digit totals and grid partials
constexpr size_t na_hist_words = 2 * ((NA_CAP + 255) / 256 + 1) * 256 + 256 + TREE_GRID_MAX;
constexpr size_t na_scan_words(size_t n) { return (n + SCAN_BLOCK * 4 - 1) / (SCAN_BLOCK * 4) + 2; }
constexpr size_t NA_BOX_BYTES = 592 * 64;  // per-block bounding-box partials of k_box

// Byte sizes of the carved arrays, in carve order.
constexpr size_t NA_SIZES[] = {
    8ull * NA_CAP, 8ull * NA_CAP,                 // keys, keys_tmp
    4ull * NA_CAP, 4ull * NA_CAP,                 // sv, sv_tmp
    4ull * NA_CAP, 4ull * NA_CAP,                 // perm, perm_tmp
    NA_CAP,                                       // lcpx
    4ull * (NA_CAP + 1), 4ull * (NA_CAP + 1),     // cnt, base
    4ull * NA_CAP, NA_CAP,                        // run_end, leafd
    4ull * NA_CAP * sizeof(Frame),                // frames
    (size_t)NA_CELLS * sizeof(Cell),              // cells
    4ull * NA_CELLS, 4ull * NA_CELLS, 4ull * NA_CELLS,  // skip, parent, counter
    (size_t)NA_CELLS, 64ull * NA_CELLS,           // pnch, rec
    4ull * NA_CAP,                                // leaf_of
    NA_BOX_BYTES,                                 // box partials
    4 * na_scan_words(na_hist_words > NA_CAP + 1 ? na_hist_words : NA_CAP + 1),  // tree scan
    4 * na_hist_words,                            // hist
    4 * sizeof(double), 16 * sizeof(uint32_t),    // extent, info
    4ull * (NA_CAP + 1), 4ull * (NA_CAP + 1),     // draws, offsets
    4 * (na_scan_words(NA_CAP + 1) > 1024 ? na_scan_words(NA_CAP + 1) : 1024),  // force scan
    16 * sizeof(uint32_t), 2 * sizeof(double),    // counters, center
    sizeof(Rng), 16 * sizeof(uint32_t),           // rng, status words
    16 * sizeof(unsigned long long),              // tree build phase stamps
};

constexpr size_t na_total() {
  size_t t = 0;
  for (size_t b : NA_SIZES) t += na_round(b);
  return t;
}

}  // namespace

// The scratch every d3_many_body_exact_noalloc call shares.
static __device__ __align__(256) unsigned char g_noalloc_scratch[na_total()];

namespace {

// Host-side addresses of g_noalloc_scratch per device (from
// cudaGetSymbolAddress; the symbol's host name is not a device address),
// each looked up once, under its own once_flag, so two threads making their
// first call at the same time do not race on it.
constexpr int NA_DEVICES = 128;
void *g_noalloc_base[NA_DEVICES] = {};
cudaError_t g_noalloc_setup_err[NA_DEVICES] = {};
std::once_flag g_noalloc_once[NA_DEVICES];

struct Carve {
  unsigned char *p;
  int k = 0;
  template <typename T>
  T *take() {
    T *r = reinterpret_cast<T *>(p);
    p += na_round(NA_SIZES[k++]);
    return r;
  }
};

__global__ void k_noalloc_rng_in(Rng *rng, uint32_t lcg) {
  Rng r;
  r.lcg = lcg;
  r.mode = 0;
  r.pos = 0;
  r.avail = 0;
  r.buf = nullptr;
  *rng = r;
}

__global__ void k_noalloc_out(const Rng *rng, const uint32_t *info, const uint32_t *status,
                              uint32_t *words) {
  words[0] = rng->lcg;
  words[1] = info[5];
  words[2] = status[0];
}

}  // namespace
}  // namespace d3

using namespace d3;

extern "C" int32_t d3_many_body_exact_noalloc(const double *x, const double *y, double *vx,
                                              double *vy, const double *strength, uint32_t n,
                                              double theta2, double distance_min2,
                                              double distance_max2, double alpha,
                                              uint32_t *lcg_state, void *stream) {
  if (n > NA_CAP) {
    fprintf(stderr, "d3_many_body_exact_noalloc: n = %u exceeds the maximum of %u nodes\n", n,
            NA_CAP);
    return D3_BAD_ARGUMENT;
  }
  if (!lcg_state || (n && (!x || !y || !vx || !vy || !strength))) return D3_BAD_ARGUMENT;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_DEVICES) return D3_WORKER_FAILED;
  // Set-up, once per device, with that device current.
  std::call_once(g_noalloc_once[dev], [dev] {
    void *base = nullptr;
    g_noalloc_setup_err[dev] = cudaGetSymbolAddress(&base, g_noalloc_scratch);
    if (g_noalloc_setup_err[dev] == cudaSuccess) g_noalloc_base[dev] = base;
  });
  if (g_noalloc_setup_err[dev] != cudaSuccess || !g_noalloc_base[dev]) return D3_WORKER_FAILED;
  Carve c{static_cast<unsigned char *>(g_noalloc_base[dev])};
  TreeDev t;
  t.cap = NA_CAP;
  t.cells_cap = NA_CELLS;
  t.keys = c.take<uint64_t>();
  t.keys_tmp = c.take<uint64_t>();
  t.sv = c.take<uint32_t>();
  t.sv_tmp = c.take<uint32_t>();
  t.perm = c.take<uint32_t>();
  t.perm_tmp = c.take<uint32_t>();
  t.lcpx = c.take<int8_t>();
  t.cnt = c.take<uint32_t>();
  t.base = c.take<uint32_t>();
  t.run_end = c.take<uint32_t>();
  t.leafd = c.take<uint8_t>();
  t.frames = c.take<Frame>();
  t.cells = c.take<Cell>();
  t.skip = c.take<uint32_t>();
  t.parent = c.take<uint32_t>();
  t.counter = c.take<uint32_t>();
  t.pnch = c.take<uint8_t>();
  t.rec = c.take<unsigned char>();
  t.leaf_of = c.take<uint32_t>();
  t.box_part = c.take<uint32_t>();
  t.scan_part = c.take<uint32_t>();
  t.hist = c.take<uint32_t>();
  t.extent = c.take<double>();
  t.info = c.take<uint32_t>();
  ForceScratch s;
  s.cap = NA_CAP;
  s.draws = c.take<uint32_t>();
  s.offsets = c.take<uint32_t>();
  s.scan_part = c.take<uint32_t>();
  s.counters = c.take<uint32_t>();
  s.center = c.take<double>();
  Rng *rng = c.take<Rng>();
  uint32_t *words = c.take<uint32_t>();  // 0 status, 8.. results
  t.stamps = c.take<unsigned long long>();

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The array keeps the previous call's contents: clear what must start at 0.
  cudaMemsetAsync(t.info, 0, 16 * sizeof(uint32_t), st);
  cudaMemsetAsync(s.counters, 0, 16 * sizeof(uint32_t), st);
  cudaMemsetAsync(words, 0, 16 * sizeof(uint32_t), st);
  D3_LAUNCH(k_noalloc_rng_in, 1, 1, 0, st)(rng, *lcg_state);
  NodeArrays a{};
  a.x = const_cast<double *>(x);
  a.y = const_cast<double *>(y);
  a.vx = vx;
  a.vy = vy;
  a.n = n;
  ManyBodyParams p{theta2, distance_min2, distance_max2, alpha};
  many_body_exact(t, a, strength, p, rng, s, words, false, st);
  D3_LAUNCH(k_noalloc_out, 1, 1, 0, st)(rng, t.info, words, words + 8);
  uint32_t out[3] = {0, 0, 0};
  if (cudaMemcpyAsync(out, words + 8, sizeof out, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return D3_WORKER_FAILED;
  // out[1] is the tree's failure mark: 1 when it needed more cells than the
  // array holds (vx, vy are then left as they were), 0xffffffff when its
  // launch did not happen. out[2] is the status word the kernels set.
  if (out[1] == 1) return D3_ARENA_FULL;
  if (out[1] || (out[2] & ST_FATAL)) return D3_WORKER_FAILED;
  *lcg_state = out[0];
  return D3_OK;
}
