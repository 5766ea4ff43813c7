// engine.cu — the C ABI (include/d3force_b200.h): simulation and force
// handles, pinned host mirrors, device arrays, random sources, dispatch.
//
// Mirrors root.zig's exports (handles 1-based with slot reuse, i32 statuses,
// node-sized force arrays padded with NaN) over device-resident state. One
// CUDA stream per simulation; the force kernels are enqueued on it and the
// host synchronises only where the ABI hands data back (sync_out, pointers
// after a tree build, the host random callback).
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "fast.cuh"
#include "forces.cuh"
#include "tree.cuh"

using namespace d3;

namespace d3 {
unsigned long long g_launches = 0;
}

namespace {

struct DForce {
  uint32_t kind = 0;
  double scalars[D3_SCALARS] = {0};
  uint32_t count = 0, cap = 0;
  double *h_f[3] = {nullptr, nullptr, nullptr};
  double *d_f[3] = {nullptr, nullptr, nullptr};
  uint32_t *h_src = nullptr, *h_tgt = nullptr, *d_src = nullptr, *d_tgt = nullptr;
  bool dirty = false;       // host mirrors may hold writes not yet uploaded
  bool plan_dirty = true;   // exact link plan must be rebuilt
  bool csr_dirty = true;    // fast link adjacency must be rebuilt
  uint32_t max_index = 0;   // largest source / target + 1 (link)
  double max_f0 = 0;        // largest f0 (collide: the largest radius)
  LinkPlan plan;
  FastLink csr;             // fast link adjacency (link_fast.zig)
};

struct DSim {
  uint32_t n = 0, cap = 0;
  double *h_x = nullptr, *h_y = nullptr, *h_vx = nullptr, *h_vy = nullptr, *h_fx = nullptr,
         *h_fy = nullptr;
  uint8_t *h_fixed = nullptr;
  double *d_x = nullptr, *d_y = nullptr, *d_vx = nullptr, *d_vy = nullptr, *d_fx = nullptr,
         *d_fy = nullptr, *d_px = nullptr, *d_py = nullptr, *d_svx = nullptr, *d_svy = nullptr;
  uint8_t *d_fixed = nullptr;
  double *h_snap = nullptr;
  uint32_t snap_cap = 0;
  TreeDev tree;
  ForceScratch scratch;
  FastScratch fast;
  CollideSpec spec;
  std::vector<DForce *> forces;
  // random
  Rng *d_rng = nullptr;
  Rng *h_rng = nullptr;  // pinned staging
  int host_random = 0;
  d3_random_fn rand_fn = nullptr;
  void *rand_ctx = nullptr;
  double *h_draws = nullptr, *d_draws = nullptr;
  uint64_t draws_cap = 0;
  // device words: 0 status, 1 link flag, 2..4 resume
  uint32_t *d_words = nullptr;
  uint32_t *h_words = nullptr;
  cudaStream_t stream = nullptr;
  // Side stream for work that may run ahead of its place in the tick (the
  // sums of a center force: they read positions, which nothing before the
  // first center force of a tick changes).
  cudaStream_t side = nullptr;
  cudaEvent_t ev_xready = nullptr, ev_sumdone = nullptr;
  // sim_sync_in copies x, y on `stream` and the rest of the node state on
  // `upload`; `stream` waits for ev_rest before anything else reads it.
  cudaStream_t upload = nullptr;
  cudaEvent_t ev_upstart = nullptr, ev_rest = nullptr;
  bool rest_pending = false;
  bool settle_after_accumulate = false;  // sim_tick: settle in the first many-body force
  // sim_tick: a many-body force of the tick runs a precision form judged by
  // RMS (not bit-exact), so the center's sums may take the tree order
  bool relaxed_center = false;
  uint32_t sync_mode = D3_SYNC_PER_CALL;
  bool fixed_from_f = false;  // sim_set_fixed_source
  // tree mirrors (tree_info)
  Cell *h_cells = nullptr;
  uint32_t h_cells_cap = 0;
  uint32_t *h_perm = nullptr;
  uint32_t h_perm_cap = 0;
  double h_extent[4] = {NAN, NAN, NAN, NAN};
  uint32_t h_len = 0, h_root = NONE, h_m = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
  double last_enqueue_ms = 0;  // host time sim_tick spent queueing work (before its final wait)
  // phase timers (sim_set_profile): pending event pairs per phase, totals
  bool profile = false;
  std::vector<cudaEvent_t> ev_pool;
  struct Pending { int phase; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  double phase_ms[16] = {0};
  uint64_t phase_n[16] = {0};
};

enum Phase { PH_MB_TREE = 0, PH_MB_ACC, PH_MB_TRAVERSE, PH_LINK, PH_COLLIDE_SETUP, PH_COLLIDE_RUN,
             PH_CENTER, PH_INTEGRATE, PH_FAST_MB, PH_FAST_LINK, PH_FAST_COLLIDE, PH_OTHER };

cudaEvent_t pool_event(DSim *s) {
  if (!s->ev_pool.empty()) {
    cudaEvent_t e = s->ev_pool.back();
    s->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// Records the start of a phase on the simulation's stream (no-op unless
// profiling); returns the event to close it with phase_end.
cudaEvent_t phase_begin(DSim *s) {
  if (!s->profile) return nullptr;
  cudaEvent_t e = pool_event(s);
  cudaEventRecord(e, s->stream);
  return e;
}

void phase_end(DSim *s, int phase, cudaEvent_t a) {
  if (!a) return;
  cudaEvent_t b = pool_event(s);
  cudaEventRecord(b, s->stream);
  s->pending.push_back({phase, a, b});
}

void phase_collect(DSim *s) {
  if (s->pending.empty()) return;
  cudaStreamSynchronize(s->stream);
  for (auto &p : s->pending) {
    float ms = 0;
    cudaEventElapsedTime(&ms, p.a, p.b);
    s->phase_ms[p.phase] += ms;
    s->phase_n[p.phase] += 1;
    s->ev_pool.push_back(p.a);
    s->ev_pool.push_back(p.b);
  }
  s->pending.clear();
}

std::vector<DSim *> g_sims;
int g_device_ok = -1;

bool device_ok() {
  if (g_device_ok < 0) {
    int count = 0;
    g_device_ok = cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
  }
  return g_device_ok == 1;
}

// The simulation's stream waits for the node state still being uploaded.
void settle(DSim *s) {
  if (!s->rest_pending) return;
  cudaStreamWaitEvent(s->stream, s->ev_rest, 0);
  s->rest_pending = false;
}

// The simulation without settling (sim_tick settles when it first needs
// the uploaded velocities).
DSim *get_sim_raw(uint32_t h) {
  if (h == 0 || h > g_sims.size()) return nullptr;
  return g_sims[h - 1];
}

// Every entry point but sim_tick: the simulation, settled.
DSim *get_sim(uint32_t h) {
  DSim *s = get_sim_raw(h);
  if (s) settle(s);
  return s;
}

DForce *get_force(DSim *s, uint32_t fh) {
  if (fh == 0 || fh > s->forces.size()) return nullptr;
  return s->forces[fh - 1];
}

bool node_sized(const DForce *f) { return f->kind != D3_LINK && f->kind != D3_CENTER; }

int float_arrays(uint32_t kind) {
  switch (kind) {
    case D3_CENTER: return 0;
    case D3_COLLIDE:
    case D3_MANY_BODY: return 1;
    case D3_LINK: return 3;
    default: return 2;
  }
}

template <typename T>
int grow_pinned(T *&p, size_t old_n, size_t new_cap) {
  T *np = nullptr;
  if (cudaMallocHost(&np, (new_cap ? new_cap : 1) * sizeof(T)) != cudaSuccess) return -1;
  if (p && old_n) memcpy(np, p, old_n * sizeof(T));
  if (p) cudaFreeHost(p);
  p = np;
  return 0;
}

template <typename T>
int grow_device(T *&p, size_t old_n, size_t new_cap, cudaStream_t st) {
  T *np = nullptr;
  if (cudaMalloc(&np, (new_cap ? new_cap : 1) * sizeof(T)) != cudaSuccess) return -1;
  if (p && old_n) cudaMemcpyAsync(np, p, old_n * sizeof(T), cudaMemcpyDeviceToDevice, st);
  if (p) {
    cudaStreamSynchronize(st);
    cudaFree(p);
  }
  p = np;
  return 0;
}

int force_set_count_impl(DSim *s, DForce *f, uint32_t count) {
  const uint32_t old = f->count;
  const int k = float_arrays(f->kind);
  if (count > f->cap) {
    uint32_t cap = count;
    for (int i = 0; i < k; ++i) {
      if (grow_pinned(f->h_f[i], old, cap) || grow_device(f->d_f[i], old, cap, s->stream)) return -1;
    }
    if (f->kind == D3_LINK) {
      if (grow_pinned(f->h_src, old, cap) || grow_pinned(f->h_tgt, old, cap) ||
          grow_device(f->d_src, old, cap, s->stream) || grow_device(f->d_tgt, old, cap, s->stream))
        return -1;
    }
    f->cap = cap;
  }
  for (int i = 0; i < k; ++i)
    for (uint32_t j = old; j < count; ++j) f->h_f[i][j] = NAN;
  if (f->kind == D3_LINK)
    for (uint32_t j = old; j < count; ++j) f->h_src[j] = f->h_tgt[j] = 0;
  f->count = count;
  f->dirty = true;
  f->plan_dirty = true;
  f->csr_dirty = true;
  return 0;
}

void force_free(DForce *f) {
  for (int i = 0; i < 3; ++i) {
    if (f->h_f[i]) cudaFreeHost(f->h_f[i]);
    cudaFree(f->d_f[i]);
  }
  if (f->h_src) cudaFreeHost(f->h_src);
  if (f->h_tgt) cudaFreeHost(f->h_tgt);
  cudaFree(f->d_src);
  cudaFree(f->d_tgt);
  link_plan_free(f->plan);
  fast_link_free(f->csr);
  delete f;
}

// Host mirrors of a force -> device, when written since the last upload.
int upload_force(DSim *s, DForce *f) {
  if (!f->dirty) return 0;
  const int k = float_arrays(f->kind);
  for (int i = 0; i < k; ++i)
    if (f->count)
      cudaMemcpyAsync(f->d_f[i], f->h_f[i], f->count * 8ull, cudaMemcpyHostToDevice, s->stream);
  if (f->kind == D3_COLLIDE) {
    double mx = 0;
    for (uint32_t i = 0; i < f->count; ++i)
      if (f->h_f[0][i] > mx) mx = f->h_f[0][i];
    f->max_f0 = mx;
  }
  if (f->kind == D3_LINK && f->count) {
    cudaMemcpyAsync(f->d_src, f->h_src, f->count * 4ull, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(f->d_tgt, f->h_tgt, f->count * 4ull, cudaMemcpyHostToDevice, s->stream);
    uint32_t mx = 0;
    for (uint32_t e = 0; e < f->count; ++e) {
      if (f->h_src[e] + 1 > mx) mx = f->h_src[e] + 1;
      if (f->h_tgt[e] + 1 > mx) mx = f->h_tgt[e] + 1;
    }
    f->max_index = mx;
    f->plan_dirty = true;
    f->csr_dirty = true;
  }
  f->dirty = false;
  return 0;
}

NodeArrays nodes_of(DSim *s) {
  NodeArrays a;
  a.x = s->d_x; a.y = s->d_y; a.vx = s->d_vx; a.vy = s->d_vy; a.fx = s->d_fx; a.fy = s->d_fy;
  a.fixed = s->d_fixed; a.px = s->d_px; a.py = s->d_py; a.snap_vx = s->d_svx; a.snap_vy = s->d_svy;
  a.n = s->n;
  return a;
}

// Host mirrors -> device. x and y go on the simulation's stream; vx, vy, fx,
// fy and the fixed bits on the upload stream after all earlier work, so that
// a tick's tree build can overlap them (defer: the caller settles later;
// otherwise settled here).
int sync_in_impl(DSim *s, bool defer = false) {
  const size_t n = s->n;
  if (n) {
    cudaStream_t st = s->stream, up = s->upload;
    cudaMemcpyAsync(s->d_x, s->h_x, n * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->d_y, s->h_y, n * 8, cudaMemcpyHostToDevice, st);
    cudaEventRecord(s->ev_upstart, st);
    cudaStreamWaitEvent(up, s->ev_upstart, 0);
    cudaMemcpyAsync(s->d_vx, s->h_vx, n * 8, cudaMemcpyHostToDevice, up);
    cudaMemcpyAsync(s->d_vy, s->h_vy, n * 8, cudaMemcpyHostToDevice, up);
    cudaMemcpyAsync(s->d_fx, s->h_fx, n * 8, cudaMemcpyHostToDevice, up);
    cudaMemcpyAsync(s->d_fy, s->h_fy, n * 8, cudaMemcpyHostToDevice, up);
    if (s->fixed_from_f) fixed_from_f(s->d_fx, s->d_fy, s->d_fixed, (uint32_t)n, up);
    else cudaMemcpyAsync(s->d_fixed, s->h_fixed, n, cudaMemcpyHostToDevice, up);
    cudaEventRecord(s->ev_rest, up);
    s->rest_pending = true;
    if (!defer) settle(s);
  }
  for (DForce *f : s->forces)
    if (f) upload_force(s, f);
  return D3_OK;
}

// Queues the copy of the status word that take_failure reads after the next
// host synchronisation.
void queue_status(DSim *s) {
  cudaMemcpyAsync(s->h_words + 24, s->d_words, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
}

// After a synchronisation that followed queue_status: D3_WORKER_FAILED (once)
// if a kernel reported a failure since the last check.
int take_failure(DSim *s) {
  const uint32_t w = s->h_words[24];
  if (!(w & ST_FATAL)) return D3_OK;
  s->h_words[25] = w & ~ST_FATAL;
  cudaMemcpy(s->d_words, s->h_words + 25, sizeof(uint32_t), cudaMemcpyHostToDevice);
  s->h_words[24] = 0;
  return D3_WORKER_FAILED;
}

int sync_out_impl(DSim *s) {
  const size_t n = s->n;
  cudaStream_t st = s->stream;
  if (n) {
    cudaMemcpyAsync(s->h_x, s->d_x, n * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s->h_y, s->d_y, n * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s->h_vx, s->d_vx, n * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s->h_vy, s->d_vy, n * 8, cudaMemcpyDeviceToHost, st);
  }
  queue_status(s);
  if (cudaStreamSynchronize(st) != cudaSuccess) return D3_WORKER_FAILED;
  return take_failure(s);
}

// Words on the device: 0 status (sticky), 1 link flag, 2..4 resume.
uint32_t *status_word(DSim *s) { return s->d_words; }
uint32_t *link_flag(DSim *s) { return s->d_words + 1; }
uint32_t *resume_words(DSim *s) { return s->d_words + 2; }

int read_words(DSim *s) {
  cudaMemcpyAsync(s->h_words, s->d_words, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
  return cudaStreamSynchronize(s->stream) == cudaSuccess ? 0 : -1;
}

// Pulls `k` draws from the caller's random function (in order) into the
// device draw buffer and points the stream at them.
int pull_draws(DSim *s, uint64_t k) {
  if (k > s->draws_cap) {
    if (s->h_draws) cudaFreeHost(s->h_draws);
    cudaFree(s->d_draws);
    uint64_t cap = k < 1024 ? 1024 : k;
    if (cudaMallocHost(&s->h_draws, cap * 8) != cudaSuccess) return -1;
    if (cudaMalloc(&s->d_draws, cap * 8) != cudaSuccess) return -1;
    s->draws_cap = cap;
  }
  for (uint64_t i = 0; i < k; ++i) s->h_draws[i] = s->rand_fn(s->rand_ctx);
  cudaMemcpyAsync(s->d_draws, s->h_draws, k * 8, cudaMemcpyHostToDevice, s->stream);
  Rng r;
  r.lcg = 0;
  r.mode = 1;
  r.pos = 0;
  r.avail = k;
  r.buf = s->d_draws;
  *s->h_rng = r;
  cudaMemcpyAsync(s->d_rng, s->h_rng, sizeof(Rng), cudaMemcpyHostToDevice, s->stream);
  return 0;
}

int run_many_body(DSim *s, DForce *f, double alpha) {
  ManyBodyParams p{f->scalars[D3_THETA2], f->scalars[D3_DISTANCE_MIN2],
                   f->scalars[D3_DISTANCE_MAX2], alpha};
  NodeArrays a = nodes_of(s);
  if (!s->host_random) {
    cudaEvent_t e = phase_begin(s);
    many_body_exact(s->tree, a, f->d_f[0], p, s->d_rng, s->scratch, status_word(s), false,
                    s->stream, [&](int ph) {
                      phase_end(s, ph, e);
                      // the traversal reads the velocities (sim_tick's first force)
                      if (ph == 1 && s->settle_after_accumulate) settle(s);
                      e = phase_begin(s);
                    });
    settle(s);
    phase_end(s, PH_MB_TRAVERSE, e);
    return D3_OK;
  }
  many_body_exact(s->tree, a, f->d_f[0], p, s->d_rng, s->scratch, status_word(s), true, s->stream);
  uint32_t total = 0;
  cudaMemcpyAsync(s->h_words + 8, s->scratch.counters, 4, cudaMemcpyDeviceToHost, s->stream);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return D3_WORKER_FAILED;
  total = s->h_words[8];
  if (total == 0) return D3_OK;
  if (pull_draws(s, total)) return D3_OUT_OF_MEMORY;
  many_body_rerun(s->tree, a, f->d_f[0], p, s->d_rng, s->scratch, s->stream);
  return D3_OK;
}

int run_link(DSim *s, DForce *f, double alpha) {
  if (f->max_index > s->n) return D3_BAD_ARGUMENT;
  if (f->count == 0) return D3_OK;
  if (f->plan_dirty) {
    if (link_plan_build(f->plan, f->h_src, f->h_tgt, f->count)) return D3_OUT_OF_MEMORY;
    f->plan_dirty = false;
  }
  NodeArrays a = nodes_of(s);
  LinkArrays l{f->d_f[0], f->d_f[1], f->d_f[2], f->d_src, f->d_tgt, f->count};
  const double iterations = f->scalars[D3_ITERATIONS];
  cudaEvent_t e = phase_begin(s);
  link_exact(a, l, f->plan, alpha, iterations, s->d_rng, link_flag(s), status_word(s),
             !s->host_random, s->stream);
  if (!s->host_random) {
    phase_end(s, PH_LINK, e);
    return D3_OK;
  }
  phase_end(s, PH_LINK, e);
  if (read_words(s)) return D3_WORKER_FAILED;
  if (s->h_words[1] == 0) return D3_OK;
  // Serial pass with exactly the draws it asks for, pulled in d3's order.
  uint32_t *res = resume_words(s);
  cudaMemsetAsync(res, 0, 3 * sizeof(uint32_t), s->stream);
  if (pull_draws(s, 0)) return D3_OUT_OF_MEMORY;
  for (;;) {
    link_serial_host(a, l, alpha, iterations, s->d_rng, res, s->stream);
    if (read_words(s)) return D3_WORKER_FAILED;
    uint32_t need = s->h_words[4];
    if (need == 0) break;
    if (pull_draws(s, need)) return D3_OUT_OF_MEMORY;
  }
  return D3_OK;
}

int run_collide(DSim *s, DForce *f) {
  NodeArrays a = nodes_of(s);
  const double strength = f->scalars[D3_STRENGTH], iterations = f->scalars[D3_ITERATIONS];
  uint32_t *res = resume_words(s);
  for (double k = 0; k < iterations; k += 1) {
    cudaEvent_t e = phase_begin(s);
    collide_setup(s->tree, a, f->d_f[0], status_word(s), s->stream);
    cudaMemsetAsync(res, 0, 3 * sizeof(uint32_t), s->stream);
    phase_end(s, PH_COLLIDE_SETUP, e);
    if (!s->host_random) {
      static const double factor = [] {
        const char *e = getenv("D3_COLLIDE_DELTA");
        double v = e ? atof(e) : 0;
        return v > 0 ? v : 1.0;
      }();
      const double delta = (f->max_f0 > 0 ? f->max_f0 : 1.0) * factor;
      e = phase_begin(s);
      if (collide_parallel(s->tree, a, f->d_f[0], strength, delta, s->d_rng, s->spec, s->stream))
        collide_serial(s->tree, a, f->d_f[0], strength, s->d_rng, false, res, s->stream);
      phase_end(s, PH_COLLIDE_RUN, e);
      continue;
    }
    if (pull_draws(s, 0)) return D3_OUT_OF_MEMORY;
    for (;;) {
      collide_serial(s->tree, a, f->d_f[0], strength, s->d_rng, true, res, s->stream);
      if (read_words(s)) return D3_WORKER_FAILED;
      uint32_t need = s->h_words[4];
      if (need == 0) break;
      if (pull_draws(s, need)) return D3_OUT_OF_MEMORY;
    }
  }
  return D3_OK;
}

// PRECISION: 0 exact; 1 fast (the reference's FMM, bit for bit); 2 fast with
// the tensor-core FMM (BF16x3 M2L, FP32 near field); 3 fast with the learned
// order-4 correction. Link and collide run the same fast kernels for 1-3.
bool fast_mode(const DSim *s, const DForce *f) {
  const double pr = f->scalars[D3_PRECISION];
  return (pr == 1 || pr == 2 || pr == 3) && s->n >= FAST_MIN_N;
}

// fuse_center: a center force's shift is left to the caller (which fuses it
// into integrate).
int run_force(DSim *s, DForce *f, double alpha, bool presummed = false, bool fuse_center = false) {
  NodeArrays a = nodes_of(s);
  // The facade's per-run SEED draw in fast mode (src/core.js:218-222), from
  // the device LCG when it is the random source.
  const double prec = f->scalars[D3_PRECISION];
  const bool seeded = (prec == 1 || prec == 2 || prec == 3) &&
                      (f->kind == D3_MANY_BODY || f->kind == D3_LINK || f->kind == D3_COLLIDE);
  double *seed_slot = s->fast.seed;
  if (seeded) {
    if (!s->host_random) draw_seed(s->d_rng, seed_slot, s->stream);
    else set_seed(seed_slot, f->scalars[D3_SEED], s->stream);
  }
  switch (f->kind) {
    case D3_CENTER: {
      cudaEvent_t e = phase_begin(s);
      if (presummed) cudaStreamWaitEvent(s->stream, s->ev_sumdone, 0);
      else if (s->relaxed_center) center_sum_tree(a, s->scratch, s->stream);
      else center_sum(a, s->scratch, status_word(s), s->stream);
      if (!fuse_center)
        center_apply(a, f->scalars[D3_CX], f->scalars[D3_CY], f->scalars[D3_STRENGTH], s->scratch,
                     s->stream);
      phase_end(s, PH_CENTER, e);
      return D3_OK;
    }
    case D3_X: axis_force(a, f->d_f[0], f->d_f[1], alpha, 0, s->stream); return D3_OK;
    case D3_Y: axis_force(a, f->d_f[0], f->d_f[1], alpha, 1, s->stream); return D3_OK;
    case D3_RADIAL:
      radial_force(a, f->d_f[0], f->d_f[1], f->scalars[D3_CX], f->scalars[D3_CY], alpha, s->stream);
      return D3_OK;
    case D3_LINK:
      if (fast_mode(s, f)) {
        if (f->max_index > s->n) return D3_BAD_ARGUMENT;
        if (f->csr_dirty || f->csr.n != s->n) {
          if (fast_link_build(f->csr, f->h_src, f->h_tgt, f->count, s->n)) return D3_OUT_OF_MEMORY;
          f->csr_dirty = false;
        }
        LinkArrays l{f->d_f[0], f->d_f[1], f->d_f[2], f->d_src, f->d_tgt, f->count};
        cudaEvent_t e = phase_begin(s);
        fast_link(a, l, f->csr, alpha, f->scalars[D3_ITERATIONS], seed_slot, s->stream);
        phase_end(s, PH_FAST_LINK, e);
        return D3_OK;
      }
      return run_link(s, f, alpha);
    case D3_MANY_BODY:
      if (fast_mode(s, f)) {
        FmmParams fp;
        fp.order = f->scalars[D3_ORDER];
        fp.opening = f->scalars[D3_OPENING];
        fp.dmin2 = f->scalars[D3_DISTANCE_MIN2];
        fp.dmax2 = f->scalars[D3_DISTANCE_MAX2];
        fp.alpha = alpha;
        cudaEvent_t e = phase_begin(s);
        int r = prec == 1 ? fmm_run(s->fast, s->tree, a, f->d_f[0], fp, seed_slot, status_word(s),
                                    s->stream)
                          : fmm_tc_run(s->fast, s->tree, a, f->d_f[0], fp, (int)prec, seed_slot,
                                       status_word(s), s->stream);
        phase_end(s, PH_FAST_MB, e);
        if (r == 1) return D3_OK;
        if (r == -3) return D3_BAD_ARGUMENT;
        if (r < 0) return D3_OUT_OF_MEMORY;
      }
      return run_many_body(s, f, alpha);
    case D3_COLLIDE:
      if (fast_mode(s, f)) {
        cudaEvent_t e = phase_begin(s);
        fast_collide(s->fast, a, f->d_f[0], f->scalars[D3_STRENGTH], f->scalars[D3_ITERATIONS],
                     seed_slot, s->stream);
        phase_end(s, PH_FAST_COLLIDE, e);
        return D3_OK;
      }
      return run_collide(s, f);
    default: return D3_BAD_ARGUMENT;
  }
}

int ensure_cap(DSim *s, uint32_t n) {
  if (n <= s->cap) return 0;
  uint32_t cap = n;
  if (s->cap * 2 > cap) cap = s->cap * 2;
  if (cap < 16) cap = 16;
  const uint32_t old = s->n < s->cap ? s->n : s->cap;
  cudaStream_t st = s->stream;
  if (grow_pinned(s->h_x, old, cap) || grow_pinned(s->h_y, old, cap) ||
      grow_pinned(s->h_vx, old, cap) || grow_pinned(s->h_vy, old, cap) ||
      grow_pinned(s->h_fx, old, cap) || grow_pinned(s->h_fy, old, cap) ||
      grow_pinned(s->h_fixed, old, cap))
    return -1;
  if (grow_device(s->d_x, old, cap, st) || grow_device(s->d_y, old, cap, st) ||
      grow_device(s->d_vx, old, cap, st) || grow_device(s->d_vy, old, cap, st) ||
      grow_device(s->d_fx, old, cap, st) || grow_device(s->d_fy, old, cap, st) ||
      grow_device(s->d_fixed, old, cap, st) || grow_device(s->d_px, 0, cap, st) ||
      grow_device(s->d_py, 0, cap, st) || grow_device(s->d_svx, 0, cap, st) ||
      grow_device(s->d_svy, 0, cap, st))
    return -1;
  if (tree_reserve(s->tree, cap) || scratch_reserve(s->scratch, cap) || fast_reserve(s->fast, cap) ||
      collide_spec_reserve(s->spec, cap))
    return -1;
  s->cap = cap;
  return 0;
}

}  // namespace

extern "C" {

uint32_t sim_create(void) {
  if (!device_ok()) return 0;
  DSim *s = new DSim();
  // The tick's stream takes the greatest priority: work that other streams
  // run beside it (the center sums, the tensor-core form's near field and
  // upward pass) fills the SMs it leaves free.
  int prio_least = 0, prio_greatest = 0;
  cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    return 0;
  }
  cudaEventCreateWithFlags(&s->ev_xready, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&s->ev_sumdone, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&s->ev_upstart, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&s->ev_rest, cudaEventDisableTiming);
  cudaMalloc(&s->d_rng, sizeof(Rng));
  cudaMallocHost(&s->h_rng, sizeof(Rng));
  cudaMalloc(&s->d_words, 16 * sizeof(uint32_t));
  cudaMallocHost(&s->h_words, 32 * sizeof(uint32_t));
  cudaMemset(s->d_words, 0, 16 * sizeof(uint32_t));
  Rng r{};
  r.lcg = 1;
  r.mode = 0;
  cudaMemcpy(s->d_rng, &r, sizeof(Rng), cudaMemcpyHostToDevice);
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  if (tree_reserve(s->tree, 16) || scratch_reserve(s->scratch, 16) || fast_reserve(s->fast, 16)) {
    delete s;
    return 0;
  }
  for (size_t i = 0; i < g_sims.size(); ++i)
    if (!g_sims[i]) {
      g_sims[i] = s;
      return (uint32_t)i + 1;
    }
  g_sims.push_back(s);
  return (uint32_t)g_sims.size();
}

int32_t sim_destroy(uint32_t h) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  cudaStreamSynchronize(s->stream);
  for (DForce *f : s->forces)
    if (f) force_free(f);
  double *hp[] = {s->h_x, s->h_y, s->h_vx, s->h_vy, s->h_fx, s->h_fy, s->h_snap};
  for (double *p : hp)
    if (p) cudaFreeHost(p);
  if (s->h_fixed) cudaFreeHost(s->h_fixed);
  double *dp[] = {s->d_x, s->d_y, s->d_vx, s->d_vy, s->d_fx, s->d_fy, s->d_px, s->d_py, s->d_svx, s->d_svy};
  for (double *p : dp) cudaFree(p);
  cudaFree(s->d_fixed);
  tree_free(s->tree);
  scratch_free(s->scratch);
  fast_free(s->fast);
  collide_spec_free(s->spec);
  cudaFree(s->d_rng);
  cudaFreeHost(s->h_rng);
  cudaFree(s->d_words);
  cudaFreeHost(s->h_words);
  if (s->h_draws) cudaFreeHost(s->h_draws);
  cudaFree(s->d_draws);
  free(s->h_cells);
  free(s->h_perm);
  cudaEventDestroy(s->ev0);
  cudaEventDestroy(s->ev1);
  cudaEventDestroy(s->ev_xready);
  cudaEventDestroy(s->ev_sumdone);
  cudaStreamSynchronize(s->side);
  cudaStreamDestroy(s->side);
  cudaStreamSynchronize(s->upload);
  cudaEventDestroy(s->ev_upstart);
  cudaEventDestroy(s->ev_rest);
  cudaStreamDestroy(s->upload);
  cudaStreamDestroy(s->stream);
  delete s;
  g_sims[h - 1] = nullptr;
  return D3_OK;
}

int32_t sim_set_node_count(uint32_t h, uint32_t n) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  bool grown = false;
  for (DForce *f : s->forces)
    if (f && node_sized(f) && f->count < n) {
      if (force_set_count_impl(s, f, n)) return D3_OUT_OF_MEMORY;
      grown = true;
    }
  if (n > s->cap) {
    if (ensure_cap(s, n)) return D3_OUT_OF_MEMORY;
    grown = true;
  }
  s->n = n;
  return grown ? D3_GROWN : D3_OK;
}

uintptr_t sim_ptr(uint32_t h, uint32_t which) {
  DSim *s = get_sim(h);
  if (!s) return 0;
  switch (which) {
    case D3_PTR_X: return (uintptr_t)s->h_x;
    case D3_PTR_Y: return (uintptr_t)s->h_y;
    case D3_PTR_VX: return (uintptr_t)s->h_vx;
    case D3_PTR_VY: return (uintptr_t)s->h_vy;
    case D3_PTR_FX: return (uintptr_t)s->h_fx;
    case D3_PTR_FY: return (uintptr_t)s->h_fy;
    case D3_PTR_FIXED: return (uintptr_t)s->h_fixed;
    case D3_PTR_PERM: return (uintptr_t)s->h_perm;
    case D3_PTR_SNAP: return (uintptr_t)s->h_snap;
    default: return 0;
  }
}

uint32_t force_create(uint32_t h, uint32_t kind) {
  DSim *s = get_sim(h);
  if (!s || kind > D3_Y) return 0;
  DForce *f = new DForce();
  f->kind = kind;
  if (node_sized(f) && force_set_count_impl(s, f, s->n)) {
    force_free(f);
    return 0;
  }
  for (size_t i = 0; i < s->forces.size(); ++i)
    if (!s->forces[i]) {
      s->forces[i] = f;
      return (uint32_t)i + 1;
    }
  s->forces.push_back(f);
  return (uint32_t)s->forces.size();
}

int32_t force_destroy(uint32_t h, uint32_t fh) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  DForce *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  cudaStreamSynchronize(s->stream);
  force_free(f);
  s->forces[fh - 1] = nullptr;
  return D3_OK;
}

int32_t force_set_count(uint32_t h, uint32_t fh, uint32_t count) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  DForce *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  if (force_set_count_impl(s, f, count)) return D3_OUT_OF_MEMORY;
  return D3_GROWN;
}

uintptr_t force_ptr(uint32_t h, uint32_t fh, uint32_t which) {
  DSim *s = get_sim(h);
  if (!s) return 0;
  DForce *f = get_force(s, fh);
  if (!f || f->count == 0) return 0;
  // The caller may write through the pointer: upload before the next run.
  f->dirty = true;
  switch (which) {
    case D3_F0: return (uintptr_t)f->h_f[0];
    case D3_F1: return (uintptr_t)f->h_f[1];
    case D3_F2: return (uintptr_t)f->h_f[2];
    case D3_SOURCE: return (uintptr_t)f->h_src;
    case D3_TARGET: return (uintptr_t)f->h_tgt;
    default: return 0;
  }
}

int32_t force_set_scalar(uint32_t h, uint32_t fh, uint32_t which, double v) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  DForce *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  if (which >= D3_SCALARS) return D3_BAD_ARGUMENT;
  f->scalars[which] = v;
  return D3_OK;
}

double force_get_scalar(uint32_t h, uint32_t fh, uint32_t which) {
  DSim *s = get_sim(h);
  if (!s) return 0;
  DForce *f = get_force(s, fh);
  if (!f) return 0;
  return which < D3_SCALARS ? f->scalars[which] : 0;
}

int32_t force_run(uint32_t h, uint32_t fh, double alpha) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  DForce *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  if (node_sized(f) && f->count < s->n) return D3_BAD_ARGUMENT;
  if (s->sync_mode == D3_SYNC_PER_CALL) sync_in_impl(s);
  else upload_force(s, f);
  int r = run_force(s, f, alpha);
  if (r < 0) return r;
  if (s->sync_mode == D3_SYNC_PER_CALL) return sync_out_impl(s);
  return D3_OK;
}

int32_t sim_integrate(uint32_t h, double velocity_decay) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (s->sync_mode == D3_SYNC_PER_CALL) sync_in_impl(s);
  integrate(nodes_of(s), velocity_decay, s->stream);
  if (s->sync_mode == D3_SYNC_PER_CALL) return sync_out_impl(s);
  return D3_OK;
}

int32_t sim_snapshot(uint32_t h, uint32_t positions) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  const uint32_t n = s->n;
  if (s->snap_cap < 4 * n) {
    if (s->h_snap) cudaFreeHost(s->h_snap);
    s->h_snap = nullptr;
    if (cudaMallocHost(&s->h_snap, 4ull * (s->cap ? s->cap : 1) * 8) != cudaSuccess)
      return D3_OUT_OF_MEMORY;
    s->snap_cap = 4 * s->cap;
  }
  cudaMemcpyAsync(s->h_snap, s->d_vx, n * 8ull, cudaMemcpyDeviceToHost, s->stream);
  cudaMemcpyAsync(s->h_snap + n, s->d_vy, n * 8ull, cudaMemcpyDeviceToHost, s->stream);
  if (positions) {
    cudaMemcpyAsync(s->h_snap + 2 * n, s->d_x, n * 8ull, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(s->h_snap + 3 * n, s->d_y, n * 8ull, cudaMemcpyDeviceToHost, s->stream);
  }
  return cudaStreamSynchronize(s->stream) == cudaSuccess ? D3_OK : D3_WORKER_FAILED;
}

int32_t tree_build(uint32_t h, uint32_t shifted) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (s->sync_mode == D3_SYNC_PER_CALL) sync_in_impl(s);
  NodeArrays a = nodes_of(s);
  if (shifted) {
    shift_positions(a, s->stream);
    d3::tree_build(s->tree, a.px, a.py, a.n, status_word(s), s->stream);
  } else {
    d3::tree_build(s->tree, a.x, a.y, a.n, status_word(s), s->stream);
  }
  uint32_t info[8];
  cudaMemcpyAsync(s->h_words + 8, s->tree.info, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                  s->stream);
  cudaMemcpyAsync(s->h_extent, s->tree.extent, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                  s->stream);
  queue_status(s);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return D3_WORKER_FAILED;
  // a tree that did not fit its cell buffer (or a build that did not launch)
  // is reported here and leaves an empty tree
  if (int fr = take_failure(s)) {
    s->h_len = 0;
    s->h_root = NONE;
    return fr;
  }
  memcpy(info, s->h_words + 8, sizeof info);
  bool grown = false;
  s->h_m = info[0];
  s->h_len = a.n ? info[1] : 0;
  s->h_root = s->h_len ? 0 : NONE;
  if (s->h_len > s->h_cells_cap) {
    free(s->h_cells);
    s->h_cells = (Cell *)malloc((size_t)s->h_len * sizeof(Cell));
    s->h_cells_cap = s->h_len;
    grown = true;
  }
  if (a.n > s->h_perm_cap || !s->h_perm) {
    free(s->h_perm);
    s->h_perm = (uint32_t *)malloc((size_t)(a.n ? a.n : 1) * 4);
    s->h_perm_cap = a.n;
    grown = true;
  }
  if (s->h_len)
    cudaMemcpyAsync(s->h_cells, s->tree.cells, (size_t)s->h_len * sizeof(Cell),
                    cudaMemcpyDeviceToHost, s->stream);
  if (a.n)
    cudaMemcpyAsync(s->h_perm, s->tree.perm, (size_t)a.n * 4, cudaMemcpyDeviceToHost, s->stream);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return D3_WORKER_FAILED;
  return grown ? D3_GROWN : D3_OK;
}

uintptr_t tree_info(uint32_t h, uint32_t which) {
  DSim *s = get_sim(h);
  if (!s) return 0;
  switch (which) {
    case 0: return s->h_len;
    case 1: return s->h_root;
    case 2: return (uintptr_t)s->h_cells;
    case 3: return (uintptr_t)s->h_extent;
    case 4: return (uintptr_t)s->h_perm;
    case 5: return sizeof(Cell);
    case 6: return s->h_m;
    default: return 0;
  }
}

int32_t tree_order(uint32_t h, uint32_t after, uint32_t *out) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (!out) return D3_BAD_ARGUMENT;
  if (s->h_root == NONE) return D3_OK;
  // tree.zig:652-684 on the downloaded cells.
  std::vector<uint32_t> stack;
  stack.push_back(s->h_root);
  uint32_t w = 0;
  while (!stack.empty()) {
    uint32_t c = stack.back();
    stack.pop_back();
    out[w++] = c;
    const uint32_t *ch = s->h_cells[c].child;
    if (after) {
      for (int i = 0; i < 4; ++i)
        if (ch[i] != NONE) stack.push_back(ch[i]);
    } else {
      for (int i = 3; i >= 0; --i)
        if (ch[i] != NONE) stack.push_back(ch[i]);
    }
  }
  if (after)
    for (uint32_t i = 0, j = w ? w - 1 : 0; i < j; ++i, --j) {
      uint32_t t = out[i];
      out[i] = out[j];
      out[j] = t;
    }
  return D3_OK;
}

int32_t sim_set_random(uint32_t h, d3_random_fn fn, void *ctx) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  s->host_random = fn != nullptr;
  s->rand_fn = fn;
  s->rand_ctx = ctx;
  return D3_OK;
}

int32_t sim_set_lcg(uint32_t h, uint32_t state) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  s->host_random = 0;
  s->rand_fn = nullptr;
  Rng r{};
  r.lcg = state;
  r.mode = 0;
  *s->h_rng = r;
  cudaMemcpyAsync(s->d_rng, s->h_rng, sizeof(Rng), cudaMemcpyHostToDevice, s->stream);
  return cudaStreamSynchronize(s->stream) == cudaSuccess ? D3_OK : D3_WORKER_FAILED;
}

uint32_t sim_get_lcg(uint32_t h) {
  DSim *s = get_sim(h);
  if (!s) return 0;
  cudaMemcpyAsync(s->h_rng, s->d_rng, sizeof(Rng), cudaMemcpyDeviceToHost, s->stream);
  cudaStreamSynchronize(s->stream);
  return s->h_rng->lcg;
}

int32_t sim_set_fixed_source(uint32_t h, uint32_t from_f) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (from_f > 1) return D3_BAD_ARGUMENT;
  s->fixed_from_f = from_f != 0;
  return D3_OK;
}

int32_t sim_set_sync(uint32_t h, uint32_t mode) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (mode > D3_SYNC_PER_CALL) return D3_BAD_ARGUMENT;
  s->sync_mode = mode;
  return D3_OK;
}

int32_t sim_sync_in(uint32_t h) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  return sync_in_impl(s, true);
}

int32_t sim_sync_out(uint32_t h) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  return sync_out_impl(s);
}

}  // extern "C"

namespace {

// The ticks of sim_tick; with copy_out the node state's device-to-host
// copies are queued behind them, before the one synchronisation.
int32_t tick_impl(DSim *s, uint32_t ticks, double *alpha, double alpha_target, double alpha_decay,
                  double velocity_decay, const uint32_t *order, uint32_t n_order, bool copy_out) {
  if (!alpha || (n_order && !order)) {
    settle(s);
    return D3_BAD_ARGUMENT;
  }
  std::vector<DForce *> fs;
  for (uint32_t i = 0; i < n_order; ++i) {
    DForce *f = get_force(s, order[i]);
    if (!f || (node_sized(f) && f->count < s->n)) {
      settle(s);
      return f ? D3_BAD_ARGUMENT : D3_BAD_HANDLE;
    }
    upload_force(s, f);
    fs.push_back(f);
  }
  // An exact many-body force first reads only positions (and its strengths)
  // until its traversal: the rest of the node state may still be uploading.
  s->settle_after_accumulate = !fs.empty() && fs[0]->kind == D3_MANY_BODY && !s->host_random &&
                               !fast_mode(s, fs[0]);
  s->relaxed_center = false;
  for (const DForce *f : fs)
    if (f->kind == D3_MANY_BODY && fast_mode(s, f) &&
        (f->scalars[D3_PRECISION] == 2 || f->scalars[D3_PRECISION] == 3))
      s->relaxed_center = true;
  if (!s->settle_after_accumulate) settle(s);
  // The first center force's sums only read positions, which no force
  // before it changes: run them on the side stream from the tick's start.
  int hoist = -1;
  for (size_t i = 0; i < fs.size(); ++i)
    if (fs[i]->kind == D3_CENTER) {
      hoist = (int)i;
      break;
    }
  const auto host0 = std::chrono::steady_clock::now();
  cudaEventRecord(s->ev0, s->stream);
  double a = *alpha;
  for (uint32_t k = 0; k < ticks; ++k) {
    a += (alpha_target - a) * alpha_decay;
    if (hoist >= 0 && s->n) {
      cudaEventRecord(s->ev_xready, s->stream);
      cudaStreamWaitEvent(s->side, s->ev_xready, 0);
      cudaEvent_t e = nullptr;
      if (s->profile) {
        e = pool_event(s);
        cudaEventRecord(e, s->side);
      }
      if (s->relaxed_center) center_sum_tree(nodes_of(s), s->scratch, s->side);
      else center_sum(nodes_of(s), s->scratch, status_word(s), s->side);
      if (e) {
        cudaEvent_t b = pool_event(s);
        cudaEventRecord(b, s->side);
        s->pending.push_back({PH_OTHER, e, b});
      }
      cudaEventRecord(s->ev_sumdone, s->side);
    }
    // a center force that comes last has its shift fused into integrate
    const bool fuse = !fs.empty() && fs.back()->kind == D3_CENTER;
    for (size_t i = 0; i < fs.size(); ++i) {
      if (i > 0 || k > 0) settle(s);
      int r = run_force(s, fs[i], a, (int)i == hoist && s->n, fuse && i + 1 == fs.size());
      if (r < 0) {
        settle(s);
        s->settle_after_accumulate = false;
        s->relaxed_center = false;
        return r;
      }
    }
    settle(s);
    cudaEvent_t e = phase_begin(s);
    if (fuse) {
      const DForce *c = fs.back();
      center_apply_integrate(nodes_of(s), c->scalars[D3_CX], c->scalars[D3_CY],
                             c->scalars[D3_STRENGTH], s->scratch, velocity_decay, s->stream);
    } else {
      integrate(nodes_of(s), velocity_decay, s->stream);
    }
    phase_end(s, PH_INTEGRATE, e);
  }
  s->settle_after_accumulate = false;
  s->relaxed_center = false;
  cudaEventRecord(s->ev1, s->stream);
  s->last_enqueue_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host0).count();
  *alpha = a;
  if (hoist >= 0) cudaStreamWaitEvent(s->stream, s->ev_sumdone, 0);
  if (copy_out && s->n) {
    const size_t n = s->n;
    cudaMemcpyAsync(s->h_x, s->d_x, n * 8, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(s->h_y, s->d_y, n * 8, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(s->h_vx, s->d_vx, n * 8, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(s->h_vy, s->d_vy, n * 8, cudaMemcpyDeviceToHost, s->stream);
  }
  queue_status(s);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return D3_WORKER_FAILED;
  float ms = 0;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  s->last_ms = ms;
  return take_failure(s);
}

}  // namespace

extern "C" {

int32_t sim_tick(uint32_t h, uint32_t ticks, double *alpha, double alpha_target, double alpha_decay,
                 double velocity_decay, const uint32_t *order, uint32_t n_order) {
  DSim *s = get_sim_raw(h);
  if (!s) return D3_BAD_HANDLE;
  return tick_impl(s, ticks, alpha, alpha_target, alpha_decay, velocity_decay, order, n_order,
                   false);
}

int32_t sim_tick_sync(uint32_t h, uint32_t ticks, double *alpha, double alpha_target,
                      double alpha_decay, double velocity_decay, const uint32_t *order,
                      uint32_t n_order) {
  DSim *s = get_sim_raw(h);
  if (!s) return D3_BAD_HANDLE;
  sync_in_impl(s, true);
  return tick_impl(s, ticks, alpha, alpha_target, alpha_decay, velocity_decay, order, n_order,
                   true);
}

int32_t sim_set_learned(uint32_t h, const float *params, uint32_t len, double tolerance,
                        uint32_t samples, uint32_t hold) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (!(tolerance > 0) || samples == 0 || samples > 4096) return D3_BAD_ARGUMENT;
  const int r = fmm_tc_set_learned(s->fast, params, len);
  if (r == -3) return D3_BAD_ARGUMENT;
  if (r < 0) return D3_OUT_OF_MEMORY;
  s->fast.learn_tol = tolerance;
  s->fast.learn_samples = samples;
  s->fast.learn_hold = hold;
  return D3_OK;
}

int32_t sim_fmm_leaves(uint32_t h, float *out, uint32_t cap) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return D3_WORKER_FAILED;
  const int n = fmm_tc_leaves(s->fast, out, cap);
  return n < 0 ? D3_WORKER_FAILED : n;
}

int32_t sim_selftest_wait(uint32_t h, uint32_t budget_us) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (budget_us == 0 || budget_us > 1000000) return D3_BAD_ARGUMENT;
  wait_selftest(status_word(s), budget_us, s->stream);
  queue_status(s);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return D3_WORKER_FAILED;
  return take_failure(s);
}

int32_t sim_set_profile(uint32_t h, uint32_t on) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  phase_collect(s);
  s->profile = on != 0;
  s->spec.profile = s->profile;
  for (int k = 0; k < 16; ++k) {
    s->phase_ms[k] = 0;
    s->phase_n[k] = 0;
  }
  return D3_OK;
}

double sim_stat(uint32_t h, uint32_t which) {
  DSim *s = get_sim(h);
  if (!s) return 0;
  if (which >= 100 && which < 116) {
    phase_collect(s);
    return s->phase_ms[which - 100];
  }
  if (which >= 200 && which < 216) {
    phase_collect(s);
    return (double)s->phase_n[which - 200];
  }
  if (which >= 1000 && which < 1144) {
    // the last parallel collide's raw stamps (globaltimer ns, and counts)
    unsigned long long st[144];
    if (cudaMemcpy(st, s->spec.stamps, sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return (double)st[which - 1000];
  }
  if (which >= 50 && which < 50 + TC_STATS) {
    // the fast many-body precision forms: 50 learned-form checks, 51 of them
    // that fell back, 52 the last check's sampled RMS, 53 cells of the last
    // run; its last pass: 54 M2L ms, 55 near-field (P2P) ms, 56 M2L tiles,
    // 57 M2L pairs, 58 P2P point pairs, 59 M2P and 60 P2L point-cell pairs,
    // 61 q; the last run's ms: 62 prepare, 63 geometry and lists, 64 upward,
    // 65 P2L, 66 downward, 67 the learned form's network, 68 the whole run,
    // 69 the far field
    double out[TC_STATS];
    fmm_tc_stats(s->fast, out);
    return out[which - 50];
  }
  if ((which >= 300 && which < 364) || (which >= 400 && which < 464)) {
    // the last parallel collide's first attempt: 300 + k microseconds from
    // the end of its list build to the last turn of depth k, 400 + k turns
    // of depth k
    unsigned long long st[144];
    if (cudaMemcpy(st, s->spec.stamps, sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (which >= 400) return (double)st[80 + (which - 400)];
    const unsigned long long a = st[10], b = st[16 + (which - 300)];
    return b > a ? (double)(b - a) * 1e-3 : 0;
  }
  uint32_t spec[16] = {0}, sc[2] = {0}, words[2] = {0};
  cudaMemcpyAsync(s->h_words, s->spec.counters, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                  s->stream);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return -1;
  memcpy(spec, s->h_words, sizeof spec);
  cudaMemcpyAsync(s->h_words + 8, s->scratch.counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                  s->stream);
  cudaMemcpyAsync(s->h_words + 10, s->d_words, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                  s->stream);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return -1;
  memcpy(sc, s->h_words + 8, sizeof sc);
  memcpy(words, s->h_words + 10, sizeof words);
  switch (which) {
    case 0: return spec[5];
    case 1: return spec[6];
    case 2: return spec[7];
    case 3: return sc[1];
    case 4: {
      uint32_t lv = 0;
      for (DForce *f : s->forces)
        if (f && f->kind == D3_LINK) lv = f->plan.levels;
      return lv;
    }
    case 5: return words[1] != 0;
    case 6: return (double)g_launches;
    case 7: return spec[8];   // collide turns that examined an unguessed head
    case 8: return spec[9];   // ... that overlapped an unguessed head
    case 9: return spec[10];  // inactive nodes whose turn would have written
    case 10: return spec[11]; // turns run from the recorded head list
    case 11: return spec[12]; // turns that traversed the tree
    case 28: return spec[13]; // turn waits that gave up
    case 19: {
      // microseconds of the first attempt's access-list build
      unsigned long long st[11];
      cudaMemcpy(st, s->spec.stamps, sizeof st, cudaMemcpyDeviceToHost);
      return st[10] > st[1] && st[1] ? (double)(st[10] - st[1]) / 1e3 : 0;
    }
    case 27: return s->last_enqueue_ms;
    case 30: case 31: case 32: case 33: case 34: case 35: case 36: case 37: {
      // microseconds of the last tree build's phases: 30 box, 31 keys, 32
      // sort, 33 runs, 34 cell counts, 35 their scan, 36 cell owners, 37 the
      // cells (block 0)
      unsigned long long st[9];
      cudaMemcpy(st, s->tree.stamps, sizeof st, cudaMemcpyDeviceToHost);
      const int k = (int)which - 30;
      return st[k + 1] >= st[k] ? (double)(st[k + 1] - st[k]) * 1e-3 : -1;
    }
    case 22: case 23: case 24: case 25: case 26: {
      // the last center sum: 22 / 23 microseconds of the exact x / y walks
      // (or serial sums, up to 65,536 nodes); the x walk's 24 record batches
      // rerun with their entry tests, 25 stretches added one by one, 26
      // records in all (24-26 are 0 for the serial sums)
      unsigned long long st[8];
      cudaMemcpy(st, s->scratch.csum_stamps, sizeof st, cudaMemcpyDeviceToHost);
      if (which >= 24) return (double)st[5 + (which - 24)];
      const unsigned long long a = st[2], b = st[3 + (which - 22)];
      return b >= a ? (double)(b - a) * 1e-3 : -1;
    }
    case 12: case 13: case 14: case 15: case 16: case 17: case 18: {
      // microseconds of the last parallel collide's phases: 12 guess, 13/14
      // attempt 1 turns / check, 15/16 attempt 2, 17/18 attempt 3
      unsigned long long st[16];
      cudaMemcpy(st, s->spec.stamps, sizeof st, cudaMemcpyDeviceToHost);
      int k = which - 12;
      if (!st[k] || !st[k + 1]) return 0;
      return (double)(st[k + 1] - st[k]) / 1e3;
    }
    default: return 0;
  }
}

int32_t sim_find(uint32_t h, double x, double y, double radius, uint32_t *index) {
  DSim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (!index) return D3_BAD_ARGUMENT;
  *index = NONE;
  if (s->n == 0) return D3_OK;
  if (s->sync_mode == D3_SYNC_PER_CALL) sync_in_impl(s);
  // d3 squares the radius it is given (a missing one is Infinity)
  find_closest(nodes_of(s), x, y, radius * radius, s->d_words + 15, s->stream);
  cudaMemcpyAsync(s->h_words + 30, s->d_words + 15, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                  s->stream);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return D3_WORKER_FAILED;
  *index = s->h_words[30];
  return D3_OK;
}

double sim_last_tick_ms(uint32_t h) {
  DSim *s = get_sim(h);
  return s ? s->last_ms : 0;
}

}  // extern "C"
