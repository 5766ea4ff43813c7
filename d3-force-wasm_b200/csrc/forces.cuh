// forces.cuh — exact-mode force kernels and their launch wrappers.
#pragma once

#include <functional>

#include "common.cuh"
#include "tree.cuh"

namespace d3 {

struct NodeArrays {
  double *x, *y, *vx, *vy, *fx, *fy;
  uint8_t *fixed;
  double *px, *py;     // shifted positions (collide, fast link)
  double *snap_vx, *snap_vy;
  uint32_t n;
};

// Per-simulation device scratch for the force kernels.
struct ForceScratch {
  uint32_t cap = 0;
  uint32_t *draws = nullptr;    // jiggle draws per node (many-body record pass)
  uint32_t *offsets = nullptr;  // exclusive scan of draws
  uint32_t *scan_part = nullptr;
  uint32_t *counters = nullptr; // 0 total draws, 1 flagged, 2.. misc
  double *center = nullptr;     // 2 sums
  void *csum_recs = nullptr;    // the center sum's records, all chunks in order
  uint32_t *csum_counts = nullptr;  // ... record counts per chunk, then their offsets
  double *csum_part = nullptr;  // ... approximate chunk sums
  uint32_t *csum_scan_part = nullptr;  // ... the offsets scan's partials
  unsigned long long *csum_stamps = nullptr;  // the last center sum's timestamps and counts
};

int scratch_reserve(ForceScratch &s, uint32_t n);

// A device wait that cannot end, bounded by budget_us: sets ST_WAIT_TIMEOUT.
void wait_selftest(uint32_t *status, uint32_t budget_us, cudaStream_t st);
void scratch_free(ForceScratch &s);

struct ManyBodyParams {
  double theta2, dmin2, dmax2, alpha;
};

// many_body.zig:31-84 on the device. `rng` is device memory; in host-draw
// mode the caller must run the rerun itself (returns the draws needed via
// scratch.counters[0] after a sync).
// `mark(phase)` is called after the tree build (0) and the accumulation (1),
// so the caller can time the phases.
void many_body_exact(TreeDev &t, const NodeArrays &a, const double *strengths,
                     const ManyBodyParams &p, Rng *rng, ForceScratch &s, uint32_t *status,
                     bool host_draws, cudaStream_t st,
                     const std::function<void(int)> &mark = std::function<void(int)>());
// The rerun of flagged nodes with their draws (after many_body_exact).
void many_body_rerun(TreeDev &t, const NodeArrays &a, const double *strengths,
                     const ManyBodyParams &p, Rng *rng, ForceScratch &s, cudaStream_t st);

// Link levels (computed on the host from source/target): links grouped by
// level so that links sharing a node keep their order (link.zig:8-40).
struct LinkPlan {
  uint32_t m = 0, levels = 0, nodes = 0;
  uint32_t *order = nullptr;        // device: link ids grouped by level
  uint32_t *level_start = nullptr;  // device: levels + 1 offsets
  uint32_t *h_level_start = nullptr;
  uint32_t *need = nullptr;         // device: per position in order, the earlier links on
                                    // its source, then on its target (2 per link)
  uint32_t *done = nullptr;         // device: per node, links on it finished (this pass)
};
int link_plan_build(LinkPlan &plan, const uint32_t *src, const uint32_t *tgt, uint32_t m);
void link_plan_free(LinkPlan &plan);

struct LinkArrays {
  const double *strength, *distance, *bias;
  const uint32_t *source, *target;
  uint32_t m;
};

// Exact link: Gauss-Seidel in dependency order. A link that meets a zero /
// NaN delta (where d3 draws from `random`) sets *flag and the pass is undone
// (velocities restored from the snapshot); with serial_lcg the serial pass on
// the device LCG then runs in the same launch, otherwise the caller runs it.
void link_exact(const NodeArrays &a, const LinkArrays &l, const LinkPlan &plan, double alpha,
                double iterations, Rng *rng, uint32_t *flag, uint32_t *status, bool serial_lcg,
                cudaStream_t st);
// The serial pass on the device LCG, only when *flag is set.
void link_fallback_lcg(const NodeArrays &a, const LinkArrays &l, double alpha, double iterations,
                       Rng *rng, const uint32_t *flag, uint32_t *status, cudaStream_t st);
// Serial link from (iteration, link) with host draws; returns via resume[]:
// resume[0] iteration, resume[1] link, resume[2] draws still needed (0 = done).
void link_serial_host(const NodeArrays &a, const LinkArrays &l, double alpha, double iterations,
                      Rng *rng, uint32_t *resume, cudaStream_t st);

struct CollideParams {
  double strength;
  double iterations;
};
// px = x + vx, py = y + vy (sim.zig:129-146).
void shift_positions(const NodeArrays &a, cudaStream_t st);
// One collide iteration's set-up: px = x + vx, tree on (px, py), radii per cell.
void collide_setup(TreeDev &t, const NodeArrays &a, const double *radii, uint32_t *status,
                   cudaStream_t st);
// The ordered node loop of one iteration from node resume[0] (serial).
void collide_serial(TreeDev &t, const NodeArrays &a, const double *radii, double strength, Rng *rng,
                    bool host_draws, uint32_t *resume, cudaStream_t st);

// Scratch of the parallel exact collide (collide_spec.cu).
struct CollideSpec {
  uint32_t cap = 0;
  uint32_t *rlist = nullptr;
  uint8_t *rcount = nullptr;
  uint64_t *wmask = nullptr, *emask = nullptr;
  uint8_t *state = nullptr;
  uint32_t *active = nullptr;
  uint32_t *cnt = nullptr, *rlen = nullptr, *roff = nullptr;  // the access lists
  uint64_t *ent = nullptr, *ents = nullptr, *pr = nullptr;
  uint32_t *lev = nullptr, *aflag = nullptr, *apos = nullptr, *sact = nullptr;
  uint32_t *grid_part = nullptr;  // 1024 words: grid scan partials
  uint32_t *work = nullptr;  // 3 * cap: items shared out to whole warps
  double *push = nullptr;
  uint32_t *min_pusher = nullptr, *max_pusher = nullptr;
  uint32_t *vlist = nullptr;
  uint32_t *vaux = nullptr;    // per recorded cell: a leaf's head (tagged) or its skip link
  uint16_t *vcount = nullptr;
  uint32_t *start = nullptr;
  double *mdelta = nullptr, *push_prev = nullptr;
  uint32_t *counters = nullptr;  // collide_spec.cu C_*
  unsigned long long *stamps = nullptr;
  int profile = 0;  // per-depth stamps of the first attempt (sim_set_profile)
};
int collide_spec_reserve(CollideSpec &s, uint32_t n);
void collide_spec_free(CollideSpec &s);
// One iteration's node loop, in parallel and bit-identical to the serial
// order (after collide_setup). `delta`: the guess margin. LCG random only.
int collide_parallel(TreeDev &t, const NodeArrays &a, const double *radii, double strength,
                     double delta, Rng *rng, CollideSpec &s, cudaStream_t st);

// simple.zig:14-31 in two steps: the sums of x and y in index order (bit-exact)
// into s.center, then the shift. The sums only read positions, so the caller
// may issue them early on another stream.
void center_sum(const NodeArrays &a, ForceScratch &s, uint32_t *status, cudaStream_t st);
// The same sums in a fixed tree order (chunk sums, then a reduction): for the
// fast many-body forms judged by RMS, where the tick is not bit-exact anyway.
void center_sum_tree(const NodeArrays &a, ForceScratch &s, cudaStream_t st);
// src/core.js:130: the fixed bits from fx / fy (NaN = not set).
void fixed_from_f(const double *fx, const double *fy, uint8_t *fixed, uint32_t n, cudaStream_t st);
// simulation.js:157-178: the closest node below radius^2 (r2) into *out.
void find_closest(const NodeArrays &a, double x, double y, double r2, uint32_t *out,
                  cudaStream_t st);
void center_apply(const NodeArrays &a, double cx, double cy, double strength, ForceScratch &s,
                  cudaStream_t st);
void axis_force(const NodeArrays &a, const double *strength, const double *target, double alpha,
                int dim, cudaStream_t st);
void radial_force(const NodeArrays &a, const double *strength, const double *radius, double cx,
                  double cy, double alpha, cudaStream_t st);
void integrate(const NodeArrays &a, double decay, cudaStream_t st);
// center_apply followed by integrate, in one launch.
void center_apply_integrate(const NodeArrays &a, double cx, double cy, double strength,
                            ForceScratch &s, double decay, cudaStream_t st);

}  // namespace d3
