/* d3force_b200.h — C ABI of the B200 d3-force tick engine.
 *
 * The export set mirrors the core of d3-force-wasm (`src/core/root.zig`):
 * flat C-style calls that take a simulation handle plus integers or f64 and
 * return an i32 status or an index. Handles are 1-based with slot reuse.
 * Pointers returned by `sim_ptr` / `force_ptr` / `tree_info` are host
 * addresses of pinned host mirrors of the device arrays (the reference
 * returned wasm linear-memory offsets); they stay valid until the next call
 * that returns D3_GROWN or resizes the simulation.
 *
 * Residency: the device copy is the working copy. Host writes through the
 * mirrors reach the device at `sim_sync_in` (or, in D3_SYNC_PER_CALL mode,
 * at the start of every force_run / sim_integrate); results reach the mirrors
 * at `sim_sync_out` (or after every call in D3_SYNC_PER_CALL mode).
 *
 * Threading: one caller thread per simulation; not reentrant (as the
 * reference, root.zig: single caller thread, `random` called back on it).
 */
#ifndef D3FORCE_B200_H
#define D3FORCE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: root.zig:16-25 (`Status`). A device-side failure (a bounded
 * wait that ran out, a buffer found too small) is reported as
 * D3_WORKER_FAILED by the next call that synchronises with the device
 * (sim_sync_out, sim_tick, or any call in D3_SYNC_PER_CALL mode). */
enum {
  D3_OK = 0,
  D3_GROWN = 1,
  D3_ARENA_FULL = 2,
  D3_RNG_EXHAUSTED = 3,
  D3_BAD_HANDLE = -1,
  D3_OUT_OF_MEMORY = -2,
  D3_BAD_ARGUMENT = -3,
  D3_WORKER_FAILED = -4 /* a device-side bounded wait expired */
};

/* Force kinds: force.zig:8 (`Kind`). */
enum { D3_CENTER = 0, D3_COLLIDE, D3_LINK, D3_MANY_BODY, D3_RADIAL, D3_X, D3_Y };

/* Scalar slots: force.zig:13 (`Scalar`). */
enum {
  D3_STRENGTH = 0, D3_CX, D3_CY, D3_THETA2, D3_DISTANCE_MIN2, D3_DISTANCE_MAX2,
  D3_ITERATIONS, D3_PRECISION, D3_ORDER, D3_OPENING, D3_SEED, D3_SCALARS
};

/* Array slots: force.zig:21 (`Array`). Per kind: many_body f0 strength;
 * collide f0 radius; x, y f0 strength, f1 target; radial f0 strength,
 * f1 radius; link f0 strength, f1 distance, f2 bias, source, target. */
enum { D3_F0 = 0, D3_F1, D3_F2, D3_SOURCE, D3_TARGET };

/* sim_ptr selectors: sim.zig:14 (`Ptr`). */
enum {
  D3_PTR_X = 0, D3_PTR_Y, D3_PTR_VX, D3_PTR_VY, D3_PTR_FX, D3_PTR_FY,
  D3_PTR_FIXED, D3_PTR_PERM, D3_PTR_RNG_BUF, D3_PTR_SNAP
};

/* ---- Exports with a counterpart in root.zig ---------------------------- */

/* root.zig:65 `sim_create`: a new empty simulation; 0 on failure. */
uint32_t sim_create(void);
/* root.zig:80 `sim_destroy`. */
int32_t sim_destroy(uint32_t h);
/* root.zig:88 `sim_set_node_count`: OK, GROWN (mirrors moved) or OUT_OF_MEMORY.
 * Node-sized force arrays follow the count, padded with NaN (sim.zig:59-73). */
int32_t sim_set_node_count(uint32_t h, uint32_t n);
/* root.zig:94 `sim_ptr`: host mirror of x, y, vx, vy, fx, fy (f64[n]),
 * fixed (u8[n], bit 0 = fx set, bit 1 = fy set), perm (u32[m] after a tree
 * build), snap (f64[4n] after sim_snapshot). 0 when empty. */
uintptr_t sim_ptr(uint32_t h, uint32_t which);
/* root.zig:147 `force_create`: a force of `kind`; 0 on failure. */
uint32_t force_create(uint32_t h, uint32_t kind);
/* root.zig:163 `force_destroy`. */
int32_t force_destroy(uint32_t h, uint32_t fh);
/* root.zig:174 `force_set_count`: resizes every array of the force to
 * `count` (nodes, or links for link); new floats NaN, new indices 0.
 * Always returns GROWN (force.zig:65-82). */
int32_t force_set_count(uint32_t h, uint32_t fh, uint32_t count);
/* root.zig:181 `force_ptr`: host mirror of f0, f1, f2 (f64), source, target (u32). */
uintptr_t force_ptr(uint32_t h, uint32_t fh, uint32_t which);
/* root.zig:188 `force_set_scalar` / root.zig:196 `force_get_scalar`. */
int32_t force_set_scalar(uint32_t h, uint32_t fh, uint32_t which, double v);
double force_get_scalar(uint32_t h, uint32_t fh, uint32_t which);
/* root.zig:211 `force_run`: applies the force with `alpha`. Exact kernels,
 * or fast kernels when PRECISION == 1 and n >= 2000 (root.zig:219-248).
 * BAD_ARGUMENT for a node-sized force with count < n or a link index >= n. */
int32_t force_run(uint32_t h, uint32_t fh, double alpha);
/* root.zig:250 `sim_integrate`: v *= decay, p += v, or pin to fx / fy. */
int32_t sim_integrate(uint32_t h, double velocity_decay);
/* root.zig:205 `sim_snapshot`: saves vx, vy (and x, y) into `snap`. */
int32_t sim_snapshot(uint32_t h, uint32_t positions);
/* root.zig:102 `tree_build`: the d3-quadtree-identical tree on positions
 * (shifted = 0) or on x + vx, y + vy (1). GROWN when tree mirrors moved. */
int32_t tree_build(uint32_t h, uint32_t shifted);
/* root.zig:113 `tree_info`: 0 cell count, 1 root, 2 cells (88-byte records:
 * child[4] u32, first u32, count u32, x0 y0 x1 y1 x y value r f64), 3 extent
 * (4 x f64), 4 perm, 5 sizeof(cell) = 88, 6 points in the tree. Pointers are
 * host addresses (the reference returned u32 offsets). */
uintptr_t tree_info(uint32_t h, uint32_t which);
/* root.zig:128 `tree_order`: cell indices in d3-quadtree `visit` order
 * (after = 0) or `visitAfter` order (after = 1) into out[cell count]. */
int32_t tree_order(uint32_t h, uint32_t after, uint32_t *out);

/* ---- Extensions (no counterpart in root.zig) -------------------------- */

/* Random source for exact-mode jiggle. The reference imports `env.random`
 * (root.zig:141) and calls it synchronously; here the caller either registers
 * a callback (called on the caller thread, in d3's draw order) or selects the
 * built-in d3 LCG (src/lcg.js: a = 1664525, c = 1013904223, m = 2^32) whose
 * state lives on the device. In LCG mode, force_run of a many_body, link or
 * collide force with PRECISION == 1 also draws that force's SEED from the
 * stream first, as the reference facade does before each run
 * (src/core.js:218-222). */
typedef double (*d3_random_fn)(void *ctx);
int32_t sim_set_random(uint32_t h, d3_random_fn fn, void *ctx);
int32_t sim_set_lcg(uint32_t h, uint32_t state);
/* The LCG state after every call issued so far (synchronises). */
uint32_t sim_get_lcg(uint32_t h);

enum { D3_SYNC_EXPLICIT = 0, D3_SYNC_PER_CALL = 1 };
int32_t sim_set_sync(uint32_t h, uint32_t mode);
/* Host mirrors -> device (node state, fixed bits, every force's arrays). */
int32_t sim_sync_in(uint32_t h);
/* Where the fixed bits come from at each upload of the node state: 0 (the
 * default, the reference core's contract) the fixed array as written; 1
 * derived on the device from fx and fy by src/core.js:130's rule, fixed =
 * (fx set) | (fy set) << 1, for a facade that stores a missing fx / fy as
 * NaN (the Python facade does; the JS copyIn stores null as 0, so it keeps
 * mode 0). In mode 1 the fixed mirror is neither read nor written, which
 * saves computing and uploading the bits on the host. */
int32_t sim_set_fixed_source(uint32_t h, uint32_t from_f);
/* Device -> host mirrors (x, y, vx, vy). */
int32_t sim_sync_out(uint32_t h);

/* Runs `ticks` ticks of simulation.js:63-79 on the device without returning
 * to the host: alpha += (alpha_target - alpha) * alpha_decay, then the forces
 * in `order[0..n_order)` with that alpha, then integrate. `*alpha` is read and
 * updated. Requires LCG random mode (or no force that may jiggle). */
int32_t sim_tick(uint32_t h, uint32_t ticks, double *alpha, double alpha_target,
                 double alpha_decay, double velocity_decay,
                 const uint32_t *order, uint32_t n_order);

/* Milliseconds of device time of the last sim_tick call (CUDA events). */
/* sim_sync_in, sim_tick and sim_sync_out in one call with one host
 * synchronisation: the node state's uploads, the ticks and the downloads are
 * queued back to back on the simulation's stream (the facade's tick() with
 * the device LCG). Same arguments and result as sim_tick. */
int32_t sim_tick_sync(uint32_t h, uint32_t ticks, double *alpha, double alpha_target,
                      double alpha_decay, double velocity_decay, const uint32_t *order,
                      uint32_t n_order);

double sim_last_tick_ms(uint32_t h);

/* simulation.js:157-178 (`find`) on the device copy of the positions (after
 * sim_sync_in, or uploaded first in D3_SYNC_PER_CALL mode): the node closest
 * to (x, y) among those with d2 = dx * dx + dy * dy < radius * radius (pass
 * INFINITY for d3's missing radius). d3's serial scan replaces its pick only
 * on a strictly smaller d2, so among equal d2 the lowest index wins; a NaN d2
 * never matches. *index = that node, or 0xffffffff when none matches.
 * Synchronises. */
int32_t sim_find(uint32_t h, double x, double y, double radius, uint32_t *index);

/* Diagnostics of the last force runs (synchronises):
 *   0 the longest chain of dependent turns of the last parallel exact
 *     collide, 1 its attempts, 2 1 if it fell back to the serial loop;
 *   3 nodes the last exact many-body traversal flagged for jiggle;
 *   4 link levels of the last exact link plan, 5 1 if the last exact link
 *     pass fell back to the serial order (a jiggle);
 *   6 kernels this library launched so far (all simulations);
 *   7, 8 turns of the last parallel collide that met an unguessed head /
 *     overlap, 9 inactive nodes whose turn would have written, 10 turns run
 *     from the recorded head list, 11 turns that traversed the tree;
 *   12-18 microseconds of the last parallel collide's phases (guess, then
 *     turns / check per attempt), 19 of its first attempt's access-list
 *     build (part of 13), 28 its turn waits that gave up (0 unless it
 *     failed);
 *   22 / 23 microseconds of the last center sum's exact x / y walks (the
 *     plain serial sums up to 65,536 nodes), 24 its x walk's record batches
 *     rerun with their entry tests, 25 stretches added one by one, 26
 *     records in all (24-26 are 0 after the serial sums);
 *   27 host milliseconds the last sim_tick spent queueing work;
 *   30-37 microseconds of the last tree build's phases (box, keys, sort,
 *     runs, cell counts, their scan, cell owners, the cells);
 *   with profiling on, 300 + k microseconds from the end of the last
 *     parallel collide's first list build to its last turn of depth k, and
 *     400 + k its turns of depth k (k < 63; 63 counts every deeper turn);
 *   1000 + k (k < 144) its raw stamps (globaltimer ns, then per-depth data);
 *   100 + k milliseconds and 200 + k count of phase k since
 *     sim_set_profile(h, 1): 0 many-body tree, 1 many-body accumulation,
 *     2 many-body traversal, 3 exact link, 4 collide tree and radii,
 *     5 collide node loop, 6 center, 7 integrate, 8 fast many-body, 9 fast
 *     link, 10 fast collide. */
double sim_stat(uint32_t h, uint32_t which);
/* Phase timers on (1) / off (0); both reset them. CUDA events on the
 * simulation's stream around each phase. */
int32_t sim_set_profile(uint32_t h, uint32_t on);

/* Test of the failure path of the engine's bounded device waits (no
 * counterpart in the reference): a kernel waits on a barrier that nothing
 * completes, gives up after budget_us microseconds (1 .. 1,000,000), and the
 * call returns D3_WORKER_FAILED; the simulation stays usable. */
int32_t sim_selftest_wait(uint32_t h, uint32_t budget_us);

/* ---- Fast many-body precision forms (no counterpart in the reference) ---
 *
 * force_set_scalar(h, fh, D3_PRECISION, v) of a many-body force picks the
 * fast-mode form: 1 the reference's FP64 FMM (bit for bit); 2 the
 * tensor-core FMM (geometric cells, level-free operators, M2L as BF16x3
 * tcgen05 contractions with FP32 accumulation, FP32 near field with an FP64
 * origin shift; ORDER up to 15, OPENING in [1, 2]); 3 the learned form:
 * order 4 plus a per-leaf network correcting L'_0, checked each tick against
 * an FP64 direct sum on sampled nodes, form 2 at ORDER (8 if below 5) when
 * the check fails. Link and collide run the fast kernels for 1, 2 and 3. A
 * finite distanceMax runs form 1. */

/* Installs the learned form's network: 5,122 floats (W1 [64][12], b1, W2
 * [64][64], b2, W3 [2][64], b3), the RMS tolerance of the sampled check, its
 * sample count (1 .. 4096) and the ticks to stay on the fallback after a
 * failed check. sim_stat 50..53: checks, fallbacks, last sampled RMS, cells;
 * of the last form-2/3 pass: 54 M2L ms, 55 near-field (P2P) ms, 56 M2L
 * tiles, 57 M2L pairs, 58 P2P point pairs, 59 M2P and 60 P2L point-cell
 * pairs, 61 q; of the last run (CUDA events): 62 prepare, 63 geometry and
 * lists, 64 upward, 65 P2L, 66 downward, 67 the network, 68 the whole run,
 * 69 the far field (from the wait on the near field to the end of L2P / M2P),
 * in ms. The near field and the upward pass run on a second stream beside
 * the other passes. */
int32_t sim_set_learned(uint32_t h, const float *params, uint32_t len, double tolerance,
                        uint32_t samples, uint32_t hold);

/* The last form-2/3 run's per-cell rows, 16 floats each: the network's 12
 * inputs, L'_0 (re, im) and its scale, then the cell index (float bits) for
 * leaves or -1. Copies when cap >= the cell count; returns the cell count. */
int32_t sim_fmm_leaves(uint32_t h, float *out, uint32_t cap);

/* The network on the device (no counterpart in the reference): x n x 12,
 * y n x 2 FP32 device pointers; params 5,122 floats (host).
 * d3_mlp_grad: the gradient of mean_i |MLP(x_i) - y_i|^2 (host grad[5122],
 * *loss). d3_mlp_train: `steps` Adam steps over consecutive batches of
 * `batch` samples, learning rate lr, params updated in place, per-step batch
 * losses into losses[steps] (may be NULL). d3_mlp_infer: y = MLP(x) on the
 * tensor cores (tensor_cores 1) or CUDA cores (0). */
int32_t d3_mlp_grad(const float *x, const float *y, uint32_t n, const float *params, float *grad,
                    float *loss);
int32_t d3_mlp_train(const float *x, const float *y, uint32_t n, uint32_t batch, uint32_t steps,
                     float lr, float *params, float *losses);
int32_t d3_mlp_infer(const float *x, uint32_t n, const float *params, float *y,
                     uint32_t tensor_cores);

/* ---- Batched fast mode (no counterpart in the reference) -----------------
 *
 * Many independent graphs, each a d3 simulation with forceManyBody (FMM order
 * 8, opening 1.5, distanceMin 1, strength -30), forceLink (distance 30, d3's
 * default strength and bias) and forceCollide (radius 3), in FP32, d3's alpha
 * schedule and velocity decay 0.4; one persistent kernel launch per tick for
 * all graphs (graphs taken largest first). Up to 16,384 nodes per graph.
 *
 * batch_create: node_counts[graphs], link_counts[graphs]; src / tgt the
 * links of every graph concatenated, as node indices local to their graph;
 * x / y the start positions of every node, concatenated. Returns a handle
 * (0 on a bad argument or no memory). batch_run: `ticks` ticks, captured
 * into one CUDA graph when `graph` is non-zero; *ms the device time.
 * batch_kick: the many-body kick alone at the current positions (x, y per
 * node, host float[2 x nodes]) and the alpha it used. batch_read: the node
 * state (any pointer may be NULL). batch_set_shape: threads per CTA (256,
 * 512, 1024), CTAs per SM (1, 2), points per FMM leaf (2 .. 256).
 * batch_autotune: times `ticks` ticks of each shape from the current state
 * (restored after each) and keeps the fastest; out[4]: threads, CTAs per SM,
 * leaf size, ms per tick. */
uint32_t batch_create(uint32_t graphs, const uint32_t *node_counts, const uint32_t *link_counts,
                      const uint32_t *src, const uint32_t *tgt, const float *x, const float *y);
int32_t batch_destroy(uint32_t h);
int32_t batch_set_shape(uint32_t h, uint32_t threads, uint32_t per_sm, uint32_t leaf_size);
int32_t batch_run(uint32_t h, uint32_t ticks, uint32_t graph, double *ms);
int32_t batch_kick(uint32_t h, float *out, double *alpha_used);
int32_t batch_read(uint32_t h, float *x, float *y, float *vx, float *vy);
int32_t batch_autotune(uint32_t h, uint32_t ticks, double *out);

/* ---- Device rates for the roofline (no counterpart in the reference) ----
 *
 * Times microbenchmarks on the current device with CUDA events and fills
 * out[0..7]: DADD/s, DMUL/s, DFMA/s, IEEE f64 divisions/s and square roots/s
 * over the whole GPU (independent chains, full occupancy); the one-way
 * handoff latency in microseconds between two SMs (a release store to a
 * global flag seen by another SM's acquire load, half a timed ping-pong
 * round trip); the SM count; the SM clock attribute in kHz. The exact tick
 * runs on the FP64 pipe without FMA and waits through L2, so these are its
 * roofline denominators; with len >= 9, out[8] = FP32 FMA/s (the fast forms'
 * near field). len must be >= 8. Every device wait is bounded;
 * D3_WORKER_FAILED if one ran out or a launch failed. Allocates and frees a
 * few bytes of device memory. */
int32_t d3_device_peaks(double *out, uint32_t len);

/* ---- Allocation-free entry point (no counterpart in the reference) ------
 *
 * For callers that cannot let a library allocate device memory (an engine
 * that owns and budgets all GPU memory, a frame or control loop where
 * cudaMalloc would add synchronisation and latency): the exact many-body
 * force of force_run (d3's Barnes-Hut, bit-identical) on caller-owned device
 * buffers x, y, vx, vy, strength (f64[n]), with all scratch taken from one
 * static device array sized for D3_NOALLOC_MAX_NODES nodes, held by every GPU
 * that loads the library until the process exits. No cudaMalloc / cudaFree is
 * called. `*lcg_state` (host) is d3's LCG state for jiggle draws, updated on
 * return. Runs on `stream` (a cudaStream_t; NULL = the default stream) and
 * returns when the work is done: every call ends by copying its status to
 * the host and synchronising `stream`, so no call can be made while that
 * stream is being captured into a CUDA graph. The first call on each device
 * looks up the array's device address (set-up, done once per device and safe
 * when threads race to it). Calls share the array: calls that overlap on the
 * GPU (other threads or streams) race. Returns D3_OK; D3_BAD_ARGUMENT when n
 * exceeds D3_NOALLOC_MAX_NODES or a pointer is missing; D3_ARENA_FULL when
 * the tree needs more cells than the array holds (4n + 1024; clustered input
 * can need that many: d3's quadtree makes a chain of single-child cells down
 * to the level that separates two close points), in which case vx and vy are
 * left unchanged; D3_WORKER_FAILED on a CUDA error, a failed launch or a
 * device-side failure (a bounded wait that ran out). */
#define D3_NOALLOC_MAX_NODES 8192u
int32_t d3_many_body_exact_noalloc(const double *x, const double *y, double *vx, double *vy,
                                   const double *strength, uint32_t n, double theta2,
                                   double distance_min2, double distance_max2, double alpha,
                                   uint32_t *lcg_state, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* D3FORCE_B200_H */
