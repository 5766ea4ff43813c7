/* d3force_oracle.c — CPU ORACLE for the d3-force tick (TEST INFRASTRUCTURE).
 *
 * This file is the checker, not the product: only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it. It restates, statement by statement
 * and single-threaded, the d3-force-wasm core (Zig, the files under
 * `src/core/`); the CPU baseline alone turns on threads (oracle_set_threads),
 * with bit-identical results. The core is itself a port of d3-force 3.0.0 /
 * d3-quadtree 3.0.1 (npm, pinned in the
 * reference's package-lock.json:29-48, not vendored). Every function cites the
 * reference file:line it follows. It exports the same C ABI as the CUDA engine
 * (include/d3force_b200.h), so one host driver runs either.
 *
 * Pinning: the exact quadtree against the reference's d3-quadtree traces
 * (test/fixtures/tree-traces.json), fast mode plus the simulation semantics
 * against test/fixtures/fast-golden.json (SHA-256 per checkpoint), exact
 * collide / center / phyllotaxis against d3's known answers (1e-6).
 *
 * Build: -O2 -ffp-contract=off -fno-fast-math (no FMA contraction, IEEE
 * semantics, as the reference's strict float mode and wasm's lack of FMA).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/d3force_b200.h"

#define NONE 0xffffffffu
#define KEY_LEVELS 32
#define MAX_DEPTH 2200 /* tree.zig:33 */

/* ------------------------------------------------------------------------ */
/* Random sources                                                            */
/* ------------------------------------------------------------------------ */

/* src/lcg.js:1-9, rng.zig:15-22: s = (a s + c) mod 2^32; s / 2^32. */
static double lcg_next(uint32_t *s) {
  uint64_t v = (1664525ull * (uint64_t)*s + 1013904223ull) % 4294967296ull;
  *s = (uint32_t)v;
  return (double)v / 4294967296.0;
}

/* hash.zig:10-15 splitmix64 finaliser of (seed, i, j, salt). */
static uint64_t hash_mix(uint64_t seed, uint32_t i, uint32_t j, uint32_t salt) {
  uint64_t h = seed ^ (((uint64_t)i << 32) | j) ^ ((uint64_t)salt * 0x9E3779B97F4A7C15ull);
  h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
  h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
  return h ^ (h >> 31);
}
/* hash.zig:18-25 */
static double hash_uniform(uint64_t seed, uint32_t i, uint32_t j, uint32_t salt) {
  return (double)(hash_mix(seed, i, j, salt) >> 11) * 0x1.0p-53;
}
static double hash_jiggle(uint64_t seed, uint32_t i, uint32_t j, uint32_t salt) {
  return (hash_uniform(seed, i, j, salt) - 0.5) * 1e-6;
}
/* hash.zig:28-30 */
static uint64_t seed_from(double v) {
  uint64_t u;
  memcpy(&u, &v, 8);
  return u;
}

/* ------------------------------------------------------------------------ */
/* Stable LSD radix sort (sort.zig:55-91), serial                            */
/* ------------------------------------------------------------------------ */

/* Sorts keys[0..m) by their low `bytes` bytes carrying vals; skips passes
 * whose digit is uniform. Results land back in keys/vals. */
static void radix_sort(uint64_t *keys, uint32_t *vals, uint64_t *kt, uint32_t *vt, uint32_t m,
                       uint32_t bytes) {
  if (m == 0) return;
  uint64_t *sk = keys, *dk = kt;
  uint32_t *sv = vals, *dv = vt;
  for (uint32_t b = 0; b < bytes; ++b) {
    uint32_t hist[256];
    memset(hist, 0, sizeof hist);
    unsigned sh = 8 * b;
    for (uint32_t k = 0; k < m; ++k) hist[(sk[k] >> sh) & 255]++;
    if (hist[(sk[0] >> sh) & 255] == m) continue;
    uint32_t run = 0;
    for (int d = 0; d < 256; ++d) {
      uint32_t c = hist[d];
      hist[d] = run;
      run += c;
    }
    for (uint32_t k = 0; k < m; ++k) {
      uint32_t d = (sk[k] >> sh) & 255;
      dk[hist[d]] = sk[k];
      dv[hist[d]] = sv[k];
      hist[d]++;
    }
    uint64_t *tk = sk; sk = dk; dk = tk;
    uint32_t *tv = sv; sv = dv; dv = tv;
  }
  if (sk != keys) {
    memcpy(keys, sk, (size_t)m * 8);
    memcpy(vals, sv, (size_t)m * 4);
  }
}

/* ------------------------------------------------------------------------ */
/* Exact quadtree (tree.zig)                                                 */
/* ------------------------------------------------------------------------ */

/* tree.zig:46-62, 88 bytes. */
typedef struct {
  uint32_t child[4];
  uint32_t first, count;
  double x0, y0, x1, y1;
  double x, y, value, r;
} Cell;

typedef struct {
  uint32_t lo, hi, depth, parent, slot;
  int sorted;
  double x0, y0, x1, y1;
} Frame;

typedef struct {
  double extent[4];
  Cell *cells;
  uint32_t len, cells_cap;
  uint32_t root;
  uint32_t m;
  uint32_t *perm, *perm_tmp;
  uint64_t *keys, *keys_tmp;
  uint32_t *diff;
  uint32_t *rest;
  uint32_t cap;
  uint32_t depth;
  Frame *stack;
  uint32_t stack_cap;
} Tree;

static int is_leaf(const Cell *c) {
  return c->child[0] == NONE && c->child[1] == NONE && c->child[2] == NONE && c->child[3] == NONE;
}

static int tree_reserve(Tree *t, uint32_t n) {
  if (n > t->cap) {
    uint32_t cap = n;
    t->perm = realloc(t->perm, (size_t)cap * 4);
    t->perm_tmp = realloc(t->perm_tmp, (size_t)cap * 4);
    t->keys = realloc(t->keys, (size_t)cap * 8);
    t->keys_tmp = realloc(t->keys_tmp, (size_t)cap * 8);
    t->diff = realloc(t->diff, (size_t)cap * 4);
    t->rest = realloc(t->rest, (size_t)cap * 4);
    if (!t->perm || !t->perm_tmp || !t->keys || !t->keys_tmp || !t->diff || !t->rest) return -1;
    t->cap = cap;
  }
  return 0;
}

static void tree_free(Tree *t) {
  free(t->cells); free(t->perm); free(t->perm_tmp); free(t->keys); free(t->keys_tmp);
  free(t->diff); free(t->rest); free(t->stack);
  memset(t, 0, sizeof *t);
}

/* tree.zig:148-187: d3-quadtree's cover(). */
static void tree_cover(Tree *t, double x, double y) {
  if (isnan(x) || isnan(y)) return;
  double x0 = t->extent[0], y0 = t->extent[1], x1 = t->extent[2], y1 = t->extent[3];
  if (isnan(x0)) {
    x0 = floor(x);
    x1 = x0 + 1;
    y0 = floor(y);
    y1 = y0 + 1;
  } else {
    double z = x1 - x0;
    if (z == 0 || z != z) z = 1;
    uint32_t guard = 0;
    while ((x0 > x || x >= x1 || y0 > y || y >= y1) && guard < MAX_DEPTH) {
      int i = ((y < y0) << 1) | (x < x0);
      z *= 2;
      switch (i) {
        case 0: x1 = x0 + z; y1 = y0 + z; break;
        case 1: x0 = x1 - z; y1 = y0 + z; break;
        case 2: x1 = x0 + z; y0 = y1 - z; break;
        default: x0 = x1 - z; y0 = y1 - z; break;
      }
      ++guard;
    }
  }
  t->extent[0] = x0; t->extent[1] = y0; t->extent[2] = x1; t->extent[3] = y1;
}

/* tree.zig:316-340 (with the per-chunk pass 230-248): bbox with addAll's strict
 * comparisons, first of -0 / 0 wins; m = points without a NaN coordinate.
 * Returns 0 when no point has finite coordinates. */
static int tree_box(Tree *t, const double *xs, const double *ys, uint32_t n, double b[4]) {
  double bx0 = INFINITY, by0 = INFINITY, bx1 = -INFINITY, by1 = -INFINITY;
  uint32_t m = 0;
  for (uint32_t i = 0; i < n; ++i) {
    double x = xs[i], y = ys[i];
    if (x != x || y != y) continue;
    if (x < bx0) bx0 = x;
    if (x > bx1) bx1 = x;
    if (y < by0) by0 = y;
    if (y > by1) by1 = y;
    ++m;
  }
  t->m = m;
  if (bx0 > bx1 || by0 > by1) return 0;
  b[0] = bx0; b[1] = by0; b[2] = bx1; b[3] = by1;
  return 1;
}

/* tree.zig:252-284 (exactKeys): the 32-level midpoint Morton key of (x, y). */
static uint64_t exact_key(const double *e, double x, double y) {
  double x0 = e[0], y0 = e[1], x1 = e[2], y1 = e[3];
  uint64_t key = 0;
  for (int lv = 0; lv < KEY_LEVELS; ++lv) {
    double xm = (x0 + x1) / 2;
    double ym = (y0 + y1) / 2;
    int right = x >= xm;
    if (right) x0 = xm; else x1 = xm;
    int bottom = y >= ym;
    if (bottom) y0 = ym; else y1 = ym;
    key = (key << 2) | ((uint64_t)bottom << 1) | (uint64_t)right;
  }
  return key;
}

/* The key pass and the stable sort over `k` worker threads, for the CPU
 * baseline only (oracle_set_threads): the reference spreads both over its
 * pool (tree.zig:371-388; sort.zig:55-91 with per-chunk histograms). Workers
 * take contiguous chunks, so the compaction keeps index order and every
 * pass stays stable: the result is the serial one bit for bit. */
typedef struct {
  Tree *t;
  const double *xs, *ys;
  uint32_t n, k;
  pthread_barrier_t bar;
  uint32_t valid[64];      /* points without a NaN coordinate, per chunk */
  uint32_t hist[64 * 256]; /* a pass's digit counts, per chunk */
} PrepShared;

typedef struct {
  PrepShared *sh;
  uint32_t w;
} PrepJob;

static void chunk_of(uint32_t n, uint32_t k, uint32_t w, uint32_t *lo, uint32_t *hi) {
  uint32_t per = (n + k - 1) / k;
  uint64_t a = (uint64_t)w * per, b = a + per;
  *lo = a < n ? (uint32_t)a : n;
  *hi = b < n ? (uint32_t)b : n;
}

static void *prep_worker(void *arg) {
  PrepJob *j = arg;
  PrepShared *sh = j->sh;
  Tree *t = sh->t;
  const uint32_t w = j->w, k = sh->k, n = sh->n, m = t->m;
  uint32_t lo, hi;
  chunk_of(n, k, w, &lo, &hi);
  /* keys of this chunk's points, by point index, into keys_tmp */
  uint32_t v = 0;
  for (uint32_t i = lo; i < hi; ++i) {
    double x = sh->xs[i], y = sh->ys[i];
    if (x != x || y != y) continue;
    t->keys_tmp[i] = exact_key(t->extent, x, y);
    ++v;
  }
  sh->valid[w] = v;
  pthread_barrier_wait(&sh->bar);
  /* compaction in index order (tree.zig:371-388): sorted candidates, then
   * the NaN points into rest */
  uint32_t off = 0, roff = 0;
  for (uint32_t u = 0; u < w; ++u) {
    uint32_t ulo, uhi;
    chunk_of(n, k, u, &ulo, &uhi);
    off += sh->valid[u];
    roff += (uhi - ulo) - sh->valid[u];
  }
  for (uint32_t i = lo; i < hi; ++i) {
    double x = sh->xs[i], y = sh->ys[i];
    if (x != x || y != y) {
      t->rest[roff++] = i;
      continue;
    }
    t->perm[off] = i;
    t->keys[off] = t->keys_tmp[i];
    ++off;
  }
  pthread_barrier_wait(&sh->bar);
  /* sort.zig:55-91 over chunks of the m candidates */
  uint32_t mlo, mhi;
  chunk_of(m, k, w, &mlo, &mhi);
  uint64_t *sk = t->keys, *dk = t->keys_tmp;
  uint32_t *sv = t->perm, *dv = t->perm_tmp;
  for (uint32_t b = 0; m && b < 8; ++b) {
    const unsigned shf = 8 * b;
    uint32_t *h = sh->hist + 256 * w;
    memset(h, 0, 256 * sizeof(uint32_t));
    for (uint32_t i = mlo; i < mhi; ++i) h[(sk[i] >> shf) & 255]++;
    pthread_barrier_wait(&sh->bar);
    /* the pass is skipped when one digit holds every key (as the serial
     * sort); else this chunk's place for each digit: all chunks' counts of
     * lower digits, then earlier chunks' counts of the same digit */
    const uint32_t d0 = (uint32_t)((sk[0] >> shf) & 255);
    uint32_t tot0 = 0;
    for (uint32_t u = 0; u < k; ++u) tot0 += sh->hist[256 * u + d0];
    const int skip = tot0 == m;
    uint32_t place[256];
    if (!skip) {
      uint32_t run = 0;
      for (int d = 0; d < 256; ++d) {
        uint32_t before = 0, all = 0;
        for (uint32_t u = 0; u < k; ++u) {
          uint32_t c = sh->hist[256 * u + d];
          if (u < w) before += c;
          all += c;
        }
        place[d] = run + before;
        run += all;
      }
      for (uint32_t i = mlo; i < mhi; ++i) {
        uint32_t d = (uint32_t)((sk[i] >> shf) & 255);
        dk[place[d]] = sk[i];
        dv[place[d]] = sv[i];
        place[d]++;
      }
    }
    pthread_barrier_wait(&sh->bar);
    if (!skip) {
      uint64_t *tk = sk; sk = dk; dk = tk;
      uint32_t *tv = sv; sv = dv; dv = tv;
    }
  }
  if (sk != t->keys) {
    memcpy(t->keys + mlo, sk + mlo, (size_t)(mhi - mlo) * 8);
    memcpy(t->perm + mlo, sv + mlo, (size_t)(mhi - mlo) * 4);
  }
  return NULL;
}

/* tree.zig:371-388 + exactKeys 252-284: extent by cover, 32-level midpoint
 * Morton keys, stable sort (over `threads` workers when threads > 1). */
static int tree_prepare(Tree *t, const double *xs, const double *ys, uint32_t n, int threads) {
  if (tree_reserve(t, n)) return -1;
  t->extent[0] = t->extent[1] = t->extent[2] = t->extent[3] = NAN;
  t->len = 0;
  t->root = NONE;
  t->m = 0;
  double b[4];
  if (!tree_box(t, xs, ys, n, b)) return 0;
  tree_cover(t, b[0], b[1]);
  tree_cover(t, b[2], b[3]);
  if (threads > 1 && n >= 8192) {
    PrepShared *sh = malloc(sizeof *sh);
    if (!sh) return -1;
    const uint32_t k = threads > 64 ? 64 : (uint32_t)threads;
    sh->t = t; sh->xs = xs; sh->ys = ys; sh->n = n; sh->k = k;
    pthread_barrier_init(&sh->bar, NULL, k);
    pthread_t th[64];
    PrepJob jobs[64];
    for (uint32_t w = 0; w < k; ++w) jobs[w] = (PrepJob){sh, w};
    for (uint32_t w = 1; w < k; ++w) pthread_create(&th[w], NULL, prep_worker, &jobs[w]);
    prep_worker(&jobs[0]);
    for (uint32_t w = 1; w < k; ++w) pthread_join(th[w], NULL);
    pthread_barrier_destroy(&sh->bar);
    free(sh);
    return 1;
  }
  const double *e = t->extent;
  uint32_t k = 0, rest = 0;
  for (uint32_t i = 0; i < n; ++i) {
    double x = xs[i], y = ys[i];
    if (x != x || y != y) {
      t->rest[rest++] = i;
      continue;
    }
    t->perm[k] = i;
    t->keys[k] = exact_key(e, x, y);
    ++k;
  }
  radix_sort(t->keys, t->perm, t->keys_tmp, t->perm_tmp, t->m, 8);
  return 1;
}

/* tree.zig:392-433: diff[k] = distinct-position changes in perm[1..k]. */
static void tree_runs(Tree *t, const double *xs, const double *ys) {
  if (t->m == 0) return;
  t->diff[0] = 0;
  uint32_t d = 0;
  for (uint32_t k = 1; k < t->m; ++k) {
    uint32_t p = t->perm[k], q = t->perm[k - 1];
    d += (xs[p] != xs[q] || ys[p] != ys[q]);
    t->diff[k] = d;
  }
}

/* tree.zig:437-444 */
static int tree_all_same(const Tree *t, const Frame *f, const double *xs, const double *ys) {
  if (f->sorted) return t->diff[f->hi - 1] == t->diff[f->lo];
  uint32_t p0 = t->perm[f->lo];
  for (uint32_t k = f->lo + 1; k < f->hi; ++k) {
    uint32_t p = t->perm[k];
    if (xs[p] != xs[p0] || ys[p] != ys[p0]) return 0;
  }
  return 1;
}

/* tree.zig:697-699 */
static int quadrant(double x, double y, double xm, double ym) {
  return ((y >= ym) << 1) | (x >= xm);
}

/* tree.zig:449-479: child ranges; stable midpoint partition below the keys. */
static void tree_split(Tree *t, const Frame *f, const double *xs, const double *ys, uint32_t out[5]) {
  out[0] = f->lo;
  out[4] = f->hi;
  if (f->sorted && f->depth < KEY_LEVELS) {
    unsigned shift = 62 - 2 * f->depth;
    uint32_t k = f->lo;
    for (uint32_t q = 1; q < 4; ++q) {
      while (k < f->hi && ((t->keys[k] >> shift) & 3) < q) ++k;
      out[q] = k;
    }
  } else {
    double xm = (f->x0 + f->x1) / 2;
    double ym = (f->y0 + f->y1) / 2;
    uint32_t counts[4] = {0, 0, 0, 0}, off[4];
    for (uint32_t k = f->lo; k < f->hi; ++k) {
      uint32_t p = t->perm[k];
      counts[quadrant(xs[p], ys[p], xm, ym)]++;
    }
    uint32_t sum = f->lo;
    for (int q = 0; q < 4; ++q) {
      off[q] = sum;
      out[q] = sum;
      sum += counts[q];
    }
    for (uint32_t k = f->lo; k < f->hi; ++k) {
      uint32_t p = t->perm[k];
      int q = quadrant(xs[p], ys[p], xm, ym);
      t->perm_tmp[off[q]++] = p;
    }
    memcpy(t->perm + f->lo, t->perm_tmp + f->lo, (size_t)(f->hi - f->lo) * 4);
  }
}

/* tree.zig:482-499 */
static Frame tree_child(const Frame *f, uint32_t q, uint32_t lo, uint32_t hi, uint32_t parent) {
  double xm = (f->x0 + f->x1) / 2;
  double ym = (f->y0 + f->y1) / 2;
  int right = (q & 1) != 0, bottom = (q & 2) != 0;
  Frame c;
  c.lo = lo;
  c.hi = hi;
  c.depth = f->depth + 1;
  c.parent = parent;
  c.slot = q;
  c.sorted = f->sorted && f->depth < KEY_LEVELS;
  c.x0 = right ? xm : f->x0;
  c.y0 = bottom ? ym : f->y0;
  c.x1 = right ? f->x1 : xm;
  c.y1 = bottom ? f->y1 : ym;
  return c;
}

/* Where a preorder walk puts its cells: the tree's own array, or a job's. */
typedef struct {
  Cell *cells;
  uint32_t len, cap;
  Frame *stack;
  uint32_t stack_cap;
  uint32_t depth;
} EmitBuf;

/* A subtree emitted on its own by the threaded emission: its root frame, its
 * cells (local indices, root at 0), and where they go in the tree. */
typedef struct {
  Frame f;
  EmitBuf b;
  uint32_t off;
  int err;
} EmitJob;

static int eb_push(EmitBuf *b, uint32_t *sp, Frame f) {
  if (*sp == b->stack_cap) {
    uint32_t cap = b->stack_cap ? 2 * b->stack_cap : 256;
    Frame *s = realloc(b->stack, (size_t)cap * sizeof(Frame));
    if (!s) return -1;
    b->stack = s;
    b->stack_cap = cap;
  }
  b->stack[(*sp)++] = f;
  return 0;
}

/* tree.zig:572-647 restated serially: the preorder walk from `root`, cells
 * appended to b (child links in b's indices). The threaded emission's top
 * walk passes cut > 0: a frame below the root with at most `cut` points is
 * then not walked but becomes a job. In its first pass (place == 0) the job
 * is appended to *jobs; in the second (place == 1) the next job in order
 * takes its subtree's cell count of indices, linked from its parent. */
static int emit_walk(Tree *t, const double *xs, const double *ys, EmitBuf *b, Frame root,
                     uint32_t cut, EmitJob **jobs, uint32_t *nj, uint32_t *jcap, int place) {
  uint32_t sp = 0;
  if (eb_push(b, &sp, root)) return -1;
  while (sp > 0) {
    Frame f = b->stack[--sp];
    if (cut && f.depth > root.depth && f.hi - f.lo <= cut) {
      if (!place) {
        if (*nj == *jcap) {
          uint32_t cap = *jcap ? 2 * *jcap : 64;
          EmitJob *js = realloc(*jobs, (size_t)cap * sizeof(EmitJob));
          if (!js) return -1;
          *jobs = js;
          *jcap = cap;
        }
        EmitJob *j = &(*jobs)[(*nj)++];
        memset(j, 0, sizeof *j);
        j->f = f;
        j->f.parent = NONE;
      } else {
        EmitJob *j = &(*jobs)[(*nj)++];
        j->off = b->len;
        if (f.parent != NONE) b->cells[f.parent].child[f.slot] = b->len;
        b->len += j->b.len;
      }
      continue;
    }
    if (b->len == b->cap) {
      uint32_t cap = b->cap ? 2 * b->cap : 2 * (root.hi - root.lo) + 64;
      Cell *c = realloc(b->cells, (size_t)cap * sizeof(Cell));
      if (!c) return -1;
      b->cells = c;
      b->cap = cap;
    }
    uint32_t me = b->len++;
    Cell *c = &b->cells[me];
    c->child[0] = c->child[1] = c->child[2] = c->child[3] = NONE;
    c->first = f.lo;
    c->count = f.hi - f.lo;
    c->x0 = f.x0; c->y0 = f.y0; c->x1 = f.x1; c->y1 = f.y1;
    c->x = c->y = c->value = c->r = 0;
    if (f.parent != NONE) b->cells[f.parent].child[f.slot] = me;
    if (f.depth > b->depth) b->depth = f.depth;
    if (f.depth >= MAX_DEPTH || tree_all_same(t, &f, xs, ys)) continue;
    uint32_t s5[5];
    tree_split(t, &f, xs, ys, s5);
    for (int q = 3; q >= 0; --q) {
      if (s5[q] == s5[q + 1]) continue;
      if (eb_push(b, &sp, tree_child(&f, (uint32_t)q, s5[q], s5[q + 1], me))) return -1;
    }
  }
  return 0;
}

static Frame root_frame(const Tree *t) {
  Frame root = {0, t->m, 0, NONE, 0, 1, t->extent[0], t->extent[1], t->extent[2], t->extent[3]};
  return root;
}

/* The serial emission: the whole walk into the tree's array. */
static int tree_emit(Tree *t, const double *xs, const double *ys) {
  EmitBuf b = {t->cells, 0, t->cells_cap, t->stack, t->stack_cap, 0};
  int r = emit_walk(t, xs, ys, &b, root_frame(t), 0, NULL, NULL, NULL, 0);
  t->cells = b.cells;
  t->cells_cap = b.cap;
  t->stack = b.stack;
  t->stack_cap = b.stack_cap;
  if (r) return -1;
  t->root = 0;
  t->len = b.len;
  t->depth = b.depth;
  return 0;
}

/* The threaded emission (CPU baseline only), as the reference's serial top
 * walk plus per-job walks: the top walk collects the subtrees of at most
 * max(m / 64, 64) points (jobs); workers walk the jobs into their own
 * buffers; a second top walk places every top cell and every job's block
 * of cells in preorder; workers copy the blocks in, their child links
 * shifted. The cells are those of the serial walk, index for index: a job's
 * block is its subtree's preorder, and the top walk visits the jobs in
 * preorder. */
typedef struct {
  Tree *t;
  const double *xs, *ys;
  EmitJob *jobs;
  uint32_t nj, k;
  pthread_barrier_t bar;
  int err;
} EmitShared;

typedef struct {
  EmitShared *sh;
  uint32_t w;
} EmitWorker;

static void *emit_worker(void *arg) {
  EmitWorker *ew = arg;
  EmitShared *sh = ew->sh;
  for (uint32_t j = ew->w; j < sh->nj; j += sh->k) {
    EmitJob *job = &sh->jobs[j];
    job->err = emit_walk(sh->t, sh->xs, sh->ys, &job->b, job->f, 0, NULL, NULL, NULL, 0);
  }
  pthread_barrier_wait(&sh->bar); /* the jobs are walked */
  pthread_barrier_wait(&sh->bar); /* the second top walk has placed them */
  if (sh->err) return NULL;
  for (uint32_t j = ew->w; j < sh->nj; j += sh->k) {
    EmitJob *job = &sh->jobs[j];
    Cell *dst = sh->t->cells + job->off;
    memcpy(dst, job->b.cells, (size_t)job->b.len * sizeof(Cell));
    for (uint32_t c = 0; c < job->b.len; ++c)
      for (int q = 0; q < 4; ++q)
        if (dst[c].child[q] != NONE) dst[c].child[q] += job->off;
  }
  return NULL;
}

static int tree_emit_threaded(Tree *t, const double *xs, const double *ys, int threads) {
  const uint32_t cut = t->m / 64 > 64 ? t->m / 64 : 64;
  EmitJob *jobs = NULL;
  uint32_t nj = 0, jcap = 0;
  EmitBuf top = {NULL, 0, 0, t->stack, t->stack_cap, 0};
  int r = emit_walk(t, xs, ys, &top, root_frame(t), cut, &jobs, &nj, &jcap, 0);
  free(top.cells);
  t->stack = top.stack;
  t->stack_cap = top.stack_cap;
  if (r) {
    free(jobs);
    return -1;
  }
  EmitShared *sh = malloc(sizeof *sh);
  if (!sh) {
    free(jobs);
    return -1;
  }
  const uint32_t k = threads > 64 ? 64 : (uint32_t)threads;
  sh->t = t; sh->xs = xs; sh->ys = ys; sh->jobs = jobs; sh->nj = nj; sh->k = k; sh->err = 0;
  pthread_barrier_init(&sh->bar, NULL, k);
  pthread_t th[64];
  EmitWorker ws[64];
  for (uint32_t w = 0; w < k; ++w) ws[w] = (EmitWorker){sh, w};
  for (uint32_t w = 1; w < k; ++w) pthread_create(&th[w], NULL, emit_worker, &ws[w]);
  /* worker 0's share of the jobs, then the second top walk between the
   * barriers, then its share of the copies */
  for (uint32_t j = 0; j < nj; j += k)
    jobs[j].err = emit_walk(t, xs, ys, &jobs[j].b, jobs[j].f, 0, NULL, NULL, NULL, 0);
  pthread_barrier_wait(&sh->bar);
  uint32_t total = top.len, depth = top.depth;
  for (uint32_t j = 0; j < nj; ++j) {
    if (jobs[j].err) sh->err = 1;
    total += jobs[j].b.len;
    if (jobs[j].b.depth > depth) depth = jobs[j].b.depth;
  }
  if (!sh->err && total > t->cells_cap) {
    Cell *c = realloc(t->cells, (size_t)total * sizeof(Cell));
    if (c) {
      t->cells = c;
      t->cells_cap = total;
    } else {
      sh->err = 1;
    }
  }
  if (!sh->err) {
    EmitBuf b = {t->cells, 0, t->cells_cap, t->stack, t->stack_cap, 0};
    uint32_t placed = 0;
    if (emit_walk(t, xs, ys, &b, root_frame(t), cut, &jobs, &placed, &jcap, 1)) sh->err = 1;
    t->cells = b.cells;
    t->cells_cap = b.cap;
    t->stack = b.stack;
    t->stack_cap = b.stack_cap;
  }
  pthread_barrier_wait(&sh->bar);
  if (!sh->err) {
    for (uint32_t j = 0; j < nj; j += k) {
      Cell *dst = t->cells + jobs[j].off;
      memcpy(dst, jobs[j].b.cells, (size_t)jobs[j].b.len * sizeof(Cell));
      for (uint32_t c = 0; c < jobs[j].b.len; ++c)
        for (int q = 0; q < 4; ++q)
          if (dst[c].child[q] != NONE) dst[c].child[q] += jobs[j].off;
    }
  }
  for (uint32_t w = 1; w < k; ++w) pthread_join(th[w], NULL);
  const int err = sh->err;
  pthread_barrier_destroy(&sh->bar);
  free(sh);
  for (uint32_t j = 0; j < nj; ++j) {
    free(jobs[j].b.cells);
    free(jobs[j].b.stack);
  }
  free(jobs);
  if (err) return -1;
  t->root = 0;
  t->len = total;
  t->depth = depth;
  return 0;
}

/* tree.zig:191-196 */
static int tree_build_xy(Tree *t, const double *xs, const double *ys, uint32_t n, int threads) {
  int r = tree_prepare(t, xs, ys, n, threads);
  if (r <= 0) return r;
  tree_runs(t, xs, ys);
  if (threads > 1 && t->m >= 8192) return tree_emit_threaded(t, xs, ys, threads);
  return tree_emit(t, xs, ys);
}

/* tree.zig:652-684: visit (preorder) / visitAfter (post-order) order. */
static int tree_order_impl(const Tree *t, int after, uint32_t *out) {
  if (t->root == NONE) return 0;
  uint32_t *stack = malloc((size_t)(t->len > 0 ? t->len : 1) * 4);
  if (!stack) return -1;
  uint32_t sp = 0, w = 0;
  stack[sp++] = t->root;
  while (sp > 0) {
    uint32_t c = stack[--sp];
    out[w++] = c;
    const uint32_t *ch = t->cells[c].child;
    if (after) {
      for (int i = 0; i < 4; ++i) if (ch[i] != NONE) stack[sp++] = ch[i];
    } else {
      for (int i = 3; i >= 0; --i) if (ch[i] != NONE) stack[sp++] = ch[i];
    }
  }
  if (after) {
    for (uint32_t i = 0, j = w ? w - 1 : 0; i < j; ++i, --j) {
      uint32_t tmp = out[i]; out[i] = out[j]; out[j] = tmp;
    }
  }
  free(stack);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Simulation and force tables (sim.zig, force.zig, root.zig)                */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint32_t kind;
  double scalars[D3_SCALARS];
  uint32_t count;
  double *f0, *f1, *f2;
  uint32_t *source, *target;
  uint32_t *csr_ptr, *csr_adj;
  uint32_t csr_n;
} Force;

/* fmm.zig:68-78 */
typedef struct {
  double cx, cy, r;
  uint32_t first, count, child0, nchild, depth, pad;
} FCell;

typedef struct {
  uint32_t n, cap;
  double *x, *y, *vx, *vy, *fx, *fy;
  uint8_t *fixed;
  int fixed_from_f; /* sim_set_fixed_source */
  double *px, *py;
  double *snap;
  uint32_t snap_cap;
  Tree tree;
  /* fast many-body */
  FCell *fcells;
  uint32_t flen, fcap;
  double *ux, *uy, *fpx, *fpy, *fps;
  uint32_t pts_cap;
  double *bx0, *by0, *bx1, *by1;
  double *mco, *lco;
  size_t coef_cap;
  /* grid */
  uint32_t *g_start, *g_items, *g_items_tmp, *g_cell_of;
  uint64_t *g_keys, *g_keys_tmp;
  uint32_t g_cap, g_start_cap;
  /* forces */
  Force **forces;
  uint32_t n_forces;
  /* random */
  int rand_mode; /* 0 = LCG, 1 = callback */
  uint32_t lcg;
  d3_random_fn rand_fn;
  void *rand_ctx;
  int threads;
} Sim;

static Sim **sims = NULL;
static uint32_t n_sims = 0;

static Sim *get_sim(uint32_t h) {
  if (h == 0 || h > n_sims) return NULL;
  return sims[h - 1];
}

static Force *get_force(Sim *s, uint32_t fh) {
  if (fh == 0 || fh > s->n_forces) return NULL;
  return s->forces[fh - 1];
}

static double sim_random(Sim *s) {
  if (s->rand_mode == 1 && s->rand_fn) return s->rand_fn(s->rand_ctx);
  return lcg_next(&s->lcg);
}

/* rng.zig:8-11, d3's jiggle.js. */
static double jiggle(Sim *s) {
  return (sim_random(s) - 0.5) * 1e-6;
}

uint32_t sim_create(void) {
  Sim *s = calloc(1, sizeof(Sim));
  if (!s) return 0;
  s->lcg = 1;
  s->threads = 1;
  for (uint32_t i = 0; i < n_sims; ++i)
    if (!sims[i]) {
      sims[i] = s;
      return i + 1;
    }
  Sim **ns = realloc(sims, (size_t)(n_sims + 1) * sizeof(Sim *));
  if (!ns) {
    free(s);
    return 0;
  }
  sims = ns;
  sims[n_sims++] = s;
  return n_sims;
}

static void force_free(Force *f) {
  free(f->f0); free(f->f1); free(f->f2); free(f->source); free(f->target);
  free(f->csr_ptr); free(f->csr_adj);
  free(f);
}

int32_t sim_destroy(uint32_t h) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  free(s->x); free(s->y); free(s->vx); free(s->vy); free(s->fx); free(s->fy); free(s->fixed);
  free(s->px); free(s->py); free(s->snap);
  tree_free(&s->tree);
  free(s->fcells); free(s->ux); free(s->uy); free(s->fpx); free(s->fpy); free(s->fps);
  free(s->bx0); free(s->by0); free(s->bx1); free(s->by1); free(s->mco); free(s->lco);
  free(s->g_start); free(s->g_items); free(s->g_items_tmp); free(s->g_cell_of);
  free(s->g_keys); free(s->g_keys_tmp);
  for (uint32_t i = 0; i < s->n_forces; ++i)
    if (s->forces[i]) force_free(s->forces[i]);
  free(s->forces);
  free(s);
  sims[h - 1] = NULL;
  return D3_OK;
}

/* force.zig:59-63 */
static int node_sized(const Force *f) {
  return f->kind != D3_LINK && f->kind != D3_CENTER;
}

/* force.zig:65-82 */
static int force_set_count_impl(Force *f, uint32_t count) {
  uint32_t old = f->count;
  int k = f->kind == D3_CENTER ? 0 : (f->kind == D3_COLLIDE || f->kind == D3_MANY_BODY) ? 1
        : f->kind == D3_LINK ? 3 : 2;
  double **arrs[3] = {&f->f0, &f->f1, &f->f2};
  for (int i = 0; i < k; ++i) {
    double *a = realloc(*arrs[i], (size_t)(count ? count : 1) * 8);
    if (!a) return -1;
    *arrs[i] = a;
    for (uint32_t j = old; j < count; ++j) a[j] = NAN;
  }
  if (f->kind == D3_LINK) {
    uint32_t *s = realloc(f->source, (size_t)(count ? count : 1) * 4);
    if (!s) return -1;
    f->source = s;
    uint32_t *t = realloc(f->target, (size_t)(count ? count : 1) * 4);
    if (!t) return -1;
    f->target = t;
    for (uint32_t j = old; j < count; ++j) f->source[j] = f->target[j] = 0;
  }
  f->count = count;
  f->csr_n = 0;
  return 0;
}

/* sim.zig:59-73 */
int32_t sim_set_node_count(uint32_t h, uint32_t n) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  s->n = n;
  int grown = 0;
  for (uint32_t i = 0; i < s->n_forces; ++i) {
    Force *f = s->forces[i];
    if (f && node_sized(f) && f->count < n) {
      if (force_set_count_impl(f, n)) return D3_OUT_OF_MEMORY;
      grown = 1;
    }
  }
  if (n <= s->cap) return grown ? D3_GROWN : D3_OK;
  uint32_t cap = n;
  if (s->cap * 2 > cap) cap = s->cap * 2;
  if (cap < 16) cap = 16;
  double **d[] = {&s->x, &s->y, &s->vx, &s->vy, &s->fx, &s->fy, &s->px, &s->py};
  for (int i = 0; i < 8; ++i) {
    double *a = realloc(*d[i], (size_t)cap * 8);
    if (!a) return D3_OUT_OF_MEMORY;
    *d[i] = a;
  }
  uint8_t *fx = realloc(s->fixed, cap);
  if (!fx) return D3_OUT_OF_MEMORY;
  s->fixed = fx;
  s->cap = cap;
  return D3_GROWN;
}

uintptr_t sim_ptr(uint32_t h, uint32_t which) {
  Sim *s = get_sim(h);
  if (!s) return 0;
  switch (which) {
    case D3_PTR_X: return (uintptr_t)s->x;
    case D3_PTR_Y: return (uintptr_t)s->y;
    case D3_PTR_VX: return (uintptr_t)s->vx;
    case D3_PTR_VY: return (uintptr_t)s->vy;
    case D3_PTR_FX: return (uintptr_t)s->fx;
    case D3_PTR_FY: return (uintptr_t)s->fy;
    case D3_PTR_FIXED: return (uintptr_t)s->fixed;
    case D3_PTR_PERM: return (uintptr_t)s->tree.perm;
    case D3_PTR_SNAP: return (uintptr_t)s->snap;
    default: return 0;
  }
}

uint32_t force_create(uint32_t h, uint32_t kind) {
  Sim *s = get_sim(h);
  if (!s || kind > D3_Y) return 0;
  Force *f = calloc(1, sizeof(Force));
  if (!f) return 0;
  f->kind = kind;
  if (node_sized(f) && force_set_count_impl(f, s->n)) {
    force_free(f);
    return 0;
  }
  for (uint32_t i = 0; i < s->n_forces; ++i)
    if (!s->forces[i]) {
      s->forces[i] = f;
      return i + 1;
    }
  Force **nf = realloc(s->forces, (size_t)(s->n_forces + 1) * sizeof(Force *));
  if (!nf) {
    force_free(f);
    return 0;
  }
  s->forces = nf;
  s->forces[s->n_forces++] = f;
  return s->n_forces;
}

int32_t force_destroy(uint32_t h, uint32_t fh) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  Force *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  force_free(f);
  s->forces[fh - 1] = NULL;
  return D3_OK;
}

int32_t force_set_count(uint32_t h, uint32_t fh, uint32_t count) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  Force *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  if (force_set_count_impl(f, count)) return D3_OUT_OF_MEMORY;
  return D3_GROWN;
}

uintptr_t force_ptr(uint32_t h, uint32_t fh, uint32_t which) {
  Sim *s = get_sim(h);
  if (!s) return 0;
  Force *f = get_force(s, fh);
  if (!f || f->count == 0) return 0;
  switch (which) {
    case D3_F0: return (uintptr_t)f->f0;
    case D3_F1: return (uintptr_t)f->f1;
    case D3_F2: return (uintptr_t)f->f2;
    case D3_SOURCE: return (uintptr_t)f->source;
    case D3_TARGET: return (uintptr_t)f->target;
    default: return 0;
  }
}

int32_t force_set_scalar(uint32_t h, uint32_t fh, uint32_t which, double v) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  Force *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  if (which >= D3_SCALARS) return D3_BAD_ARGUMENT;
  f->scalars[which] = v;
  return D3_OK;
}

double force_get_scalar(uint32_t h, uint32_t fh, uint32_t which) {
  Sim *s = get_sim(h);
  if (!s) return 0;
  Force *f = get_force(s, fh);
  if (!f) return 0;
  return which < D3_SCALARS ? f->scalars[which] : 0;
}

/* sim.zig:91-100 */
int32_t sim_snapshot(uint32_t h, uint32_t positions) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  uint32_t n = s->n;
  if (s->snap_cap < 4 * n) {
    double *a = realloc(s->snap, (size_t)4 * (s->cap ? s->cap : 1) * 8);
    if (!a) return D3_OUT_OF_MEMORY;
    s->snap = a;
    s->snap_cap = 4 * s->cap;
  }
  memcpy(s->snap, s->vx, (size_t)n * 8);
  memcpy(s->snap + n, s->vy, (size_t)n * 8);
  if (positions) {
    memcpy(s->snap + 2 * n, s->x, (size_t)n * 8);
    memcpy(s->snap + 3 * n, s->y, (size_t)n * 8);
  }
  return D3_OK;
}

/* sim.zig:118-146 */
static int sim_build_tree(Sim *s, int shifted) {
  uint32_t n = s->n;
  if (shifted) {
    for (uint32_t i = 0; i < n; ++i) {
      s->px[i] = s->x[i] + s->vx[i];
      s->py[i] = s->y[i] + s->vy[i];
    }
    return tree_build_xy(&s->tree, s->px, s->py, n, s->threads);
  }
  return tree_build_xy(&s->tree, s->x, s->y, n, s->threads);
}

int32_t tree_build(uint32_t h, uint32_t shifted) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  Cell *cb = s->tree.cells;
  uint32_t *pb = s->tree.perm;
  if (sim_build_tree(s, shifted != 0) < 0) return D3_OUT_OF_MEMORY;
  return (s->tree.cells != cb || s->tree.perm != pb) ? D3_GROWN : D3_OK;
}

uintptr_t tree_info(uint32_t h, uint32_t which) {
  Sim *s = get_sim(h);
  if (!s) return 0;
  Tree *t = &s->tree;
  switch (which) {
    case 0: return t->len;
    case 1: return t->root;
    case 2: return (uintptr_t)t->cells;
    case 3: return (uintptr_t)t->extent;
    case 4: return (uintptr_t)t->perm;
    case 5: return sizeof(Cell);
    case 6: return t->m;
    default: return 0;
  }
}

int32_t tree_order(uint32_t h, uint32_t after, uint32_t *out) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (!out) return D3_BAD_ARGUMENT;
  if (tree_order_impl(&s->tree, after != 0, out)) return D3_OUT_OF_MEMORY;
  return D3_OK;
}

/* ------------------------------------------------------------------------ */
/* Exact many-body (many_body.zig)                                           */
/* ------------------------------------------------------------------------ */

/* many_body.zig:101-135: visitAfter accumulate. */
static void mb_accumulate(Tree *t, const double *xs, const double *ys, const double *strengths) {
  Cell *cells = t->cells;
  for (uint32_t c = t->len; c-- > 0;) {
    Cell *quad = &cells[c];
    double strength = 0;
    if (!is_leaf(quad)) {
      double weight = 0, x = 0, y = 0;
      for (int k = 0; k < 4; ++k) {
        uint32_t ch = quad->child[k];
        if (ch == NONE) continue;
        const Cell *q = &cells[ch];
        double w = fabs(q->value);
        if (w > 0) {
          strength += q->value;
          weight += w;
          x += w * q->x;
          y += w * q->y;
        }
      }
      quad->x = x / weight;
      quad->y = y / weight;
    } else {
      uint32_t head = t->perm[quad->first + quad->count - 1];
      quad->x = xs[head];
      quad->y = ys[head];
      for (uint32_t k = quad->first + quad->count; k > quad->first;) {
        --k;
        strength += strengths[t->perm[k]];
      }
    }
    quad->value = strength;
  }
}

typedef struct {
  const Tree *t;
  const double *xs, *ys, *strengths;
  double *vxs, *vys;
  double theta2, dmin2, dmax2, alpha;
  Sim *s; /* random source; NULL = record mode (report, do not draw) */
} MbTrav;

/* Work counters of the exact many-body traversal (for the roofline, not part
 * of the reference): cells visited, accepted far-field approximations, leaf
 * point interactions. */
static uint64_t mb_visits, mb_accepts, mb_points;

static void mb_count(uint64_t v, uint64_t a, uint64_t pts) {
  __atomic_add_fetch(&mb_visits, v, __ATOMIC_RELAXED);
  __atomic_add_fetch(&mb_accepts, a, __ATOMIC_RELAXED);
  __atomic_add_fetch(&mb_points, pts, __ATOMIC_RELAXED);
}

/* many_body.zig:176-263: d3's traversal for node i. With s == NULL it returns
 * 0 without writing at the first point where d3 would draw. */
static int mb_node(const MbTrav *p, uint32_t i, uint32_t *stack) {
  uint64_t nv = 0, na = 0, np = 0;
  const Cell *cells = p->t->cells;
  const uint32_t *perm = p->t->perm;
  double nx = p->xs[i], ny = p->ys[i];
  double vx = p->vxs[i], vy = p->vys[i];
  uint32_t sp = 1;
  stack[0] = p->t->root;
  while (sp > 0) {
    const Cell *quad = &cells[stack[--sp]];
    double value = quad->value;
    if (!(value != 0 && value == value)) continue;
    ++nv;
    double x = quad->x - nx, y = quad->y - ny;
    double w = quad->x1 - quad->x0;
    double l = x * x + y * y;
    if (w * w / p->theta2 < l) {
      if (l < p->dmax2) {
        ++na;
        if (!p->s && (x == 0 || y == 0)) { mb_count(nv, na, np); return 0; }
        if (x == 0) { x = jiggle(p->s); l += x * x; }
        if (y == 0) { y = jiggle(p->s); l += y * y; }
        if (l < p->dmin2) l = sqrt(p->dmin2 * l);
        vx += x * value * p->alpha / l;
        vy += y * value * p->alpha / l;
      }
      continue;
    }
    if (!is_leaf(quad)) {
      for (int q = 3; q >= 0; --q)
        if (quad->child[q] != NONE) stack[sp++] = quad->child[q];
      continue;
    }
    if (l >= p->dmax2) continue;
    uint32_t head = perm[quad->first + quad->count - 1];
    if (head != i || quad->count > 1) {
      if (!p->s && (x == 0 || y == 0)) { mb_count(nv, na, np); return 0; }
      if (x == 0) { x = jiggle(p->s); l += x * x; }
      if (y == 0) { y = jiggle(p->s); l += y * y; }
      if (l < p->dmin2) l = sqrt(p->dmin2 * l);
    }
    for (uint32_t k = quad->first + quad->count; k > quad->first;) {
      --k;
      uint32_t j = perm[k];
      if (j != i) {
        ++np;
        double wj = p->strengths[j] * p->alpha / l;
        vx += x * wj;
        vy += y * wj;
      }
    }
  }
  p->vxs[i] = vx;
  p->vys[i] = vy;
  mb_count(nv, na, np);
  return 1;
}

typedef struct {
  const MbTrav *p;
  uint32_t lo, hi, n;
  uint8_t *flags;
  uint32_t depth;
} MbJob;

static void *mb_worker(void *arg) {
  MbJob *j = arg;
  uint32_t *stack = malloc((size_t)(3 * j->depth + 8) * 4);
  for (uint32_t i = j->lo; i < j->hi; ++i) j->flags[i] = !mb_node(j->p, i, stack);
  free(stack);
  return NULL;
}

/* many_body.zig:31-84. Serial (threads == 1): nodes in index order with the
 * real random. Threaded (CPU baseline only): the reference's record pass over
 * all nodes in parallel, then flagged nodes rerun in index order. */
static int many_body_exact(Sim *s, Force *f, double alpha) {
  if (sim_build_tree(s, 0) < 0) return D3_OUT_OF_MEMORY;
  Tree *t = &s->tree;
  if (t->root == NONE) return D3_OK;
  mb_accumulate(t, s->x, s->y, f->f0);
  MbTrav p = {t, s->x, s->y, f->f0, s->vx, s->vy, f->scalars[D3_THETA2],
              f->scalars[D3_DISTANCE_MIN2], f->scalars[D3_DISTANCE_MAX2], alpha, s};
  uint32_t *stack = malloc((size_t)(3 * t->depth + 8) * 4);
  if (!stack) return D3_OUT_OF_MEMORY;
  if (s->threads <= 1) {
    for (uint32_t i = 0; i < s->n; ++i) mb_node(&p, i, stack);
  } else {
    uint8_t *flags = calloc(s->n ? s->n : 1, 1);
    MbTrav rec = p;
    rec.s = NULL;
    int k = s->threads;
    pthread_t th[64];
    MbJob jobs[64];
    uint32_t per = (s->n + k - 1) / k;
    for (int w = 0; w < k; ++w) {
      uint32_t lo = w * per, hi = lo + per > s->n ? s->n : lo + per;
      if (lo > hi) lo = hi;
      jobs[w] = (MbJob){&rec, lo, hi, s->n, flags, t->depth};
      pthread_create(&th[w], NULL, mb_worker, &jobs[w]);
    }
    for (int w = 0; w < k; ++w) pthread_join(th[w], NULL);
    for (uint32_t i = 0; i < s->n; ++i)
      if (flags[i]) mb_node(&p, i, stack);
    free(flags);
  }
  free(stack);
  return D3_OK;
}

/* ------------------------------------------------------------------------ */
/* Exact link (link.zig), collide (collide.zig), simple.zig                  */
/* ------------------------------------------------------------------------ */

/* link.zig:8-40: Gauss-Seidel over links in user order. */
static int link_exact(Sim *s, Force *f, double alpha) {
  for (uint32_t i = 0; i < f->count; ++i)
    if (f->source[i] >= s->n || f->target[i] >= s->n) return D3_BAD_ARGUMENT;
  double iterations = f->scalars[D3_ITERATIONS];
  double *xs = s->x, *ys = s->y, *vxs = s->vx, *vys = s->vy;
  for (double k = 0; k < iterations; k += 1) {
    for (uint32_t i = 0; i < f->count; ++i) {
      uint32_t src = f->source[i], tgt = f->target[i];
      double x = xs[tgt] + vxs[tgt] - xs[src] - vxs[src];
      if (x == 0 || x != x) x = jiggle(s);
      double y = ys[tgt] + vys[tgt] - ys[src] - vys[src];
      if (y == 0 || y != y) y = jiggle(s);
      double l = sqrt(x * x + y * y);
      l = (l - f->f1[i]) / l * alpha * f->f0[i];
      x *= l;
      y *= l;
      double b = f->f2[i];
      vxs[tgt] -= x * b;
      vys[tgt] -= y * b;
      b = 1 - b;
      vxs[src] += x * b;
      vys[src] += y * b;
    }
  }
  return D3_OK;
}

/* collide.zig:117-129: max radius per cell, visitAfter. */
static void collide_prep(Tree *t, const double *radii) {
  Cell *cells = t->cells;
  for (uint32_t c = t->len; c-- > 0;) {
    Cell *quad = &cells[c];
    if (is_leaf(quad)) {
      quad->r = radii[t->perm[quad->first + quad->count - 1]];
    } else {
      quad->r = 0;
      for (int k = 0; k < 4; ++k) {
        uint32_t ch = quad->child[k];
        if (ch != NONE && cells[ch].r > quad->r) quad->r = cells[ch].r;
      }
    }
  }
}

/* collide.zig:17-102: tree on x + vx, then the ordered node loop. */
static int collide_exact(Sim *s, Force *f) {
  const double *radii = f->f0;
  double strength = f->scalars[D3_STRENGTH], iterations = f->scalars[D3_ITERATIONS];
  double *xs = s->x, *ys = s->y, *vxs = s->vx, *vys = s->vy;
  for (double k = 0; k < iterations; k += 1) {
    if (sim_build_tree(s, 1) < 0) return D3_OUT_OF_MEMORY;
    Tree *t = &s->tree;
    if (t->root == NONE) continue;
    const uint32_t *perm = t->perm;
    const Cell *cells = t->cells;
    collide_prep(t, radii);
    uint32_t *stack = malloc((size_t)(3 * t->depth + 8) * 4);
    if (!stack) return D3_OUT_OF_MEMORY;
    for (uint32_t i = 0; i < s->n; ++i) {
      double ri = radii[i], ri2 = ri * ri;
      double xi = xs[i] + vxs[i], yi = ys[i] + vys[i];
      uint32_t sp = 1;
      stack[0] = t->root;
      while (sp > 0) {
        const Cell *quad = &cells[stack[--sp]];
        double rj = quad->r;
        double r = ri + rj;
        if (is_leaf(quad)) {
          uint32_t j = perm[quad->first + quad->count - 1];
          if (j > i) {
            double x = xi - xs[j] - vxs[j];
            double y = yi - ys[j] - vys[j];
            double l = x * x + y * y;
            if (l < r * r) {
              if (x == 0) { x = jiggle(s); l += x * x; }
              if (y == 0) { y = jiggle(s); l += y * y; }
              l = sqrt(l);
              l = (r - l) / l * strength;
              x *= l;
              y *= l;
              rj *= rj;
              r = rj / (ri2 + rj);
              vxs[i] += x * r;
              vys[i] += y * r;
              r = 1 - r;
              vxs[j] -= x * r;
              vys[j] -= y * r;
            }
          }
          continue;
        }
        if (quad->x0 > xi + r || quad->x1 < xi - r || quad->y0 > yi + r || quad->y1 < yi - r) continue;
        for (int q = 3; q >= 0; --q)
          if (quad->child[q] != NONE) stack[sp++] = quad->child[q];
      }
    }
    free(stack);
  }
  return D3_OK;
}

/* simple.zig:14-31 */
static void center_force(Sim *s, Force *f) {
  uint32_t n = s->n;
  double sx = 0, sy = 0;
  for (uint32_t i = 0; i < n; ++i) {
    sx += s->x[i];
    sy += s->y[i];
  }
  double nf = (double)n, strength = f->scalars[D3_STRENGTH];
  sx = (sx / nf - f->scalars[D3_CX]) * strength;
  sy = (sy / nf - f->scalars[D3_CY]) * strength;
  for (uint32_t i = 0; i < n; ++i) {
    s->x[i] -= sx;
    s->y[i] -= sy;
  }
}

/* simple.zig:51-62: forceX (dim 0) / forceY (dim 1). */
static void axis_force(Sim *s, Force *f, double alpha, int dim) {
  double *pos = dim ? s->y : s->x, *v = dim ? s->vy : s->vx;
  for (uint32_t i = 0; i < s->n; ++i) v[i] += (f->f1[i] - pos[i]) * f->f0[i] * alpha;
}

/* simple.zig:64-86 */
static void radial_force(Sim *s, Force *f, double alpha) {
  double cx = f->scalars[D3_CX], cy = f->scalars[D3_CY];
  for (uint32_t i = 0; i < s->n; ++i) {
    double dx = s->x[i] - cx;
    if (dx == 0 || dx != dx) dx = 1e-6;
    double dy = s->y[i] - cy;
    if (dy == 0 || dy != dy) dy = 1e-6;
    double l = sqrt(dx * dx + dy * dy);
    double k = (f->f1[i] - l) * f->f0[i] * alpha / l;
    s->vx[i] += dx * k;
    s->vy[i] += dy * k;
  }
}

/* simple.zig:90-123 */
int32_t sim_integrate(uint32_t h, double velocity_decay) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  for (uint32_t i = 0; i < s->n; ++i) {
    uint8_t fixed = s->fixed[i];
    if ((fixed & 1) == 0) {
      s->vx[i] *= velocity_decay;
      s->x[i] += s->vx[i];
    } else {
      s->x[i] = s->fx[i];
      s->vx[i] = 0;
    }
    if ((fixed & 2) == 0) {
      s->vy[i] *= velocity_decay;
      s->y[i] += s->vy[i];
    } else {
      s->y[i] = s->fy[i];
      s->vy[i] = 0;
    }
  }
  return D3_OK;
}

/* ------------------------------------------------------------------------ */
/* Fast tree keys (tree.zig:287-309, 346-364)                                */
/* ------------------------------------------------------------------------ */

/* tree.zig:688-695 */
static uint64_t spread16(uint32_t v) {
  uint64_t x = v & 0xFFFF;
  x = (x | (x << 8)) & 0x00FF00FF;
  x = (x | (x << 4)) & 0x0F0F0F0F;
  x = (x | (x << 2)) & 0x33333333;
  x = (x | (x << 1)) & 0x55555555;
  return x;
}

static int tree_prepare_fast(Tree *t, const double *xs, const double *ys, uint32_t n) {
  if (tree_reserve(t, n)) return -1;
  t->extent[0] = t->extent[1] = t->extent[2] = t->extent[3] = NAN;
  t->len = 0;
  t->root = NONE;
  double b[4];
  if (!tree_box(t, xs, ys, n, b)) return 0;
  double w = b[2] - b[0], hgt = b[3] - b[1];
  double side = w > hgt ? w : hgt; /* @max of two finite values */
  if (!(side > 0)) side = 1;
  t->extent[0] = b[0]; t->extent[1] = b[1]; t->extent[2] = b[0] + side; t->extent[3] = b[1] + side;
  double scale = 65536.0 / side;
  uint32_t k = 0, rest = 0;
  for (uint32_t i = 0; i < n; ++i) {
    double x = xs[i], y = ys[i];
    if (x != x || y != y) {
      t->rest[rest++] = i;
      continue;
    }
    double fx = floor((x - b[0]) * scale), fy = floor((y - b[1]) * scale);
    uint32_t qx = (uint32_t)(fx < 65535 ? fx : 65535);
    uint32_t qy = (uint32_t)(fy < 65535 ? fy : 65535);
    t->perm[k] = i;
    t->keys[k] = spread16(qx) | (spread16(qy) << 1);
    ++k;
  }
  radix_sort(t->keys, t->perm, t->keys_tmp, t->perm_tmp, t->m, 4);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* Fast many-body: FMM (fmm.zig), serial recursion                           */
/* ------------------------------------------------------------------------ */

#define FMM_MAX_ORDER 24
#define FMM_DEFAULT_ORDER 8
#define FMM_DEFAULT_OPENING 1.4
#define FMM_MIN_N 2000
#define FMM_LEAF 32
#define FMM_LEVELS 16
#define FMM_MIN_SEP2 1e-28

typedef struct {
  Sim *s;
  FCell *cells;
  const uint32_t *perm;
  double *ux, *uy, *px, *py, *ps;
  double *vx, *vy;
  double alpha;
  uint32_t p;
  size_t stride;
  double inv_w, mac_far;
  int ring, has_dmax;
  double dmax_scaled, dmin_scaled, dmin2, dmax2;
  uint64_t seed;
  double binom[(2 * FMM_MAX_ORDER + 2) * (2 * FMM_MAX_ORDER + 2)];
  size_t bstride;
  double fact[2 * FMM_MAX_ORDER + 2];
  double dpow[2 * (FMM_MAX_ORDER + 1)];
  uint64_t stat_m2l, stat_p2p_pairs, stat_visits;
} Fmm;

/* zig @min / @max on finite operands */
static double zmin(double a, double b) { return b < a ? b : a; }
static double zmax(double a, double b) { return b > a ? b : a; }

/* fmm.zig:223-238 */
static void fmm_binomials(Fmm *c) {
  size_t nmax = 2 * c->p + 2;
  c->bstride = nmax;
  memset(c->binom, 0, sizeof c->binom);
  for (size_t n = 0; n < nmax; ++n) {
    c->binom[n * nmax] = 1;
    for (size_t k = 1; k <= n; ++k)
      c->binom[n * nmax + k] = c->binom[(n - 1) * nmax + k - 1] + (k < n ? c->binom[(n - 1) * nmax + k] : 0);
  }
  c->fact[0] = 1;
  for (size_t k = 1; k < nmax; ++k) c->fact[k] = c->fact[k - 1] * (double)k;
}

static double fbin(const Fmm *c, size_t n, size_t k) { return c->binom[n * c->bstride + k]; }

/* fmm.zig:685-717: level-order cells over the sorted keys. */
static int fmm_build_cells(Sim *s) {
  Tree *t = &s->tree;
  uint32_t m = t->m;
  uint32_t need = 2 * (m / FMM_LEAF + 1);
  if (need < 64) need = 64;
  if (s->fcap < need) {
    s->fcells = realloc(s->fcells, (size_t)need * sizeof(FCell));
    if (!s->fcells) return -1;
    s->fcap = need;
  }
  s->flen = 0;
#define APPEND(lo_, hi_, d_)                                                         \
  do {                                                                               \
    if (s->flen == s->fcap) {                                                        \
      s->fcap *= 2;                                                                  \
      s->fcells = realloc(s->fcells, (size_t)s->fcap * sizeof(FCell));               \
      if (!s->fcells) return -1;                                                     \
    }                                                                                \
    FCell nc = {0, 0, 0, (lo_), (hi_) - (lo_), 0, 0, (d_), 0};                       \
    s->fcells[s->flen++] = nc;                                                       \
  } while (0)
  APPEND(0, m, 0);
  for (uint32_t c = 0; c < s->flen; ++c) {
    uint32_t d = s->fcells[c].depth, lo = s->fcells[c].first, hi = lo + s->fcells[c].count;
    if (s->fcells[c].count <= FMM_LEAF || d >= FMM_LEVELS) continue;
    unsigned shift = 2 * (FMM_LEVELS - 1 - d);
    uint32_t k = lo, c0 = s->flen, nc = 0;
    for (uint32_t q = 0; q < 4; ++q) {
      uint32_t start = k;
      while (k < hi && ((t->keys[k] >> shift) & 3) == q) ++k;
      if (k > start) {
        APPEND(start, k, d + 1);
        ++nc;
      }
    }
    s->fcells[c].child0 = c0;
    s->fcells[c].nchild = nc;
  }
#undef APPEND
  return 0;
}

/* fmm.zig:721-754 */
static void fmm_geometry(Fmm *c, uint32_t i) {
  Sim *s = c->s;
  FCell *cell = &c->cells[i];
  double x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
  if (cell->nchild == 0) {
    for (uint32_t k = cell->first; k < cell->first + cell->count; ++k) {
      double x = c->ux[k], y = c->uy[k];
      x0 = zmin(x0, x);
      x1 = zmax(x1, x);
      y0 = zmin(y0, y);
      y1 = zmax(y1, y);
    }
  } else {
    for (uint32_t ch = cell->child0; ch < cell->child0 + cell->nchild; ++ch) {
      x0 = zmin(x0, s->bx0[ch]);
      x1 = zmax(x1, s->bx1[ch]);
      y0 = zmin(y0, s->by0[ch]);
      y1 = zmax(y1, s->by1[ch]);
    }
  }
  s->bx0[i] = x0; s->by0[i] = y0; s->bx1[i] = x1; s->by1[i] = y1;
  cell->cx = (x0 + x1) / 2;
  cell->cy = (y0 + y1) / 2;
  double dx = x1 - x0, dy = y1 - y0;
  cell->r = 0.5 * sqrt(dx * dx + dy * dy);
}

/* fmm.zig:614-623 */
static void fmm_shift_powers(Fmm *c, double dre, double dim) {
  double *pre = c->dpow, *pim = c->dpow + FMM_MAX_ORDER + 1;
  pre[0] = 1;
  pim[0] = 0;
  for (uint32_t k = 1; k <= c->p; ++k) {
    pre[k] = pre[k - 1] * dre - pim[k - 1] * dim;
    pim[k] = pre[k - 1] * dim + pim[k - 1] * dre;
  }
}

/* fmm.zig:757-806: P2M at a leaf, M2M from the children. */
static void fmm_upward(Fmm *c, uint32_t i) {
  Sim *s = c->s;
  FCell *cell = &c->cells[i];
  uint32_t q = c->p + 1;
  double *mre = s->mco + i * c->stride, *mim = mre + q;
  if (cell->nchild == 0) {
    for (uint32_t k = cell->first; k < cell->first + cell->count; ++k) {
      double sv = c->ps[k];
      if (sv != sv) continue;
      double zre = c->ux[k] - cell->cx, zim = c->uy[k] - cell->cy;
      double pre = 1, pim = 0;
      mre[0] += sv;
      for (uint32_t o = 1; o < q; ++o) {
        double nre = pre * zre - pim * zim;
        double nim = pre * zim + pim * zre;
        pre = nre;
        pim = nim;
        mre[o] += sv * pre;
        mim[o] += sv * pim;
      }
    }
  } else {
    const double *dre = c->dpow, *dim = c->dpow + FMM_MAX_ORDER + 1;
    for (uint32_t ch = cell->child0; ch < cell->child0 + cell->nchild; ++ch) {
      FCell *child = &c->cells[ch];
      fmm_shift_powers(c, child->cx - cell->cx, child->cy - cell->cy);
      const double *cre = s->mco + ch * c->stride, *cim = cre + q;
      for (uint32_t nn = 0; nn < q; ++nn) {
        double sre = 0, sim = 0;
        for (uint32_t k = 0; k <= nn; ++k) {
          double b = fbin(c, nn, k);
          double xre = cre[k] * b, xim = cim[k] * b;
          sre += xre * dre[nn - k] - xim * dim[nn - k];
          sim += xre * dim[nn - k] + xim * dre[nn - k];
        }
        mre[nn] += sre;
        mim[nn] += sim;
      }
    }
  }
}

/* fmm.zig:528-553: d3's pair formula (hashed jiggle). */
static void fmm_pair(Fmm *c, uint32_t ti, uint32_t tj, double xi, double yi, double *vx, double *vy) {
  if (tj == ti) return;
  double sj = c->ps[tj];
  double x = c->px[tj] - xi, y = c->py[tj] - yi;
  double l = x * x + y * y;
  if (l >= c->dmax2) return;
  if (x == 0 || y == 0) {
    uint32_t i = c->perm[ti], j = c->perm[tj];
    if (x == 0) { x = hash_jiggle(c->seed, i, j, 0); l += x * x; }
    if (y == 0) { y = hash_jiggle(c->seed, i, j, 1); l += y * y; }
  }
  if (l < c->dmin2) l = sqrt(c->dmin2 * l);
  double wj = sj / l;
  *vx += x * wj;
  *vy += y * wj;
}

/* fmm.zig:477-526: one target against sources [b0, b1), four pairs per
 * division on two f64 lanes (lane 0: k, k+2; lane 1: k+1, k+3). */
static void fmm_target(Fmm *c, int has_dmax, uint32_t ti, uint32_t b0, uint32_t b1) {
  uint32_t i = c->perm[ti];
  double xi = c->px[ti], yi = c->py[ti];
  double vx = c->vx[i], vy = c->vy[i];
  double ax0 = 0, ax1 = 0, ay0 = 0, ay1 = 0;
  uint32_t k = b0;
  for (; k + 4 <= b1; k += 4) {
    double sa0 = c->ps[k], sa1 = c->ps[k + 1], sb0 = c->ps[k + 2], sb1 = c->ps[k + 3];
    double xa0 = c->px[k] - xi, xa1 = c->px[k + 1] - xi;
    double ya0 = c->py[k] - yi, ya1 = c->py[k + 1] - yi;
    double xb0 = c->px[k + 2] - xi, xb1 = c->px[k + 3] - xi;
    double yb0 = c->py[k + 2] - yi, yb1 = c->py[k + 3] - yi;
    double la0 = xa0 * xa0 + ya0 * ya0, la1 = xa1 * xa1 + ya1 * ya1;
    double lb0 = xb0 * xb0 + yb0 * yb0, lb1 = xb1 * xb1 + yb1 * yb1;
    double z0 = xa0 * ya0 * xb0 * yb0, z1 = xa1 * ya1 * xb1 * yb1;
    double mn = zmin(zmin(la0, lb0), zmin(la1, lb1));
    if (z0 == 0 || z1 == 0 || !(mn >= c->dmin2) || (ti >= k && ti < k + 4)) {
      for (uint32_t q = 0; q < 4; ++q) fmm_pair(c, ti, k + q, xi, yi, &vx, &vy);
      continue;
    }
    double pa0 = la0 * la1, pa1 = la1 * la0;
    double pb0 = lb0 * lb1, pb1 = lb1 * lb0;
    double inv0 = 1 / (pa0 * pb0), inv1 = 1 / (pa1 * pb1);
    double wa0 = sa0 * la1 * pb0 * inv0, wa1 = sa1 * la0 * pb1 * inv1;
    double wb0 = sb0 * lb1 * pa0 * inv0, wb1 = sb1 * lb0 * pa1 * inv1;
    if (has_dmax) {
      if (!(la0 < c->dmax2)) wa0 = 0;
      if (!(la1 < c->dmax2)) wa1 = 0;
      if (!(lb0 < c->dmax2)) wb0 = 0;
      if (!(lb1 < c->dmax2)) wb1 = 0;
    }
    ax0 += xa0 * wa0 + xb0 * wb0;
    ax1 += xa1 * wa1 + xb1 * wb1;
    ay0 += ya0 * wa0 + yb0 * wb0;
    ay1 += ya1 * wa1 + yb1 * wb1;
  }
  for (; k < b1; ++k) fmm_pair(c, ti, k, xi, yi, &vx, &vy);
  c->vx[i] = vx + (ax0 + ax1);
  c->vy[i] = vy + (ay0 + ay1);
}

/* fmm.zig:561-610: M2L as a complex correlation on two lanes. */
static void fmm_m2l(Fmm *c, uint32_t A, uint32_t B, double dx, double dy) {
  Sim *s = c->s;
  uint32_t p = c->p, q = p + 1;
  double d2 = dx * dx + dy * dy;
  double ire = dx / d2, iim = -dy / d2;
  double tre[2 * FMM_MAX_ORDER + 1], tim[2 * FMM_MAX_ORDER + 1];
  double are = ire, aim = iim;
  tre[0] = are;
  tim[0] = aim;
  for (uint32_t m = 1; m < 2 * p + 1; ++m) {
    double nre = are * ire - aim * iim;
    double nim = are * iim + aim * ire;
    are = nre;
    aim = nim;
    tre[m] = are * c->fact[m];
    tim[m] = aim * c->fact[m];
  }
  const double *mre = s->mco + B * c->stride, *mim = mre + q;
  double *lre = s->lco + A * c->stride, *lim = lre + q;
  for (uint32_t l = 0; l < q; ++l) {
    double v0re = 0, v1re = 0, v0im = 0, v1im = 0;
    uint32_t k = 0;
    for (; k + 2 <= q; k += 2) {
      v0re += mre[k] * tre[l + k] - mim[k] * tim[l + k];
      v1re += mre[k + 1] * tre[l + k + 1] - mim[k + 1] * tim[l + k + 1];
      v0im += mre[k] * tim[l + k] + mim[k] * tre[l + k];
      v1im += mre[k + 1] * tim[l + k + 1] + mim[k + 1] * tre[l + k + 1];
    }
    double sre = v0re + v1re, sim = v0im + v1im;
    if (k < q) {
      sre += mre[k] * tre[l + k] - mim[k] * tim[l + k];
      sim += mre[k] * tim[l + k] + mim[k] * tre[l + k];
    }
    lre[l] += sre;
    lim[l] += sim;
  }
}

/* fmm.zig:400-453: dual-tree traversal, serial recursion from (root, root). */
static void fmm_interact(Fmm *c, uint32_t A, uint32_t B) {
  c->stat_visits++;
  FCell *ca = &c->cells[A];
  if (A == B) {
    if (ca->nchild == 0) {
      c->stat_p2p_pairs += (uint64_t)ca->count * ca->count;
      for (uint32_t ti = ca->first; ti < ca->first + ca->count; ++ti)
        fmm_target(c, c->has_dmax, ti, ca->first, ca->first + ca->count);
    } else {
      uint32_t c0 = ca->child0, k = ca->nchild;
      for (uint32_t i = 0; i < k; ++i)
        for (uint32_t j = 0; j < k; ++j) fmm_interact(c, c0 + i, c0 + j);
    }
    return;
  }
  FCell *cb = &c->cells[B];
  double ra = ca->r, rb = cb->r;
  double dx = ca->cx - cb->cx, dy = ca->cy - cb->cy;
  double d2 = dx * dx + dy * dy;
  double rmax = zmax(ra, rb), rmin = zmin(ra, rb);
  double thr = c->mac_far * rmax + rmin;
  if (d2 > FMM_MIN_SEP2 && d2 >= thr * thr) {
    int separated = 1;
    if (c->ring) {
      double gap = sqrt(d2) - ra - rb;
      if (gap >= c->dmax_scaled) return;
      if (gap + 2 * (ra + rb) > c->dmax_scaled || gap < c->dmin_scaled) separated = 0;
    }
    if (separated) {
      c->stat_m2l++;
      fmm_m2l(c, A, B, dx, dy);
      return;
    }
  }
  int la = ca->nchild == 0, lb = cb->nchild == 0;
  if (la && lb) {
    c->stat_p2p_pairs += (uint64_t)ca->count * cb->count;
    for (uint32_t ti = ca->first; ti < ca->first + ca->count; ++ti)
      fmm_target(c, c->has_dmax, ti, cb->first, cb->first + cb->count);
  } else if (la || (!lb && rb > ra)) {
    uint32_t c0 = cb->child0, k = cb->nchild;
    for (uint32_t j = 0; j < k; ++j) fmm_interact(c, A, c0 + j);
  } else {
    uint32_t c0 = ca->child0, k = ca->nchild;
    for (uint32_t i = 0; i < k; ++i) fmm_interact(c, c0 + i, B);
  }
}

/* fmm.zig:823-849 */
static void fmm_l2l(Fmm *c, uint32_t i, uint32_t ch) {
  Sim *s = c->s;
  uint32_t q = c->p + 1;
  FCell *cell = &c->cells[i], *child = &c->cells[ch];
  const double *lre = s->lco + i * c->stride, *lim = lre + q;
  const double *dre = c->dpow, *dim = c->dpow + FMM_MAX_ORDER + 1;
  fmm_shift_powers(c, child->cx - cell->cx, child->cy - cell->cy);
  double *cre = s->lco + ch * c->stride, *cim = cre + q;
  for (uint32_t mm = 0; mm < q; ++mm) {
    double sre = 0, sim = 0;
    for (uint32_t l = mm; l < q; ++l) {
      double b = fbin(c, l, mm);
      double xre = lre[l] * b, xim = lim[l] * b;
      sre += xre * dre[l - mm] - xim * dim[l - mm];
      sim += xre * dim[l - mm] + xim * dre[l - mm];
    }
    cre[mm] += sre;
    cim[mm] += sim;
  }
}

/* fmm.zig:853-886 (top = false everywhere in the serial order). */
static void fmm_downward(Fmm *c, uint32_t i) {
  Sim *s = c->s;
  FCell *cell = &c->cells[i];
  uint32_t p = c->p, q = p + 1;
  const double *lre = s->lco + i * c->stride, *lim = lre + q;
  if (cell->nchild == 0) {
    for (uint32_t k = cell->first; k < cell->first + cell->count; ++k) {
      uint32_t j = c->perm[k];
      double wre = c->ux[k] - cell->cx, wim = c->uy[k] - cell->cy;
      double are = lre[p], aim = lim[p];
      for (uint32_t l = p; l > 0;) {
        --l;
        double nre = are * wre - aim * wim + lre[l];
        double nim = are * wim + aim * wre + lim[l];
        are = nre;
        aim = nim;
      }
      c->vx[j] -= are * c->inv_w;
      c->vy[j] += aim * c->inv_w;
    }
  } else {
    for (uint32_t ch = cell->child0; ch < cell->child0 + cell->nchild; ++ch) fmm_l2l(c, i, ch);
  }
}

static uint64_t fmm_last_m2l, fmm_last_p2p_pairs, fmm_last_visits;

/* fmm.zig:247-354. Returns 1 when handled, 0 when the exact kernel must run
 * instead (non-finite extent), < 0 on allocation failure. */
static int fmm_run(Sim *s, Force *f, double alpha) {
  Tree *t = &s->tree;
  int r = tree_prepare_fast(t, s->x, s->y, s->n);
  if (r < 0) return -1;
  if (r == 0) return 1;
  double w = t->extent[2] - t->extent[0];
  if (!(w > 0 && w < INFINITY)) return 0;
  static Fmm c; /* large tables; the oracle is single-threaded */
  memset(&c, 0, sizeof c);
  c.s = s;
  c.p = FMM_DEFAULT_ORDER;
  double po = f->scalars[D3_ORDER];
  if (po >= 1 && po <= (double)FMM_MAX_ORDER) c.p = (uint32_t)po;
  double kappa = f->scalars[D3_OPENING];
  if (!(kappa > 1)) kappa = FMM_DEFAULT_OPENING;
  fmm_binomials(&c);
  if (fmm_build_cells(s)) return -1;
  uint32_t nc = s->flen;
  c.stride = 2 * (c.p + 1);
  size_t need = (size_t)nc * c.stride;
  if (s->coef_cap < need) {
    free(s->mco);
    free(s->lco);
    s->mco = malloc(need * 8);
    s->lco = malloc(need * 8);
    s->bx0 = realloc(s->bx0, (size_t)nc * 8);
    s->by0 = realloc(s->by0, (size_t)nc * 8);
    s->bx1 = realloc(s->bx1, (size_t)nc * 8);
    s->by1 = realloc(s->by1, (size_t)nc * 8);
    if (!s->mco || !s->lco || !s->bx0 || !s->by0 || !s->bx1 || !s->by1) return -1;
    s->coef_cap = need;
  }
  double dmax_scaled = INFINITY, dmax2 = f->scalars[D3_DISTANCE_MAX2];
  if (dmax2 < INFINITY) dmax_scaled = sqrt(dmax2) / w;
  double dmin2 = f->scalars[D3_DISTANCE_MIN2];
  double dmin_scaled = dmin2 > 0 ? sqrt(dmin2) / w : 0;
  if (s->pts_cap < t->m) {
    s->ux = realloc(s->ux, (size_t)t->m * 8);
    s->uy = realloc(s->uy, (size_t)t->m * 8);
    s->fpx = realloc(s->fpx, (size_t)t->m * 8);
    s->fpy = realloc(s->fpy, (size_t)t->m * 8);
    s->fps = realloc(s->fps, (size_t)t->m * 8);
    if (!s->ux || !s->uy || !s->fpx || !s->fpy || !s->fps) return -1;
    s->pts_cap = t->m;
  }
  c.cells = s->fcells;
  c.perm = t->perm;
  c.ux = s->ux; c.uy = s->uy; c.px = s->fpx; c.py = s->fpy; c.ps = s->fps;
  c.vx = s->vx; c.vy = s->vy;
  c.alpha = alpha;
  c.inv_w = 1 / w;
  c.mac_far = 2 * kappa - 1;
  c.ring = dmin_scaled > 0 || dmax_scaled < INFINITY;
  c.has_dmax = dmax_scaled < INFINITY;
  c.dmax_scaled = dmax_scaled;
  c.dmin_scaled = dmin_scaled;
  c.dmin2 = dmin2;
  c.dmax2 = dmax2;
  c.seed = seed_from(f->scalars[D3_SEED]);
  double ox = (t->extent[0] + t->extent[2]) / 2, oy = (t->extent[1] + t->extent[3]) / 2;
  memset(s->mco, 0, need * 8);
  memset(s->lco, 0, need * 8);
  /* fmm.zig:668-682 gather */
  for (uint32_t j = 0; j < t->m; ++j) {
    uint32_t i = t->perm[j];
    double x = s->x[i], y = s->y[i];
    c.px[j] = x;
    c.py[j] = y;
    double st = f->f0[i] * alpha;
    c.ps[j] = st != st ? 0 : st;
    c.ux[j] = (x - ox) * c.inv_w;
    c.uy[j] = (y - oy) * c.inv_w;
  }
  /* upward: children before parents (cells are in level order) */
  for (uint32_t i = nc; i-- > 0;) {
    fmm_geometry(&c, i);
    fmm_upward(&c, i);
  }
  /* fmm.zig:629-642 scale M_k by 1/k! */
  for (uint32_t i = 0; i < nc; ++i) {
    uint32_t q = c.p + 1;
    double *mre = s->mco + i * c.stride, *mim = mre + q;
    for (uint32_t o = 2; o < q; ++o) {
      double inv = 1 / c.fact[o];
      mre[o] *= inv;
      mim[o] *= inv;
    }
  }
  fmm_interact(&c, 0, 0);
  /* fmm.zig:645-657 unscale L_l by (-1)^l / l! */
  for (uint32_t i = 0; i < nc; ++i) {
    uint32_t q = c.p + 1;
    double *lre = s->lco + i * c.stride, *lim = lre + q;
    double sign = 1;
    for (uint32_t o = 0; o < q; ++o) {
      double inv = sign / c.fact[o];
      lre[o] *= inv;
      lim[o] *= inv;
      sign = -sign;
    }
  }
  for (uint32_t i = 0; i < nc; ++i) fmm_downward(&c, i);
  fmm_last_m2l = c.stat_m2l;
  fmm_last_p2p_pairs = c.stat_p2p_pairs;
  fmm_last_visits = c.stat_visits;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* Fast collide (grid.zig) and fast link (link_fast.zig)                     */
/* ------------------------------------------------------------------------ */

#define NO_CELL 0xffffffffu

/* grid.zig:198-286 */
static int grid_run(Sim *s, Force *f) {
  uint32_t n = s->n;
  if (s->g_cap < n) {
    s->g_items = realloc(s->g_items, (size_t)s->cap * 4);
    s->g_items_tmp = realloc(s->g_items_tmp, (size_t)s->cap * 4);
    s->g_cell_of = realloc(s->g_cell_of, (size_t)s->cap * 4);
    s->g_keys = realloc(s->g_keys, (size_t)s->cap * 8);
    s->g_keys_tmp = realloc(s->g_keys_tmp, (size_t)s->cap * 8);
    if (!s->g_items || !s->g_items_tmp || !s->g_cell_of || !s->g_keys || !s->g_keys_tmp) return -1;
    s->g_cap = s->cap;
  }
  const double *radii = f->f0;
  double strength = f->scalars[D3_STRENGTH];
  uint64_t seed = seed_from(f->scalars[D3_SEED]);
  double iterations = f->scalars[D3_ITERATIONS];
  for (double it = 0; it < iterations; it += 1) {
    double x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY, rmax = 0;
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; ++i) {
      double x = s->x[i] + s->vx[i], y = s->y[i] + s->vy[i];
      s->px[i] = x;
      s->py[i] = y;
      if (x != x || y != y) continue;
      ++m;
      if (x < x0) x0 = x;
      if (x > x1) x1 = x;
      if (y < y0) y0 = y;
      if (y > y1) y1 = y;
      double rad = radii[i];
      if (rad > rmax) rmax = rad;
    }
    if (m < 2 || !(rmax > 0)) continue;
    double h = 2 * rmax;
    uint32_t gx = (uint32_t)(floor((x1 - x0) / h) + 1);
    uint32_t gy = (uint32_t)(floor((y1 - y0) / h) + 1);
    while ((uint64_t)gx * gy > 4 * (uint64_t)n + 16) {
      h *= 2;
      gx = (uint32_t)(floor((x1 - x0) / h) + 1);
      gy = (uint32_t)(floor((y1 - y0) / h) + 1);
    }
    uint32_t cells = gx * gy;
    if (s->g_start_cap < cells + 1) {
      s->g_start = realloc(s->g_start, (size_t)(cells + 1) * 4);
      if (!s->g_start) return -1;
      s->g_start_cap = cells + 1;
    }
    double inv_h = 1 / h;
    for (uint32_t k = 0; k < n; ++k) {
      uint32_t i = n - 1 - k;
      uint32_t cell = cells;
      if (s->px[i] == s->px[i] && s->py[i] == s->py[i]) {
        uint32_t cx = (uint32_t)floor((s->px[i] - x0) * inv_h);
        uint32_t cy = (uint32_t)floor((s->py[i] - y0) * inv_h);
        cell = cy * gx + cx;
      }
      s->g_cell_of[i] = cell == cells ? NO_CELL : cell;
      s->g_keys[k] = cell;
      s->g_items[k] = i;
    }
    uint32_t bytes = cells < (1u << 8) ? 1 : cells < (1u << 16) ? 2 : cells < (1u << 24) ? 3 : 4;
    radix_sort(s->g_keys, s->g_items, s->g_keys_tmp, s->g_items_tmp, n, bytes);
    uint32_t *start = s->g_start;
    for (uint32_t k = 0; k < n; ++k) {
      uint32_t lo = k == 0 ? 0 : (uint32_t)(s->g_keys[k - 1] + 1);
      uint32_t hi = (uint32_t)(s->g_keys[k] < cells ? s->g_keys[k] : cells);
      if (k == 0 || s->g_keys[k] != s->g_keys[k - 1])
        for (uint32_t cell = lo; cell <= hi; ++cell) start[cell] = k;
    }
    uint32_t cell = s->g_keys[n - 1] == cells ? cells + 1 : (uint32_t)(s->g_keys[n - 1] + 1);
    for (; cell <= cells; ++cell) start[cell] = m;
    start[cells] = m;
    for (uint32_t i = 0; i < n; ++i) {
      uint32_t ci = s->g_cell_of[i];
      if (ci == NO_CELL) continue;
      double ri = radii[i], ri2 = ri * ri;
      double xi = s->px[i], yi = s->py[i];
      double vx = s->vx[i], vy = s->vy[i];
      uint32_t cxi = ci % gx, cyi = ci / gx;
      uint32_t xa = cxi > 0 ? cxi - 1 : 0, xb = cxi + 1 < gx - 1 ? cxi + 1 : gx - 1;
      uint32_t ya = cyi > 0 ? cyi - 1 : 0, yb = cyi + 1 < gy - 1 ? cyi + 1 : gy - 1;
      for (uint32_t cy = ya; cy <= yb; ++cy) {
        for (uint32_t cx = xa; cx <= xb; ++cx) {
          uint32_t cc = cy * gx + cx;
          for (uint32_t kk = start[cc]; kk < start[cc + 1]; ++kk) {
            uint32_t j = s->g_items[kk];
            if (j == i) continue;
            double rj = radii[j];
            double rr = ri + rj;
            double x = xi - s->px[j], y = yi - s->py[j];
            double l = x * x + y * y;
            if (l < rr * rr) {
              if (x == 0 || y == 0) {
                uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
                double sign = i == lo ? 1 : -1;
                if (x == 0) { x = sign * hash_jiggle(seed, lo, hi, 0); l += x * x; }
                if (y == 0) { y = sign * hash_jiggle(seed, lo, hi, 1); l += y * y; }
              }
              l = sqrt(l);
              l = (rr - l) / l * strength;
              x *= l;
              y *= l;
              rr = rj * rj / (ri2 + rj * rj);
              vx += x * rr;
              vy += y * rr;
            }
          }
        }
      }
      s->vx[i] = vx;
      s->vy[i] = vy;
    }
  }
  return 0;
}

#define TARGET_BIT 0x80000000u

/* link_fast.zig:105-130 */
static int link_build_csr(Force *f, uint32_t n) {
  uint32_t m = f->count;
  f->csr_ptr = realloc(f->csr_ptr, (size_t)(n + 1) * 4);
  f->csr_adj = realloc(f->csr_adj, (size_t)(m > 0 ? 2 * m : 1) * 4);
  if (!f->csr_ptr || !f->csr_adj) return -1;
  uint32_t *row = f->csr_ptr;
  memset(row, 0, (size_t)(n + 1) * 4);
  for (uint32_t e = 0; e < m; ++e) {
    row[f->source[e] + 1]++;
    row[f->target[e] + 1]++;
  }
  for (uint32_t i = 1; i <= n; ++i) row[i] += row[i - 1];
  for (uint32_t e = 0; e < m; ++e) {
    f->csr_adj[row[f->source[e] + 1] - 1] = e;
    row[f->source[e] + 1]--;
    f->csr_adj[row[f->target[e] + 1] - 1] = e | TARGET_BIT;
    row[f->target[e] + 1]--;
  }
  for (uint32_t i = 0; i < n; ++i) row[i] = row[i + 1];
  row[n] = 2 * m;
  return 0;
}

/* link_fast.zig:22-99 */
static int link_fast(Sim *s, Force *f, double alpha) {
  uint32_t n = s->n, m = f->count;
  for (uint32_t e = 0; e < m; ++e)
    if (f->source[e] >= n || f->target[e] >= n) return D3_BAD_ARGUMENT;
  if (f->csr_n != n) {
    if (link_build_csr(f, n)) return D3_OUT_OF_MEMORY;
    f->csr_n = n;
  }
  uint64_t seed = seed_from(f->scalars[D3_SEED]);
  double iterations = f->scalars[D3_ITERATIONS];
  for (double it = 0; it < iterations; it += 1) {
    for (uint32_t i = 0; i < n; ++i) {
      s->px[i] = s->x[i] + s->vx[i];
      s->py[i] = s->y[i] + s->vy[i];
    }
    for (uint32_t i = 0; i < n; ++i) {
      double vx = s->vx[i], vy = s->vy[i];
      double pxi = s->px[i], pyi = s->py[i];
      for (uint32_t a = f->csr_ptr[i]; a < f->csr_ptr[i + 1]; ++a) {
        uint32_t entry = f->csr_adj[a];
        uint32_t e = entry & ~TARGET_BIT;
        int is_target = (entry & TARGET_BIT) != 0;
        uint32_t j = is_target ? f->source[e] : f->target[e];
        double x = is_target ? pxi - s->px[j] : s->px[j] - pxi;
        double y = is_target ? pyi - s->py[j] : s->py[j] - pyi;
        if (x == 0 || x != x) x = hash_jiggle(seed, e, 0, 0);
        if (y == 0 || y != y) y = hash_jiggle(seed, e, 0, 1);
        double l = sqrt(x * x + y * y);
        l = (l - f->f1[e]) / l * alpha * f->f0[e];
        x *= l;
        y *= l;
        double b = f->f2[e];
        if (is_target) {
          vx -= x * b;
          vy -= y * b;
        } else {
          vx += x * (1 - b);
          vy += y * (1 - b);
        }
      }
      s->vx[i] = vx;
      s->vy[i] = vy;
    }
  }
  return D3_OK;
}

/* ------------------------------------------------------------------------ */
/* force_run dispatch (root.zig:211-248)                                     */
/* ------------------------------------------------------------------------ */

static int fast_mode(const Sim *s, const Force *f) {
  return f->scalars[D3_PRECISION] == 1 && s->n >= FMM_MIN_N;
}

int32_t force_run(uint32_t h, uint32_t fh, double alpha) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  Force *f = get_force(s, fh);
  if (!f) return D3_BAD_HANDLE;
  if (node_sized(f) && f->count < s->n) return D3_BAD_ARGUMENT;
  /* LCG mode: the facade's per-run SEED draw (src/core.js:218-222). */
  if (s->rand_mode == 0 && f->scalars[D3_PRECISION] == 1 &&
      (f->kind == D3_MANY_BODY || f->kind == D3_LINK || f->kind == D3_COLLIDE))
    f->scalars[D3_SEED] = sim_random(s);
  switch (f->kind) {
    case D3_CENTER: center_force(s, f); return D3_OK;
    case D3_X: axis_force(s, f, alpha, 0); return D3_OK;
    case D3_Y: axis_force(s, f, alpha, 1); return D3_OK;
    case D3_RADIAL: radial_force(s, f, alpha); return D3_OK;
    case D3_LINK: return fast_mode(s, f) ? link_fast(s, f, alpha) : link_exact(s, f, alpha);
    case D3_MANY_BODY:
      if (fast_mode(s, f)) {
        int r = fmm_run(s, f, alpha);
        if (r < 0) return D3_OUT_OF_MEMORY;
        if (r == 1) return D3_OK;
      }
      return many_body_exact(s, f, alpha);
    case D3_COLLIDE:
      if (fast_mode(s, f)) return grid_run(s, f) ? D3_OUT_OF_MEMORY : D3_OK;
      return collide_exact(s, f);
    default: return D3_BAD_ARGUMENT;
  }
}

/* ------------------------------------------------------------------------ */
/* Extensions                                                                */
/* ------------------------------------------------------------------------ */

int32_t sim_set_random(uint32_t h, d3_random_fn fn, void *ctx) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  s->rand_mode = fn ? 1 : 0;
  s->rand_fn = fn;
  s->rand_ctx = ctx;
  return D3_OK;
}

int32_t sim_set_lcg(uint32_t h, uint32_t state) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  s->rand_mode = 0;
  s->rand_fn = NULL;
  s->lcg = state;
  return D3_OK;
}

uint32_t sim_get_lcg(uint32_t h) {
  Sim *s = get_sim(h);
  return s ? s->lcg : 0;
}

int32_t sim_set_sync(uint32_t h, uint32_t mode) {
  (void)mode;
  return get_sim(h) ? D3_OK : D3_BAD_HANDLE;
}
/* The node state is the oracle's own memory: an upload only derives the fixed
 * bits when asked to (src/core.js:130, NaN = not set). */
int32_t sim_sync_in(uint32_t h) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (s->fixed_from_f)
    for (uint32_t i = 0; i < s->n; ++i)
      s->fixed[i] = (uint8_t)((s->fx[i] == s->fx[i] ? 1 : 0) | (s->fy[i] == s->fy[i] ? 2 : 0));
  return D3_OK;
}

int32_t sim_set_fixed_source(uint32_t h, uint32_t from_f) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (from_f > 1) return D3_BAD_ARGUMENT;
  s->fixed_from_f = from_f != 0;
  return D3_OK;
}
int32_t sim_sync_out(uint32_t h) { return get_sim(h) ? D3_OK : D3_BAD_HANDLE; }

int32_t sim_tick(uint32_t h, uint32_t ticks, double *alpha, double alpha_target, double alpha_decay,
                 double velocity_decay, const uint32_t *order, uint32_t n_order) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  for (uint32_t k = 0; k < ticks; ++k) {
    *alpha += (alpha_target - *alpha) * alpha_decay;
    for (uint32_t i = 0; i < n_order; ++i) {
      int32_t r = force_run(h, order[i], *alpha);
      if (r < 0) return r;
    }
    sim_integrate(h, velocity_decay);
  }
  return D3_OK;
}

int32_t sim_tick_sync(uint32_t h, uint32_t ticks, double *alpha, double alpha_target,
                      double alpha_decay, double velocity_decay, const uint32_t *order,
                      uint32_t n_order) {
  int32_t r = sim_sync_in(h);
  if (r < 0) return r;
  return sim_tick(h, ticks, alpha, alpha_target, alpha_decay, velocity_decay, order, n_order);
}

double sim_last_tick_ms(uint32_t h) {
  (void)h;
  return 0;
}

double sim_stat(uint32_t h, uint32_t which) {
  (void)h;
  (void)which;
  return 0;
}

/* src/simulation.js:157-178 (find): radius *= radius (a missing radius is
 * Infinity), then the serial scan keeping each strictly closer node. */
int32_t sim_find(uint32_t h, double x, double y, double radius, uint32_t *index) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  if (!index) return D3_BAD_ARGUMENT;
  double r2 = radius * radius;
  uint32_t closest = NONE;
  for (uint32_t i = 0; i < s->n; ++i) {
    double dx = x - s->x[i], dy = y - s->y[i], d2 = dx * dx + dy * dy;
    if (d2 < r2) closest = i, r2 = d2;
  }
  *index = closest;
  return D3_OK;
}

/* The engine's device-wait self test has no CPU meaning: report a bad
 * argument. */
int32_t sim_selftest_wait(uint32_t h, uint32_t budget_us) {
  (void)h;
  (void)budget_us;
  return D3_BAD_ARGUMENT;
}

int32_t sim_set_profile(uint32_t h, uint32_t on) {
  (void)on;
  return get_sim(h) ? D3_OK : D3_BAD_HANDLE;
}

/* Oracle-only: worker threads for the tree builds (key pass, sort, emission
 * jobs) and the exact many-body record pass, the CPU baseline's stand-in for
 * the reference's thread pool. The results do not change. */
int32_t oracle_set_threads(uint32_t h, uint32_t k) {
  Sim *s = get_sim(h);
  if (!s) return D3_BAD_HANDLE;
  s->threads = k < 1 ? 1 : k > 64 ? 64 : (int)k;
  return D3_OK;
}

/* Oracle-only: the exact many-body work counters since the last reset
 * (which 0 visits, 1 accepted approximations, 2 leaf point interactions;
 * which 3 resets them and returns 0). */
uint64_t oracle_mb_stat(uint32_t which) {
  if (which == 3) {
    mb_visits = mb_accepts = mb_points = 0;
    return 0;
  }
  return which == 0 ? mb_visits : which == 1 ? mb_accepts : mb_points;
}

/* Oracle-only: interaction counters of the last FMM run (fmm.zig:59). */
uint64_t oracle_fmm_stat(uint32_t which) {
  return which == 0 ? fmm_last_m2l : which == 1 ? fmm_last_p2p_pairs : fmm_last_visits;
}
