/* Oracle twins of the library's synthetic graph generators -- test
 * infrastructure.
 *
 * The reference's CPU arm of bench.py must build the RMAT-24 and 4096^2 grid
 * workloads without loading libb200sssp.so, and tests/test_graph_gen_twin.py
 * pins these functions byte for byte to b2_gen_rmat / b2_gen_grid.  The
 * generators are defined by their random streams, not by their code: every
 * arc and weight is a pure function of (seed, stream, index) through the
 * splitmix64 finalizer (Steele, Lea and Flood), so an independent
 * implementation reproduces the same graph.
 *
 *   RMAT: edge i of edge_factor * 2^scale draws one 64-bit word per two
 *         levels (stream 3, index 16 i + level / 2; high half first), picks
 *         the (a, b, c, d) quadrant against 32-bit thresholds floor(p 2^32),
 *         scrambles both ids by x -> (x A + B) mod 2^scale (A odd), drops
 *         self-loops, symmetrises and deduplicates; the weight of the
 *         undirected pair {x < y} is wmin + hi32(rnd(stream 4, x << 32 | y))
 *         scaled to the range.
 *   Grid: 4-neighbour bidirectional lattice, plus round(frac * lattice arcs)
 *         random pairs (stream 5, retried past self-pairs) in both directions;
 *         arc (u, v) weighs ceil(exp(mu + sigma z)) with z from Box-Muller on
 *         streams 6 and 7 keyed by u << 32 | v.
 * Output: OUTGOING CSR, columns sorted and unique in each row.
 *
 * Build structure here (degree count, atomic scatter, per-row sort) is this
 * file's own; threads only change the order of work, never the result. */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t sm64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static uint64_t draw(uint64_t seed, uint64_t stream, uint64_t i) {
  return sm64(sm64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + i);
}
static uint32_t scale32(uint32_t r, uint64_t range) { return (uint32_t)(((uint64_t)r * range) >> 32); }

/* ---- a tiny fork/join over index ranges ---------------------------------- */
typedef void (*range_fn)(void* ctx, int64_t lo, int64_t hi);
typedef struct {
  range_fn fn;
  void* ctx;
  int64_t lo, hi;
} job;
static void* job_main(void* p) {
  job* j = (job*)p;
  j->fn(j->ctx, j->lo, j->hi);
  return NULL;
}
static void run_ranges(int threads, int64_t n, range_fn fn, void* ctx) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  if (threads == 1 || n < 65536) {
    fn(ctx, 0, n);
    return;
  }
  pthread_t th[256];
  job jobs[256];
  const int64_t step = (n + threads - 1) / threads;
  int used = 0;
  for (int t = 0; t < threads; ++t) {
    const int64_t lo = t * step, hi = lo + step < n ? lo + step : n;
    if (lo >= hi) break;
    jobs[t].fn = fn;
    jobs[t].ctx = ctx;
    jobs[t].lo = lo;
    jobs[t].hi = hi;
    pthread_create(&th[t], NULL, job_main, &jobs[t]);
    ++used;
  }
  for (int t = 0; t < used; ++t) pthread_join(th[t], NULL);
}

static int cmp_u32(const void* a, const void* b) {
  const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return (x > y) - (x < y);
}

/* ---- symmetric arc sets: count, scatter, sort, compact --------------------
 * An arc source produces undirected pairs by index; both directions go in. */
typedef int (*pair_fn)(const void* gen, int64_t i, uint32_t* u, uint32_t* v);  /* 0: no pair */

typedef struct {
  const void* gen;
  pair_fn pair;
  uint32_t* deg;       /* atomic counters, then cursors */
  int64_t* start;
  uint32_t* slots;     /* scattered neighbour ids */
  int64_t* kept;
} build_ctx;

static void count_range(void* p, int64_t lo, int64_t hi) {
  build_ctx* c = (build_ctx*)p;
  for (int64_t i = lo; i < hi; ++i) {
    uint32_t u, v;
    if (!c->pair(c->gen, i, &u, &v)) continue;
    __atomic_fetch_add(&c->deg[u], 1u, __ATOMIC_RELAXED);
    __atomic_fetch_add(&c->deg[v], 1u, __ATOMIC_RELAXED);
  }
}
static void scatter_range(void* p, int64_t lo, int64_t hi) {
  build_ctx* c = (build_ctx*)p;
  for (int64_t i = lo; i < hi; ++i) {
    uint32_t u, v;
    if (!c->pair(c->gen, i, &u, &v)) continue;
    const uint32_t pu = __atomic_fetch_add(&c->deg[u], 1u, __ATOMIC_RELAXED);
    const uint32_t pv = __atomic_fetch_add(&c->deg[v], 1u, __ATOMIC_RELAXED);
    c->slots[c->start[u] + pu] = v;
    c->slots[c->start[v] + pv] = u;
  }
}
static void sort_range(void* p, int64_t lo, int64_t hi) {
  build_ctx* c = (build_ctx*)p;
  for (int64_t v = lo; v < hi; ++v) {
    uint32_t* a = c->slots + c->start[v];
    const int64_t len = c->start[v + 1] - c->start[v];
    if (len > 1) qsort(a, (size_t)len, 4, cmp_u32);
    int64_t k = 0;
    for (int64_t j = 0; j < len; ++j)
      if (k == 0 || a[j] != a[k - 1]) a[k++] = a[j];
    c->kept[v] = k;
  }
}

typedef struct {
  build_ctx* b;
  int64_t* rowptr;
  int32_t* colind;
} compact_ctx;
static void compact_range(void* p, int64_t lo, int64_t hi) {
  compact_ctx* c = (compact_ctx*)p;
  for (int64_t v = lo; v < hi; ++v)
    for (int64_t j = 0; j < c->b->kept[v]; ++j)
      c->colind[c->rowptr[v] + j] = (int32_t)c->b->slots[c->b->start[v] + j];
}

/* Builds rowptr / colind (malloc'd) of the symmetric graph on n vertices. */
static int build_symmetric(int64_t n, int64_t npairs, const void* gen, pair_fn pair, int threads,
                           int64_t** rowptr_out, int32_t** colind_out, int64_t* m_out) {
  build_ctx c;
  memset(&c, 0, sizeof(c));
  c.gen = gen;
  c.pair = pair;
  c.deg = (uint32_t*)calloc((size_t)n, 4);
  c.start = (int64_t*)malloc((size_t)(n + 1) * 8);
  c.kept = (int64_t*)malloc((size_t)n * 8);
  if (!c.deg || !c.start || !c.kept) goto fail;
  run_ranges(threads, npairs, count_range, &c);
  c.start[0] = 0;
  for (int64_t v = 0; v < n; ++v) {
    c.start[v + 1] = c.start[v] + c.deg[v];
    c.deg[v] = 0;
  }
  c.slots = (uint32_t*)malloc((size_t)(c.start[n] > 0 ? c.start[n] : 1) * 4);
  if (!c.slots) goto fail;
  run_ranges(threads, npairs, scatter_range, &c);
  run_ranges(threads, n, sort_range, &c);
  {
    int64_t* rp = (int64_t*)malloc((size_t)(n + 1) * 8);
    if (!rp) goto fail;
    rp[0] = 0;
    for (int64_t v = 0; v < n; ++v) rp[v + 1] = rp[v] + c.kept[v];
    int32_t* ci = (int32_t*)malloc((size_t)(rp[n] > 0 ? rp[n] : 1) * 4);
    if (!ci) { free(rp); goto fail; }
    compact_ctx cc = {&c, rp, ci};
    run_ranges(threads, n, compact_range, &cc);
    *rowptr_out = rp;
    *colind_out = ci;
    *m_out = rp[n];
  }
  free(c.deg);
  free(c.start);
  free(c.kept);
  free(c.slots);
  return 0;
fail:
  free(c.deg);
  free(c.start);
  free(c.kept);
  free(c.slots);
  return -1;
}

/* ---- RMAT ----------------------------------------------------------------- */
typedef struct {
  uint64_t seed, ta, tab, tabc, mask, mul, add;
  int scale;
} rmat_gen;

static int rmat_pair(const void* p, int64_t i, uint32_t* pu, uint32_t* pv) {
  const rmat_gen* g = (const rmat_gen*)p;
  uint64_t u = 0, v = 0;
  for (int level = 0; level < g->scale; ++level) {
    const uint64_t word = draw(g->seed, 3, (uint64_t)i * 16 + (uint64_t)(level >> 1));
    const uint64_t r = (level & 1) ? (word & 0xffffffffull) : (word >> 32);
    const uint64_t right = r >= g->tab;                                   /* quadrants c, d: u bit */
    const uint64_t down = (r >= g->ta && r < g->tab) || r >= g->tabc;    /* quadrants b, d: v bit */
    u = (u << 1) | right;
    v = (v << 1) | down;
  }
  u = (u * g->mul + g->add) & g->mask;
  v = (v * g->mul + g->add) & g->mask;
  if (u == v) return 0;
  *pu = (uint32_t)u;
  *pv = (uint32_t)v;
  return 1;
}

typedef struct {
  const int64_t* rp;
  const int32_t* ci;
  uint32_t* w;
  uint64_t seed, range;
  uint32_t wmin;
} rmat_w_ctx;
static void rmat_weights(void* p, int64_t lo, int64_t hi) {
  rmat_w_ctx* c = (rmat_w_ctx*)p;
  for (int64_t u = lo; u < hi; ++u)
    for (int64_t e = c->rp[u]; e < c->rp[u + 1]; ++e) {
      const uint64_t v = (uint64_t)(uint32_t)c->ci[e];
      const uint64_t lo_id = (uint64_t)u < v ? (uint64_t)u : v;
      const uint64_t hi_id = (uint64_t)u < v ? v : (uint64_t)u;
      c->w[e] = c->wmin + scale32((uint32_t)(draw(c->seed, 4, (lo_id << 32) | hi_id) >> 32), c->range);
    }
}

int orc_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint32_t wmin, uint32_t wmax,
                 uint64_t seed, int threads, int64_t* n_out, int64_t* m_out, int64_t** rowptr, int32_t** colind,
                 uint32_t** weights) {
  if (scale < 2 || scale > 30 || edge_factor < 1 || wmax < wmin) return -1;
  rmat_gen g;
  g.seed = seed;
  g.scale = scale;
  g.ta = (uint64_t)floor(a * 4294967296.0);
  g.tab = (uint64_t)floor((a + b) * 4294967296.0);
  g.tabc = (uint64_t)floor((a + b + c) * 4294967296.0);
  const int64_t n = (int64_t)1 << scale;
  g.mask = (uint64_t)n - 1;
  g.mul = (sm64(seed ^ 0x5bd1e995ull) | 1ull) & g.mask;
  if (g.mul == 0) g.mul = 1;
  g.add = sm64(seed ^ 0x27d4eb2full) & g.mask;
  int64_t m = 0;
  if (build_symmetric(n, (int64_t)edge_factor * n, &g, rmat_pair, threads, rowptr, colind, &m) != 0) return -2;
  *weights = (uint32_t*)malloc((size_t)(m > 0 ? m : 1) * 4);
  if (!*weights) return -2;
  rmat_w_ctx wc = {*rowptr, *colind, *weights, seed, (uint64_t)wmax - wmin + 1, wmin};
  run_ranges(threads, n, rmat_weights, &wc);
  *n_out = n;
  *m_out = m;
  return 0;
}

/* ---- grid ----------------------------------------------------------------- */
typedef struct {
  int64_t rows, cols, n, lattice_pairs, shortcut_pairs;
  uint64_t seed;
} grid_gen;

/* Pair index i: the lattice's horizontal pairs, then vertical ones, then the
 * shortcut pairs (the arc set, not the index order, defines the graph). */
static int grid_pair(const void* p, int64_t i, uint32_t* pu, uint32_t* pv) {
  const grid_gen* g = (const grid_gen*)p;
  const int64_t horiz = g->rows * (g->cols - 1);
  if (i < horiz) {
    const int64_t r = i / (g->cols - 1), cc = i % (g->cols - 1);
    *pu = (uint32_t)(r * g->cols + cc);
    *pv = *pu + 1;
    return 1;
  }
  if (i < g->lattice_pairs) {
    const int64_t k = i - horiz;   /* vertex k joins k + cols */
    *pu = (uint32_t)k;
    *pv = (uint32_t)(k + g->cols);
    return 1;
  }
  const uint64_t s = (uint64_t)(i - g->lattice_pairs);
  for (uint64_t t = 0;; ++t) {
    const uint64_t r = draw(g->seed, 5, s * 1024 + t);
    const uint32_t u = scale32((uint32_t)(r >> 32), (uint64_t)g->n);
    const uint32_t v = scale32((uint32_t)r, (uint64_t)g->n);
    if (u != v) {
      *pu = u;
      *pv = v;
      return 1;
    }
  }
}

typedef struct {
  const int64_t* rp;
  const int32_t* ci;
  uint32_t* w;
  uint64_t seed;
  double mu, sigma;
  uint32_t max_w;      /* largest weight drawn (atomic max) */
} grid_w_ctx;
static void grid_weights(void* p, int64_t lo, int64_t hi) {
  grid_w_ctx* c = (grid_w_ctx*)p;
  uint32_t mx = 0;
  for (int64_t u = lo; u < hi; ++u)
    for (int64_t e = c->rp[u]; e < c->rp[u + 1]; ++e) {
      const uint64_t key = ((uint64_t)u << 32) | (uint32_t)c->ci[e];
      const uint64_t r1 = draw(c->seed, 6, key), r2 = draw(c->seed, 7, key);
      const double u1 = ((double)(r1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);
      const double u2 = (double)(r2 >> 11) * (1.0 / 9007199254740992.0);
      const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
      double w = ceil(exp(c->mu + c->sigma * z));
      if (!(w >= 1.0)) w = 1.0;
      if (w > 2147483647.0) w = 2147483647.0;
      c->w[e] = (uint32_t)w;
      if ((uint32_t)w > mx) mx = (uint32_t)w;
    }
  uint32_t old = __atomic_load_n(&c->max_w, __ATOMIC_RELAXED);
  while (mx > old && !__atomic_compare_exchange_n(&c->max_w, &old, mx, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
}

int orc_gen_grid(int rows, int cols, double shortcut_frac, double mu, double sigma, uint64_t seed, int threads,
                 int64_t* n_out, int64_t* m_out, int64_t** rowptr, int32_t** colind, uint32_t** weights,
                 uint32_t* max_weight) {
  if (rows < 1 || cols < 1 || shortcut_frac < 0 || !(sigma >= 0)) return -1;
  grid_gen g;
  g.rows = rows;
  g.cols = cols;
  g.n = (int64_t)rows * cols;
  if (g.n < 2 || g.n >= ((int64_t)1 << 31)) return -1;
  g.lattice_pairs = (int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols;
  g.shortcut_pairs = llround(shortcut_frac * (double)(2 * g.lattice_pairs));
  g.seed = seed;
  int64_t m = 0;
  if (build_symmetric(g.n, g.lattice_pairs + g.shortcut_pairs, &g, grid_pair, threads, rowptr, colind, &m) != 0)
    return -2;
  *weights = (uint32_t*)malloc((size_t)(m > 0 ? m : 1) * 4);
  if (!*weights) return -2;
  grid_w_ctx wc;
  memset(&wc, 0, sizeof(wc));
  wc.rp = *rowptr;
  wc.ci = *colind;
  wc.w = *weights;
  wc.seed = seed;
  wc.mu = mu;
  wc.sigma = sigma;
  run_ranges(threads, g.n, grid_weights, &wc);
  *n_out = g.n;
  *m_out = m;
  *max_weight = wc.max_w;
  return 0;
}

void orc_free(void* p) { free(p); }
