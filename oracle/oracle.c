/*
 * oracle.c -- CPU restatement of the reference algorithms, used ONLY as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 * The product (libb200sssp.so) never links or calls this code.
 *
 * Parity is pinned against the reference's own golden vectors and outputs
 * (tests/golden/, generated by importing the reference's Python code), see
 * tests/test_oracle_golden.py.
 *
 * Functions and the reference code they follow (paths inside the reference
 * project charlottesylvie/rips2026-amd):
 *   orc_dijkstra_u32 / _f32 / _f64
 *       dijkstra_reference_incoming_csr,
 *       HIP_kernel/delta_stepping/testing/verify_bf_delta_vs_dijkstra.cpp:203-242
 *       (binary heap with lazy deletion; stale entries skipped when the
 *       popped key differs from dist[u]).  Run here on OUTGOING CSR.  uint32
 *       sums saturate to 0xFFFFFFFF like DistanceOps<uint32_t>::add
 *       (faster_GPU_algo/jasper_oneshot_untested/hip_adds_sssp.cpp:200-213);
 *       the f32 variant accumulates in float so it reproduces the unique
 *       fixpoint of float relaxation bit for bit.
 *   orc_bf_jacobi_f32 / _f64
 *       sssp_min_plus_bellman_ford + tropical_spmv,
 *       pytorch_testing/bellman_ford_attempts/Attempt1_June23/minplus_bellman_ford.py:51-102,
 *       minplus_algebra.py:58-102 (d <- min(d, A (x) d) on INCOMING CSR;
 *       iterations_used / converged / has_negative_cycle rules).  Unlike the
 *       python, convergence is exact equality (the python's np.isclose
 *       tolerance is irrelevant for the integer and float cases tested).
 *   orc_minplus_gemm_f32 / _i32
 *       minplus_kernel_f32, HIP_kernel/minplus_mm/src/minplus_hip.cpp:13-118
 *       (acc = candidate < acc ? candidate : acc, start +inf); the int32 twin
 *       clamps the result to INT32_MAX/2.
 *   orc_minplus_spgemm_f32
 *       minplus_spgemm_{symbolic,numeric}_kernel,
 *       HIP_kernel/minplus_mm/src/minplus_sparse_hip.cpp:93-99, 170-398
 *       (skip NaN/+inf entries and candidates, min-reduce duplicates);
 *       output columns sorted.
 *   orc_validate_spt
 *       shortest-path-tree check of a predecessor array (no reference
 *       counterpart on the GPU; the python keeps pred via _update_predecessors,
 *       minplus_bellman_ford.py:105-126).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- binary heap of (key, vertex) ------------------------------------ */
typedef struct { double k; uint64_t ku; uint32_t v; } hitem;
typedef struct { hitem* a; int64_t n, cap; int use_u; } heap;

static int lessh(const heap* h, const hitem* x, const hitem* y) {
  return h->use_u ? (x->ku < y->ku) : (x->k < y->k);
}
static void hpush(heap* h, hitem it) {
  if (h->n == h->cap) {
    h->cap = h->cap ? h->cap * 2 : 1024;
    h->a = (hitem*)realloc(h->a, (size_t)h->cap * sizeof(hitem));
  }
  int64_t i = h->n++;
  h->a[i] = it;
  while (i > 0) {
    int64_t p = (i - 1) / 2;
    if (!lessh(h, &h->a[i], &h->a[p])) break;
    hitem t = h->a[i]; h->a[i] = h->a[p]; h->a[p] = t;
    i = p;
  }
}
static hitem hpop(heap* h) {
  hitem top = h->a[0];
  h->a[0] = h->a[--h->n];
  int64_t i = 0;
  for (;;) {
    int64_t l = 2 * i + 1, r = l + 1, s = i;
    if (l < h->n && lessh(h, &h->a[l], &h->a[s])) s = l;
    if (r < h->n && lessh(h, &h->a[r], &h->a[s])) s = r;
    if (s == i) break;
    hitem t = h->a[i]; h->a[i] = h->a[s]; h->a[s] = t;
    i = s;
  }
  return top;
}

/* uint32 weights, saturating sums; INF = 0xFFFFFFFF.
 * keep_labels = 0: every label starts at INF.  keep_labels = 1: the labels
 * already in `dist` are kept as upper bounds and only the source (set to 0)
 * starts in the queue, so only vertices that a path from the source improves
 * are ever expanded -- the warm start of hip_adds::sssp with
 * Options::initialize_distances = false (hip_adds_sssp.hpp:64-66, its
 * init_kernel hip_adds_sssp.cpp:873-908). */
void orc_dijkstra_u32_from(int64_t n, const int64_t* rp, const int32_t* ci, const uint32_t* w, int64_t src,
                           uint32_t* dist, int keep_labels) {
  heap h = {0, 0, 0, 1};
  if (!keep_labels)
    for (int64_t i = 0; i < n; ++i) dist[i] = 0xFFFFFFFFu;
  dist[src] = 0;
  hitem s0 = {0.0, 0, (uint32_t)src};
  hpush(&h, s0);
  while (h.n) {
    hitem it = hpop(&h);
    const uint32_t u = it.v;
    if (it.ku != dist[u]) continue;
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e) {
      uint64_t nd = (uint64_t)dist[u] + w[e];
      if (nd > 0xFFFFFFFFull) nd = 0xFFFFFFFFull;
      const uint32_t v = (uint32_t)ci[e];
      if (nd < dist[v]) {
        dist[v] = (uint32_t)nd;
        hitem x = {0.0, nd, v};
        hpush(&h, x);
      }
    }
  }
  free(h.a);
}

void orc_dijkstra_u32(int64_t n, const int64_t* rp, const int32_t* ci, const uint32_t* w, int64_t src,
                      uint32_t* dist) {
  orc_dijkstra_u32_from(n, rp, ci, w, src, dist, 0);
}

/* uint32 Dijkstra ordered by (dist, hops): hops[v] = fewest arcs among the
 * shortest paths to v.  Jacobi Bellman-Ford converges after max(hops) rounds
 * and reports max(hops) + 1 iterations (the round that changes nothing).
 * Returns max hops over reached vertices. */
int64_t orc_dijkstra_u32_hops(int64_t n, const int64_t* rp, const int32_t* ci, const uint32_t* w, int64_t src,
                              uint32_t* dist, uint32_t* hops) {
  heap h = {0, 0, 0, 1};
  for (int64_t i = 0; i < n; ++i) { dist[i] = 0xFFFFFFFFu; hops[i] = 0xFFFFFFFFu; }
  dist[src] = 0;
  hops[src] = 0;
  hitem s0 = {0.0, 0, (uint32_t)src};
  hpush(&h, s0);
  int64_t mx = 0;
  while (h.n) {
    hitem it = hpop(&h);
    const uint32_t u = it.v;
    const uint64_t key = ((uint64_t)dist[u] << 32) | hops[u];
    if (it.ku != key) continue;
    if (hops[u] > mx) mx = hops[u];
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e) {
      uint64_t nd = (uint64_t)dist[u] + w[e];
      if (nd > 0xFFFFFFFFull) nd = 0xFFFFFFFFull;
      if (nd == 0xFFFFFFFFull) continue;
      const uint32_t v = (uint32_t)ci[e];
      const uint32_t nh = hops[u] + 1;
      if (nd < dist[v] || (nd == dist[v] && nh < hops[v])) {
        dist[v] = (uint32_t)nd;
        hops[v] = nh;
        hitem x = {0.0, (nd << 32) | nh, v};
        hpush(&h, x);
      }
    }
  }
  free(h.a);
  return mx;
}

/* float weights >= 0, float accumulation; unreachable = +inf.  keep_labels as
 * for orc_dijkstra_u32_from. */
void orc_dijkstra_f32_from(int64_t n, const int64_t* rp, const int32_t* ci, const float* w, int64_t src,
                           float* dist, int keep_labels) {
  heap h = {0, 0, 0, 0};
  if (!keep_labels)
    for (int64_t i = 0; i < n; ++i) dist[i] = INFINITY;
  dist[src] = 0.0f;
  hitem s0 = {0.0, 0, (uint32_t)src};
  hpush(&h, s0);
  while (h.n) {
    hitem it = hpop(&h);
    const uint32_t u = it.v;
    if ((float)it.k != dist[u]) continue;
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e) {
      volatile float nd = dist[u] + w[e];   /* one float rounding */
      const uint32_t v = (uint32_t)ci[e];
      if (nd < dist[v]) {
        dist[v] = nd;
        hitem x = {(double)nd, 0, v};
        hpush(&h, x);
      }
    }
  }
  free(h.a);
}

void orc_dijkstra_f32(int64_t n, const int64_t* rp, const int32_t* ci, const float* w, int64_t src,
                      float* dist) {
  orc_dijkstra_f32_from(n, rp, ci, w, src, dist, 0);
}

void orc_dijkstra_f64(int64_t n, const int64_t* rp, const int32_t* ci, const double* w, int64_t src,
                      double* dist) {
  heap h = {0, 0, 0, 0};
  for (int64_t i = 0; i < n; ++i) dist[i] = INFINITY;
  dist[src] = 0.0;
  hitem s0 = {0.0, 0, (uint32_t)src};
  hpush(&h, s0);
  while (h.n) {
    hitem it = hpop(&h);
    const uint32_t u = it.v;
    if (it.k != dist[u]) continue;
    for (int64_t e = rp[u]; e < rp[u + 1]; ++e) {
      const double nd = dist[u] + w[e];
      const uint32_t v = (uint32_t)ci[e];
      if (nd < dist[v]) {
        dist[v] = nd;
        hitem x = {nd, 0, v};
        hpush(&h, x);
      }
    }
  }
  free(h.a);
}

/* Jacobi Bellman-Ford on INCOMING CSR (row v lists in-edges u -> v).
 * out[0] = iterations_used, out[1] = converged, out[2] = has_negative_cycle,
 * out[3] = first iteration that changed nothing (0 if none observed).
 * max_iters < 0 means n - 1.  detect_neg: one extra round after the loop. */
#define BF_BODY(T, ADD)                                                                    \
  T* d = dist;                                                                             \
  T* nd = (T*)malloc((size_t)(n > 0 ? n : 1) * sizeof(T));                                 \
  for (int64_t i = 0; i < n; ++i) d[i] = (T)INFINITY;                                      \
  d[src] = 0;                                                                              \
  if (max_iters < 0) max_iters = n - 1;                                                    \
  int64_t used = 0, conv = 0, first_same = 0, neg = 0;                                     \
  for (int64_t it = 0; it < max_iters; ++it) {                                             \
    int changed = 0;                                                                       \
    for (int64_t v = 0; v < n; ++v) {                                                      \
      T best = d[v];                                                                       \
      for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {                                        \
        volatile T c = ADD(d[ci[e]], w[e]);                                                \
        if (c < best) best = c;                                                            \
      }                                                                                    \
      nd[v] = best;                                                                        \
      if (best < d[v]) changed = 1;                                                        \
    }                                                                                      \
    memcpy(d, nd, (size_t)n * sizeof(T));                                                  \
    used = it + 1;                                                                         \
    if (!changed) { conv = 1; first_same = used; break; }                                  \
  }                                                                                        \
  if (detect_neg && !conv) {                                                               \
    for (int64_t v = 0; v < n && !neg; ++v)                                                \
      for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {                                        \
        volatile T c = ADD(d[ci[e]], w[e]);                                                \
        if (c < d[v]) { neg = 1; break; }                                                  \
      }                                                                                    \
  }                                                                                        \
  free(nd);                                                                                \
  out[0] = used; out[1] = conv; out[2] = neg; out[3] = first_same;

#define FADD(a, b) ((a) + (b))
void orc_bf_jacobi_f32(int64_t n, const int64_t* rp, const int32_t* ci, const float* w, int64_t src,
                       int64_t max_iters, int detect_neg, float* dist, int64_t* out) {
  BF_BODY(float, FADD)
}
void orc_bf_jacobi_f64(int64_t n, const int64_t* rp, const int32_t* ci, const double* w, int64_t src,
                       int64_t max_iters, int detect_neg, double* dist, int64_t* out) {
  BF_BODY(double, FADD)
}

/* ---- dense min-plus -------------------------------------------------- */
void orc_minplus_gemm_f32(const float* A, const float* B, float* Cm, int64_t M, int64_t N, int64_t K,
                          int64_t lda, int64_t ldb, int64_t ldc) {
  for (int64_t i = 0; i < M; ++i)
    for (int64_t j = 0; j < N; ++j) {
      float acc = INFINITY;
      for (int64_t k = 0; k < K; ++k) {
        volatile float c = A[i * lda + k] + B[k * ldb + j];
        acc = c < acc ? c : acc;
      }
      Cm[i * ldc + j] = acc;
    }
}

void orc_minplus_gemm_i32(const int32_t* A, const int32_t* B, int32_t* Cm, int64_t M, int64_t N, int64_t K,
                          int64_t lda, int64_t ldb, int64_t ldc) {
  const int32_t cap = 1073741823;
  for (int64_t i = 0; i < M; ++i)
    for (int64_t j = 0; j < N; ++j) {
      int64_t acc = cap;
      for (int64_t k = 0; k < K; ++k) {
        const int64_t c = (int64_t)A[i * lda + k] + (int64_t)B[k * ldb + j];
        if (c < acc) acc = c;
      }
      Cm[i * ldc + j] = (int32_t)acc;
    }
}

/* ---- CSR x CSR min-plus -------------------------------------------------
 * Returns nnz(C); C arrays must hold `cap` entries (call with cap = 0 to size).
 * Dense accumulator per row (fine for the oracle's small sizes). */
/* columns touched by one output row (sorted before the row is written) */
typedef struct { int32_t* a; int64_t n, cap; } cols_t;
static void cols_push(cols_t* t, int32_t j) {
  if (t->n == t->cap) {
    t->cap = t->cap ? t->cap * 2 : 256;
    t->a = (int32_t*)realloc(t->a, (size_t)t->cap * sizeof(int32_t));
  }
  t->a[t->n++] = j;
}
static int cmp_i32(const void* x, const void* y) {
  const int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
  return (a > b) - (a < b);
}

int64_t orc_minplus_spgemm_f32(int64_t M, int64_t K, int64_t N, const int64_t* arp, const int32_t* aci,
                               const float* av, const int64_t* brp, const int32_t* bci, const float* bv,
                               int64_t* crp, int32_t* cci, float* cv, int64_t cap) {
  float* acc = (float*)malloc((size_t)(N > 0 ? N : 1) * sizeof(float));
  unsigned char* has = (unsigned char*)calloc((size_t)(N > 0 ? N : 1), 1);
  cols_t t = {0, 0, 0};
  int64_t nnz = 0;
  (void)K;
  for (int64_t i = 0; i < M; ++i) {
    if (crp) crp[i] = nnz;
    t.n = 0;
    for (int64_t p = arp[i]; p < arp[i + 1]; ++p) {
      const float a = av[p];
      if (a != a || a == INFINITY) continue;
      const int32_t k = aci[p];
      for (int64_t q = brp[k]; q < brp[k + 1]; ++q) {
        volatile float c = a + bv[q];
        if (c != c || c == INFINITY) continue;
        const int32_t j = bci[q];
        if (!has[j]) { has[j] = 1; acc[j] = c; cols_push(&t, j); }
        else if (c < acc[j]) acc[j] = c;
      }
    }
    qsort(t.a, (size_t)t.n, sizeof(int32_t), cmp_i32);
    for (int64_t x = 0; x < t.n; ++x) {
      const int32_t j = t.a[x];
      if (cci && nnz < cap) { cci[nnz] = j; cv[nnz] = acc[j]; }
      ++nnz;
      has[j] = 0;
    }
  }
  if (crp) crp[M] = nnz;
  free(acc);
  free(has);
  free(t.a);
  return nnz;
}

/* int32 twin: entries >= INT32_MAX/2 are absent; sums clamped to it and dropped. */
int64_t orc_minplus_spgemm_i32(int64_t M, int64_t K, int64_t N, const int64_t* arp, const int32_t* aci,
                               const int32_t* av, const int64_t* brp, const int32_t* bci, const int32_t* bv,
                               int64_t* crp, int32_t* cci, int32_t* cv, int64_t cap) {
  const int64_t miss = 1073741823;
  int64_t* acc = (int64_t*)malloc((size_t)(N > 0 ? N : 1) * sizeof(int64_t));
  unsigned char* has = (unsigned char*)calloc((size_t)(N > 0 ? N : 1), 1);
  cols_t t = {0, 0, 0};
  int64_t nnz = 0;
  (void)K;
  for (int64_t i = 0; i < M; ++i) {
    if (crp) crp[i] = nnz;
    t.n = 0;
    for (int64_t p = arp[i]; p < arp[i + 1]; ++p) {
      const int64_t a = av[p];
      if (a >= miss) continue;
      const int32_t k = aci[p];
      for (int64_t q = brp[k]; q < brp[k + 1]; ++q) {
        const int64_t b = bv[q];
        if (b >= miss) continue;
        const int64_t c = a + b;
        if (c >= miss) continue;
        const int32_t j = bci[q];
        if (!has[j]) { has[j] = 1; acc[j] = c; cols_push(&t, j); }
        else if (c < acc[j]) acc[j] = c;
      }
    }
    qsort(t.a, (size_t)t.n, sizeof(int32_t), cmp_i32);
    for (int64_t x = 0; x < t.n; ++x) {
      const int32_t j = t.a[x];
      if (cci && nnz < cap) { cci[nnz] = j; cv[nnz] = (int32_t)acc[j]; }
      ++nnz;
      has[j] = 0;
    }
  }
  if (crp) crp[M] = nnz;
  free(acc);
  free(has);
  free(t.a);
  return nnz;
}

/* ---- shortest-path tree check ------------------------------------------
 * OUTGOING CSR.  kind 0: uint32 (saturating), 1: float.  Returns 0 if pred is
 * a valid SPT for dist, else a positive code:
 *   1 source pred not -1, 2 reached vertex without pred, 3 pred edge missing,
 *   4 dist[pred] + w != dist[v], 5 unreached vertex with pred, 6 cycle. */
int orc_validate_spt(int64_t n, const int64_t* rp, const int32_t* ci, const void* wts, int kind,
                     int64_t src, const void* dist, const int32_t* pred) {
  if (pred[src] != -1) return 1;
  for (int64_t v = 0; v < n; ++v) {
    if (v == src) continue;
    int reached;
    if (kind == 0) reached = ((const uint32_t*)dist)[v] != 0xFFFFFFFFu;
    else reached = isfinite(((const float*)dist)[v]);
    if (!reached) { if (pred[v] != -1) return 5; continue; }
    const int32_t u = pred[v];
    if (u < 0 || u >= n) return 2;
    int ok = 0;
    for (int64_t e = rp[u]; e < rp[u + 1] && !ok; ++e) {
      if (ci[e] != v) continue;
      if (kind == 0) {
        uint64_t s = (uint64_t)((const uint32_t*)dist)[u] + ((const uint32_t*)wts)[e];
        if (s > 0xFFFFFFFFull) s = 0xFFFFFFFFull;
        ok = (uint32_t)s == ((const uint32_t*)dist)[v];
      } else {
        volatile float s = ((const float*)dist)[u] + ((const float*)wts)[e];
        ok = s == ((const float*)dist)[v];
      }
    }
    if (!ok) {
      int has_edge = 0;
      for (int64_t e = rp[u]; e < rp[u + 1]; ++e) if (ci[e] == v) has_edge = 1;
      return has_edge ? 4 : 3;
    }
  }
  /* every reached vertex reaches the source following pred (no cycles) */
  unsigned char* state = (unsigned char*)calloc((size_t)n, 1); /* 0 new, 1 on path, 2 done */
  int64_t* stack = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  state[src] = 2;
  int bad = 0;
  for (int64_t v = 0; v < n && !bad; ++v) {
    if (state[v] || pred[v] < 0) continue;
    int64_t top = 0, x = v;
    while (!state[x] && pred[x] >= 0) { state[x] = 1; stack[top++] = x; x = pred[x]; }
    if (state[x] == 1) bad = 1;
    while (top) state[stack[--top]] = 2;
  }
  free(state);
  free(stack);
  return bad ? 6 : 0;
}
