/*
 * b200sssp.h -- C ABI of the B200 SSSP / min-plus library (libb200sssp.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, never
 * throws, and reports failure through b2_status.  Device pointers are CUDA
 * device memory owned by the caller unless stated otherwise.  `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Reference interfaces replaced (charlottesylvie/rips2026-amd, paths inside
 * that project):
 *   b2_sssp_bf            <- bellman_ford_minplus_hip_csr
 *                            (HIP_kernel/bellman_ford/src/bf_hip_CSR.hpp:41-66),
 *                            _no_checks (bf_hip_no_checks_CSR.hpp:17-42),
 *                            _var_checks (bf_var_checks.hpp:32-71),
 *                            bellman_ford_sssp_hip
 *                            (HIP_kernel/faster_GPU_algo/Charlotte_oneshot/sssp_hip.hpp:51-54)
 *   b2_sssp_bf_dense      <- bellman_ford_minplus_hip
 *                            (HIP_kernel/bellman_ford/src/bellman_ford_hip.hpp:15-60)
 *   b2_sssp_delta         <- delta_stepping_minplus_hip_csr
 *                            (HIP_kernel/delta_stepping/src/delta_stepping_hip_CSR.hpp:15-67)
 *   b2_sssp_adds          <- adds_sssp_hip (Charlotte_oneshot/sssp_hip.hpp:56-59) and
 *                            hip_adds::sssp
 *                            (faster_GPU_algo/jasper_oneshot_untested/hip_adds_sssp.hpp:101-113)
 *   b2_minplus_gemm_f32   <- minplus_gemm_f32 (HIP_kernel/minplus_mm/src/minplus_hip.hpp:24-33)
 *   b2_minplus_gemm_i32   <- (int32 twin of the above; the reference is fp32 only)
 *   b2_minplus_spgemm_f32 <- minplus_sparse::minplus_spgemm_csr_f32 / _large_rows / _tuned
 *                            (HIP_kernel/minplus_mm/src/minplus_sparse_hip.hpp:64-150)
 *   b2_minplus_spgemm_i32 <- (int32 twin of the above)
 *   b2_delta_heuristic    <- choose_initial_delta (Charlotte_oneshot/sssp_hip.cpp:59-81),
 *                            estimate_initial_delta (hip_adds_sssp.cpp:1080-1127)
 *   b2_dimacs_read, b2_dimacs_to_csrbin <- load_dimacs_gr_as_incoming_csr and the converter main
 *                            (HIP_kernel/bellman_ford/src/gr_to_csr.cpp:124-326)
 *   b2_lonestar_read/write <- CSRGraph::readFromGR
 *                            (faster_GPU_algo/Charlotte_ADS_Float_Attempt/csr_graph.cpp:153-291)
 *   b2_csrbin_read/write  <- RIPSCSR1 writer/loaders (HIP_kernel/bellman_ford/src/gr_to_csr.cpp:34-57,
 *                            :243-278; tests/big_test.cpp:160-276)
 */
#ifndef B200SSSP_H_
#define B200SSSP_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2_ABI_VERSION 1

typedef enum b2_status {
  B2_SUCCESS = 0,
  B2_INVALID_ARGUMENT = 1, /* bad pointer, size, source, orientation, weight */
  B2_CUDA_ERROR = 2,       /* a CUDA runtime call failed */
  B2_OUT_OF_MEMORY = 3,
  B2_POOL_EXHAUSTED = 4,   /* a device worklist ran out of capacity */
  B2_BUCKET_OVERFLOW = 5,
  B2_DEVICE_ERROR = 6,     /* a device-side consistency check failed */
  B2_TIMEOUT = 7,          /* a bounded device wait ran out (kernel exited cleanly) */
  B2_NOT_SUPPORTED = 8,    /* valid request outside this build's limits */
  B2_INVALID_INDEX = 9,    /* CSR column index out of range */
  B2_INVALID_ROWPTR = 10,  /* CSR row pointer not monotone / out of range */
  B2_INVALID_WEIGHT = 11,  /* negative / NaN weight where the method forbids it */
  B2_CANCELLED = 12        /* serving: the query was cancelled before it ran */
} b2_status;

typedef void* b2_stream; /* cudaStream_t */

typedef enum b2_weight_type { B2_W_U32 = 0, B2_W_F32 = 1 } b2_weight_type;

/* Incoming: row v lists edges u -> v (column u); the Bellman-Ford / delta /
 * RIPSCSR1 convention.  Outgoing: row u lists edges u -> v; the oneshot / ADDS
 * convention. */
typedef enum b2_orientation { B2_INCOMING = 0, B2_OUTGOING = 1 } b2_orientation;

/* Non-owning CSR view.  rowptr is int64 (rowptr_bits = 64, the
 * minplus_sparse::Offset convention) or 32-bit (rowptr_bits = 32, the oneshot
 * int / hip_adds uint32 convention).  colind is 32-bit.  values are uint32 or
 * float according to weight_type. */
typedef struct b2_csr {
  int64_t rows;
  int64_t cols;
  int64_t nnz;
  const void* rowptr;
  const int32_t* colind;
  const void* values;
  int32_t rowptr_bits;
  int32_t weight_type;
  int32_t orientation;
  int32_t on_device; /* 1: arrays are device pointers; 0: host pointers */
} b2_csr;

/* Resident graph: outgoing CSR packed as (dst, weight) pairs in HBM plus the
 * solver workspace; built once, reused by every solve. */
typedef struct b2_graph_s* b2_graph;

typedef struct b2_graph_info {
  int64_t n;
  int64_t m;
  int32_t weight_type;
  int32_t max_out_degree;
  double mean_weight;       /* over edges with weight > 0 */
  double mean_degree;
  size_t device_bytes;      /* graph + workspace */
} b2_graph_info;

typedef enum b2_method {
  B2_METHOD_BF = 0,      /* frontier Bellman-Ford, Jacobi rounds (hop-exact) */
  B2_METHOD_DELTA = 1,   /* delta-stepping, device ring buckets, one persistent launch */
  B2_METHOD_ADDS = 2     /* asynchronous worklist (no phase barriers inside a bucket window) */
} b2_method;

typedef enum b2_bf_check {
  B2_BF_CHECKED = 0,    /* stop at the first iteration with no change */
  B2_BF_NO_CHECKS = 1,  /* report exactly max_iters iterations */
  B2_BF_VAR_CHECKS = 2  /* convergence observed only every check_interval iterations */
} b2_bf_check;

/* Progress of a running solve, reported to b2_sssp_opts.progress from the
 * calling thread while the persistent kernel runs (it publishes each finished
 * round or bucket to mapped host memory; the call polls it).  The reference
 * calls its BellmanFordCsrProgressCallback once per iteration from its host
 * loop (bf_hip_CSR.cpp:79-95). */
typedef struct b2_progress {
  int32_t iteration;        /* BF: rounds finished; delta / ADDS: non-empty buckets settled */
  int32_t max_iters;        /* the solve's limit (-1: none) */
  int32_t changed;          /* BF: the round changed a distance; delta / ADDS: 1 */
  int32_t reserved;
  double elapsed_ms;        /* device time from the solve's start to the round's end */
} b2_progress;
typedef void (*b2_progress_fn)(const b2_progress* progress, void* user_data);

typedef struct b2_sssp_opts {
  int32_t max_iters;        /* BF: rounds (<0: n-1).  delta: buckets (<0: unbounded). */
  int32_t bf_check;         /* b2_bf_check */
  int32_t check_interval;   /* for B2_BF_VAR_CHECKS */
  int32_t policy;           /* 0: fixed delta (opts.delta or the Near-Far heuristic);
                               1: learned (b2_policy_activate); overrides delta,
                               the push/pull switch and a zero fusion_threshold */
  double delta;             /* bucket width; <=0 selects the Near-Far heuristic */
  double delta_scale;       /* Near-Far constant C in delta = C * mean_w / mean_deg (16) */
  uint32_t hub_degree;      /* vertices with out-degree >= this are split into edge chunks */
  uint32_t fusion_threshold;/* frontier size under which one block runs sub-phases alone (0 = off) */
  float pull_fraction;      /* push/pull switch of the delta-stepping heavy pass: pull (each
                               unsettled vertex scans its heavy in-edges, weight order, early
                               exit) when the bucket's members hold more than pull_fraction x n
                               heavy out-edges (default 8); the incoming CSR is built on first
                               use, only for graphs with m >= pull_fraction x n; <= 0: push only */
  uint32_t grid_blocks;     /* 0: the co-resident persistent grid (BF / delta: at most one thread
                               per vertex on small graphs); k: at most k blocks */
  double timeout_ms;        /* bound on the whole solve and on every device wait, in ms
                               (default 20000; fractions of a millisecond allowed): past it the
                               kernel stops at its next wait or phase boundary and the call
                               returns B2_TIMEOUT; the graph handle stays usable */
  int32_t collect_reach;    /* fill stats.reached / reached_edges (one extra O(n) pass) */
  int32_t detect_negative_cycle; /* BF: one extra round after max_iters (python reference rule) */
  int32_t light_heavy;      /* delta: relax light edges (w <= delta) per sub-phase and heavy
                               edges once per settled vertex (default 1) */
  int32_t trace;            /* record one b2_trace_entry per phase (b2_graph_trace) */
  float dense_fraction;     /* delta / ADDS: a near or window-slot frontier of at least
                               dense_fraction x n vertices is found by sweeping the per-vertex
                               push / bucket stamps in vertex order instead of reading its
                               queue (ordered access to labels and rows); 0 (default): 1/16
                               on graphs whose largest out-degree is <= 64, else the queue;
                               < 0: always the queue */
  uint32_t worklist_capacity; /* delta / ADDS / BF: entries each device worklist may hold; 0
                               (default): n, which no solve can exceed.  A smaller value bounds
                               the queues like the reference's fixed-capacity frontier queues
                               (delta_stepping_hip_CSR.cpp:616-620): a solve that would push
                               past it stops and returns B2_POOL_EXHAUSTED */
  int32_t keep_distances;   /* ADDS only: 1 = warm start -- d_dist holds starting distances
                               (input ids; uint32 0xFFFFFFFF or float +inf = none) that stay
                               as upper bounds; only the source (set to 0) starts queued, so
                               only vertices a path from the source improves are expanded.
                               hip_adds::Options::initialize_distances = false
                               (hip_adds_sssp.hpp:64-66).  0 (default): every distance starts
                               at infinity.  Other methods return B2_NOT_SUPPORTED for 1. */
  uint32_t active_buckets;  /* ADDS: buckets from the lowest unfinished one that warps may take
                               entries from at the start of a window (0: 2); grows while warps
                               idle and later buckets hold work (the reference's dynamic
                               active-bucket count, hip_adds_sssp.hpp:37-38) */
  int32_t adds_fixed_delta; /* ADDS: 1 keeps the bucket width fixed (the reference's
                               dynamic_delta = false); 0 (default): growth 1.5 / shrink 0.75 at
                               every new window from the last window's utilization */
  b2_progress_fn progress;  /* nullable: called once per finished round / bucket, in order,
                               while the solve runs (every call precedes the return) */
  void* progress_user;
  uint32_t max_active_buckets; /* ADDS: the active range never widens past this many buckets
                               (0: 32, the whole window; hip_adds::Options::max_active_buckets,
                               hip_adds_sssp.hpp:37-38).  Equal to active_buckets: no widening
                               (the reference's dynamic_active_buckets = false). */
  int32_t reserved[2];
} b2_sssp_opts;

typedef struct b2_trace_entry {
  uint32_t kind;        /* 1 relax, 2 commit, 3 far split, 4 probe, 5 output, 7 fused (one block),
                           8 heavy pass by pull; | 0x100 heavy pass; | 0x200 frontier found by
                           a stamp sweep */
  uint32_t frontier;    /* frontier entries of the phase */
  uint32_t hub_chunks;  /* 256-edge chunks of split high-degree vertices */
  uint32_t bucket;      /* delta: bucket index; BF: round */
  uint64_t t_ns;        /* phase end, ns after the solve's first barrier */
} b2_trace_entry;

typedef struct b2_stats {
  int32_t iterations_used;  /* BF: rounds; delta/ADDS: non-empty buckets processed */
  int32_t converged;
  int32_t has_negative_cycle;
  int32_t phases;           /* barrier-separated phases executed by the persistent kernel */
  uint64_t edges_scanned;   /* edges read during relaxation */
  uint64_t improvements;    /* successful atomic-min updates */
  uint64_t pushes;          /* worklist insertions */
  uint64_t reached;         /* vertices with finite distance */
  uint64_t reached_edges;   /* out-edges of reached vertices (TEPS numerator) */
  double delta_used;
  float kernel_ms;          /* device time of the persistent launch */
  uint32_t device_error;
  uint32_t grid_blocks;
  uint32_t first_unchanged; /* BF: first round that changed nothing (0: none observed) */
  uint32_t local_subphases; /* delta/ADDS: sub-phases run by one block under bucket fusion */
  uint32_t delta_updates;   /* ADDS: bucket-width changes */
  double delta_final;       /* ADDS: bucket width at the end (delta: = delta_used) */
  uint32_t policy_used;     /* 1: the learned policy chose delta / fusion / light-heavy */
  uint32_t heavy_pulls;     /* heavy passes run in the pull direction */
  uint64_t work_items;      /* ADDS: bucket-queue entries and hub chunks taken by warps */
  uint32_t active_buckets_max; /* ADDS: widest range of buckets warps took entries from */
  uint32_t device_error_site; /* where in the kernel device_error was raised (0: none) */
} b2_stats;

/* ---- library ---------------------------------------------------------- */
const char* b2_status_string(b2_status s);
int b2_abi_version(void);
void b2_sssp_opts_default(b2_sssp_opts* opts);
/* cudaFree / cudaMemcpyAsync(D2D) for callers without their own CUDA runtime
 * (ctypes, cgo): frees the callee-allocated SpGEMM outputs. */
b2_status b2_device_free(void* d_ptr);
b2_status b2_device_copy(void* d_dst, const void* d_src, size_t bytes, b2_stream stream);

/* ---- resident graphs -------------------------------------------------- */
b2_status b2_graph_create(const b2_csr* csr, b2_stream stream, b2_graph* out);
b2_status b2_graph_destroy(b2_graph g);
b2_status b2_graph_info_get(b2_graph g, b2_graph_info* info);
/* Degree order (no reference counterpart): renumber the resident graph's
 * vertices internally by out-degree, descending, so the few hot vertices of a
 * skewed graph share cache lines.  Every interface keeps input vertex ids:
 * sources are mapped in and distances / predecessors scattered back.
 * b2_graph_create applies it by itself to graphs with >= 2^23 vertices and
 * max degree >= 64 x mean degree; this call forces it (idempotent). */
b2_status b2_graph_set_degree_order(b2_graph g, b2_stream stream);
int32_t b2_graph_degree_ordered(b2_graph g);
/* Near-Far delta = scale * mean(w > 0) / mean degree (>= 1 for uint32). */
b2_status b2_delta_heuristic(b2_graph g, double scale, double* delta_out);
/* Phase trace of the last solve on g that ran with opts.trace = 1. */
b2_status b2_graph_trace(b2_graph g, b2_trace_entry* entries, int32_t capacity, int32_t* count);

/* ---- SSSP -------------------------------------------------------------
 * d_dist: n words of the graph's weight type (uint32: 0xFFFFFFFF = unreachable;
 * float: +inf = unreachable).  d_pred: n int32 (nullable); -1 = none/source.
 * Predecessors form a shortest-path tree when every cycle has positive weight;
 * ties pick the smallest predecessor id. */
b2_status b2_sssp_bf(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred,
                     const b2_sssp_opts* opts, b2_stream stream, b2_stats* stats);
b2_status b2_sssp_delta(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred,
                        const b2_sssp_opts* opts, b2_stream stream, b2_stats* stats);
b2_status b2_sssp_adds(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred,
                       const b2_sssp_opts* opts, b2_stream stream, b2_stats* stats);
/* Dense incoming adjacency (d_adj[v*n+u] = w(u->v), +inf/NaN = no edge). */
b2_status b2_sssp_bf_dense(const float* d_adj, int32_t n, uint32_t source, float* d_dist,
                           const b2_sssp_opts* opts, b2_stream stream, b2_stats* stats);

/* ---- min-plus products ------------------------------------------------
 * C[i,j] = min_k A[i,k] + B[k,j], row-major with leading dimensions.
 * f32: NaN candidates are ignored, empty min = +inf.
 * i32: inputs must lie in [-2^30, 2^30-1]; C is clamped to <= INT32_MAX/2
 *      (1073741823, the "missing" sentinel).  Asynchronous on `stream`: the
 * return value covers the launch only; b2_minplus_status reports a product
 * whose bounded wait gave up. */
b2_status b2_minplus_gemm_f32(const float* dA, const float* dB, float* dC, int32_t M,
                              int32_t N, int32_t K, int32_t lda, int32_t ldb, int32_t ldc,
                              b2_stream stream);
b2_status b2_minplus_gemm_i32(const int32_t* dA, const int32_t* dB, int32_t* dC, int32_t M,
                              int32_t N, int32_t K, int32_t lda, int32_t ldb, int32_t ldc,
                              b2_stream stream);
/* All-pairs shortest paths by repeated squaring of an N x N matrix in place
 * (d_D must have a zero diagonal).  Stops early when a squaring changes
 * nothing.  *squarings_out = products computed. */
b2_status b2_apsp_f32(float* d_D, int32_t N, b2_stream stream, int32_t* squarings_out);
b2_status b2_apsp_i32(int32_t* d_D, int32_t N, b2_stream stream, int32_t* squarings_out);
/* Waits for `stream`, then returns B2_TIMEOUT if a min-plus product launched
 * on this device since the last b2_minplus_gemm_* / b2_apsp_* call began had
 * a bounded shared-memory wait give up (its output is then not valid), else
 * B2_SUCCESS.  The record is one word per device, cleared in stream order by
 * every GEMM and APSP call: products that overlap on different streams share
 * it.  No counterpart in the reference (its waits are unbounded). */
b2_status b2_minplus_status(b2_stream stream);
/* b2_apsp_f32 without any device allocation, for callers that cannot call
 * cudaMalloc while they run (a plugin whose host owns the device memory pool,
 * a serving loop with a fixed memory budget).  No counterpart in the
 * reference.  Its scratch is a fixed 16 MiB module array, so N <= 2048
 * (larger N returns B2_NOT_SUPPORTED); each GPU that loads the library holds
 * that array until exit.  All calls on a device share it: calls that overlap
 * on the GPU race and must be serialized by the caller.  The first call on a
 * device resolves the array's device address (cudaGetSymbolAddress) with that
 * device current.  Every call synchronizes `stream` after each squaring (it
 * reads the change flag on the host), so no call may be made on a stream that
 * is being captured. */
b2_status b2_apsp_f32_noalloc(float* d_D, int32_t N, b2_stream stream, int32_t* squarings_out);
/* Sustained (min,+) pairs per second of this GPU's CUDA cores, measured by a
 * register-only kernel of the same instruction mix as the GEMM inner loop
 * (int32: DPX add-min; fp32: FADD + three-input min).  The roofline
 * denominator for the min-plus GEMM.  Synchronous, current device. */
b2_status b2_minplus_calibrate(int32_t is_float, double* pairs_per_second);

/* CSR x CSR min-plus.  Outputs are cudaMalloc'd by the callee and owned by
 * the caller (cudaFree).  Absent = +inf; explicit +inf / NaN entries and
 * candidates are skipped; duplicates are min-reduced.  Output columns are
 * sorted within each row.  A, B: on_device = 1, rowptr_bits = 64. */
b2_status b2_minplus_spgemm_f32(const b2_csr* A, const b2_csr* B, int64_t** dC_rowptr,
                                int32_t** dC_colind, float** dC_values, int64_t* hC_nnz,
                                b2_stream stream);
/* int32 values: absent = missing; entries >= INT32_MAX/2 are skipped. */
b2_status b2_minplus_spgemm_i32(const b2_csr* A, const b2_csr* B, int64_t** dC_rowptr,
                                int32_t** dC_colind, int32_t** dC_values, int64_t* hC_nnz,
                                b2_stream stream);
/* The same product in two steps, for callers that allocate C themselves (no
 * reference counterpart).  b2_minplus_spgemm_plan computes C into library
 * scratch (stream-ordered pool memory) and returns nnz(C) on the host; the
 * caller allocates C.rowptr (rows + 1 int64), C.colind (nnz int32) and
 * C.values (nnz, A's weight type: float or int32), and b2_minplus_spgemm_fill
 * writes them asynchronously on `stream` and releases the plan.
 * b2_minplus_spgemm_plan_free releases a plan that is not filled.  A and B
 * must have the same weight_type. */
typedef struct b2_spgemm_plan_s* b2_spgemm_plan;
b2_status b2_minplus_spgemm_plan(const b2_csr* A, const b2_csr* B, b2_stream stream, b2_spgemm_plan* plan,
                                 int64_t* hC_nnz);
b2_status b2_minplus_spgemm_fill(b2_spgemm_plan plan, int64_t* dC_rowptr, int32_t* dC_colind, void* dC_values,
                                 b2_stream stream);
b2_status b2_minplus_spgemm_plan_free(b2_spgemm_plan plan);

/* ---- learned schedule policy -------------------------------------------
 * No counterpart in the reference (it picks delta with the Near-Far rule,
 * Charlotte_oneshot/sssp_hip.cpp:59-81, which stays the fallback).
 * Graph features (24 floats) -> MLP 24-64-64-3 (ReLU; BF16 weights, FP32
 * accumulation; 5955 parameters in the order W1[64x24] b1 W2[64x64] b2
 * W3[3x64] b3) -> y0 = log2(delta / Near-Far delta) (clamped to [-4, 6]),
 * y1 > 0: bucket fusion on (threshold 1024), y2 > 0: light/heavy split on.
 * Features are standardized with the policy's mean/std before the MLP.
 * Solves with opts.policy = 1 use the active policy; without one they run the
 * fixed Near-Far schedule (stats.policy_used = 0).  Distances never depend on
 * the policy. */
typedef struct b2_policy_s* b2_policy;
int32_t b2_policy_param_count(void);
b2_status b2_policy_create(uint64_t seed, b2_policy* out);
b2_status b2_policy_destroy(b2_policy p);
/* params: 5955 floats; mu, sigma: 24 floats each (both NULL: unchanged). */
b2_status b2_policy_set_params(b2_policy p, const float* params, const float* mu, const float* sigma);
b2_status b2_policy_get_params(b2_policy p, float* params, float* mu, float* sigma);
/* Solves keep the Near-Far delta when the network's |log2 multiplier| is below
 * log2_dead_zone (chosen by cross-validation when the weights are trained;
 * stored in the weight file).  Default 0. */
b2_status b2_policy_set_dead_zone(b2_policy p, float log2_dead_zone);
/* Clamp each raw feature to [lo[k], hi[k]] before it is normalized (the range
   of the training graphs; training sets it from its X).  lo = hi = NULL: no
   clamping. */
b2_status b2_policy_set_feature_range(b2_policy p, const float* lo, const float* hi);
/* X: B x 24 raw features; Y: B x 3 outputs. */
b2_status b2_policy_forward(b2_policy p, const float* X, int32_t B, float* Y);
/* Gradient of the mean loss (y0-t0)^2 + BCE(y1,t1) + BCE(y2,t2) over the
 * batch at the current weights; grad: 5955 floats (nullable). */
b2_status b2_policy_gradient(b2_policy p, const float* X, const float* T, int32_t B, float* grad,
                             float* loss);
/* Full-batch AdamW (decoupled weight decay) for `epochs` steps; the first
 * call also fixes mu/sigma from X. */
b2_status b2_policy_train(b2_policy p, const float* X, const float* T, int32_t B, int32_t epochs,
                          float lr, float weight_decay, float* loss_out);
/* Make p the policy of opts.policy = 1 solves (NULL: none). */
b2_status b2_policy_activate(b2_policy p);
/* The 24 schedule features of g (cached on the handle). */
b2_status b2_graph_features(b2_graph g, float* features);

/* ---- batched serving ----------------------------------------------------
 * No counterpart in the reference (it answers one query per launch
 * sequence).  A server holds resident graphs (b2_graph handles that must
 * outlive it), a device arena of hbm_budget_bytes, and a few CUDA streams.
 * Submitted single-source queries wait in FIFO order until their arena slot
 * fits in the budget (b2_server_slot_bytes; a query that can never fit is
 * refused with B2_OUT_OF_MEMORY at submit), then run in batch launches where
 * one thread block solves one query alone (delta-stepping, block barriers
 * only).  Every query owns its slot: results do not depend on what else runs.
 * out_dist / out_pred must be device memory or page-locked host memory
 * (cudaHostAlloc / cudaHostRegister); the block writes the result there
 * directly and a query completes on its own, not with its batch.  Graphs
 * with negative weights are refused (B2_INVALID_WEIGHT).  Calls on one
 * server are serialized internally. */
typedef struct b2_server_s* b2_server;
typedef struct b2_server_opts {
  size_t hbm_budget_bytes;  /* device arena (default 1 GiB) */
  int32_t max_batch;        /* queries per batch launch (default 512) */
  int32_t lanes;            /* streams with one batch in flight each (default 16) */
  int32_t max_inflight;     /* completion records (default 8192) */
  int32_t blocks_per_sm;    /* 0: occupancy limit */
  double timeout_ms;        /* per-query device budget (default 20000) */
  double delta_scale;       /* Near-Far constant for each graph's bucket width (default 4:
                               one block's phases end with block barriers, so narrower buckets
                               with fewer wasted relaxations pay off) */
  int32_t big_vertices;     /* graphs with at least this many vertices are solved by a cluster of
                               8 blocks (distributed shared memory, cluster barriers) on a
                               quarter of the lanes; 0: 2^19; < 0: never */
  int32_t autotune;         /* 1: b2_server_add_graph times batches that fill the GPU under each
                               team (block / cluster) x Near-Far constant (2, 4, 8) and keeps the
                               fastest for that graph (needs an idle server); 0: the defaults */
  int32_t reserved[2];
} b2_server_opts;
typedef struct b2_completion {
  uint64_t ticket;
  int32_t status;           /* B2_SUCCESS, B2_TIMEOUT, B2_CANCELLED, ... */
  int32_t graph_id;
  uint32_t source;
  uint32_t phases;
  uint64_t edges_scanned;
  uint64_t reached;
  uint64_t reached_edges;
  double latency_us;        /* submit -> result in the caller's buffer, observed by the host */
} b2_completion;
typedef struct b2_server_info_t {
  int32_t graphs;
  uint32_t blocks;          /* resident blocks of one batch launch */
  int64_t pending;
  int64_t running;
  int64_t completed_unpolled;
  size_t arena_bytes;
  size_t arena_used;
} b2_server_info_t;
void b2_server_opts_default(b2_server_opts* opts);
b2_status b2_server_create(const b2_server_opts* opts, b2_server* out);
b2_status b2_server_destroy(b2_server s);
b2_status b2_server_add_graph(b2_server s, b2_graph g, int32_t* graph_id);
/* The configuration a graph's queries run with: cluster team (1) or one block
 * (0), the Near-Far constant of its bucket width, and whether the autotuner
 * picked them. */
b2_status b2_server_graph_config(b2_server s, int32_t graph_id, int32_t* cluster_team, double* delta_scale,
                                 int32_t* tuned);
/* Arena bytes one query on an n-vertex graph holds while it runs. */
size_t b2_server_slot_bytes(int64_t n, int32_t with_pred);
b2_status b2_server_submit(b2_server s, int32_t graph_id, uint32_t source, void* out_dist,
                           int32_t* out_pred, uint64_t* ticket);
/* A pending query completes with B2_CANCELLED; a running one is never
 * interrupted (B2_NOT_SUPPORTED). */
b2_status b2_server_cancel(b2_server s, uint64_t ticket);
/* Admit and launch what fits, collect finished queries; wait_all = 1 keeps
 * going until nothing is pending or running. */
b2_status b2_server_progress(b2_server s, int32_t wait_all);
b2_status b2_server_poll(b2_server s, b2_completion* out, int32_t capacity, int32_t* count);
b2_status b2_server_info(b2_server s, b2_server_info_t* info);

/* Built-in load generator over the server's graphs. */
typedef struct b2_load_opts {
  int64_t queries;
  double rate_qps;          /* Poisson arrival rate; <= 0: every query arrives at t = 0 */
  uint64_t seed;
  int32_t mode;             /* 0: this server; 1: one query at a time with b2_sssp_delta
                               on the whole GPU plus a device-to-host copy (baseline) */
  int32_t with_pred;
  size_t host_result_bytes; /* page-locked result pool (default 1 GiB); back-pressure when full */
  const int32_t* graph_ids; /* queries pick uniformly among these (NULL: all graphs) */
  int32_t n_graph_ids;
  int32_t reserved0;
  uint64_t* checksums;      /* nullable [queries]: 64-bit hash of each result's distance words */
  int32_t* query_graph;     /* nullable [queries]: graph of each query */
  uint32_t* query_source;   /* nullable [queries]: source of each query */
  int32_t reserved[4];
} b2_load_opts;
typedef struct b2_load_report {
  int64_t completed;
  int64_t failed;
  double elapsed_s;         /* first arrival -> last result in host memory */
  double qps;
  double p50_us;            /* latency: scheduled arrival -> result in host memory */
  double p99_us;
  double mean_us;
  double max_us;
  double gteps;             /* sum of reached out-edges / elapsed */
  uint64_t reached_edges;
  double reserved[4];
} b2_load_report;
void b2_load_opts_default(b2_load_opts* opts);
b2_status b2_server_run_load(b2_server s, const b2_load_opts* opts, b2_load_report* report);

/* ---- synthetic graphs (host memory, deterministic, multi-threaded) ----- */
typedef struct b2_host_csr {
  int64_t n;
  int64_t m;
  int64_t* rowptr;   /* n+1 */
  int32_t* colind;   /* m  */
  uint32_t* weights; /* m  (uint32 weights) */
  float* fweights;   /* m  (float variant, same law scaled to [0,1)) */
} b2_host_csr;

/* Outgoing CSR, columns sorted within each row, no self-loops or duplicates. */
b2_status b2_gen_er(int64_t n, int64_t m, uint32_t wmin, uint32_t wmax, uint64_t seed,
                    b2_host_csr* out);
b2_status b2_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                      uint32_t wmin, uint32_t wmax, uint64_t seed, b2_host_csr* out);
b2_status b2_gen_grid(int32_t rows, int32_t cols, double shortcut_frac, double mu,
                      double sigma, uint64_t seed, b2_host_csr* out);
void b2_host_csr_free(b2_host_csr* g);
/* Incoming <-> outgoing (stable: rows list columns in increasing order). */
b2_status b2_host_csr_transpose(const b2_host_csr* in, b2_host_csr* out);

/* RIPSCSR1 .csrbin (incoming CSR, float weights). */
b2_status b2_csrbin_write(const char* path, int64_t n, int64_t nnz, const int64_t* rowptr,
                          const int32_t* colind, const float* values);
b2_status b2_csrbin_read(const char* path, b2_host_csr* out);

/* DIMACS shortest-path text graph (.gr: "c" comments, "p <kind> n m", "a u v w" with 1-based
 * ids) as an INCOMING CSR with float weights, read under the rules of the reference's converter
 * (HIP_kernel/bellman_ford/src/gr_to_csr.cpp:124-230): columns ascending in each row, repeated
 * arcs reduced to their smallest weight, self-loops kept, unknown line kinds ignored.  Errors:
 * B2_INVALID_ARGUMENT (unreadable file, bad or missing problem line, arc before it, malformed
 * arc), B2_INVALID_INDEX (endpoint outside [1, n]), B2_INVALID_WEIGHT (non-finite weight).
 * declared_arcs / loaded_arcs (nullable): the problem line's m and the arc lines read. */
b2_status b2_dimacs_read(const char* path, b2_host_csr* out, int64_t* declared_arcs, int64_t* loaded_arcs);
/* The reference converter in one call (gr_to_csr.cpp:232-326): DIMACS .gr -> RIPSCSR1 .csrbin,
 * byte-identical to its output.  nnz_out (nullable): arcs after duplicate reduction. */
b2_status b2_dimacs_to_csrbin(const char* gr_path, const char* csrbin_path, int64_t* nnz_out);
/* Galois / Lonestar binary .gr, version 1, as the ADDS port loads it
 * (HIP_kernel/faster_GPU_algo/Charlotte_ADS_Float_Attempt/csr_graph.cpp:153-291): OUTGOING CSR;
 * no edge data = weight 1; 4-byte edge data are floats when data_is_float (the port's reading:
 * finite and >= 0 required, else B2_INVALID_WEIGHT) or uint32 otherwise.  Bad header or
 * truncated file: B2_INVALID_ARGUMENT; offsets not monotone / not ending at m:
 * B2_INVALID_ROWPTR; destination >= n: B2_INVALID_INDEX. */
b2_status b2_lonestar_read(const char* path, int32_t data_is_float, b2_host_csr* out);
/* Write an OUTGOING CSR as Lonestar .gr version 1 with 4-byte edge data (fweights when
 * data_is_float, else weights). */
b2_status b2_lonestar_write(const char* path, const b2_host_csr* g, int32_t data_is_float);

#ifdef __cplusplus
}
#endif
#endif /* B200SSSP_H_ */
