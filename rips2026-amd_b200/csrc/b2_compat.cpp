// The reference's C++ entry points (include/b200sssp/compat.hpp) on top of
// the C ABI.  Argument checks and error conventions follow the reference:
//   bf_hip_CSR.cpp:29-149, bf_hip_no_checks_CSR.cpp:29-93, bf_var_checks.cpp:43-188,
//   bellman_ford_hip.cpp:64-264, delta_stepping_hip_CSR.cpp:142-185 and 648-815,
//   Charlotte_oneshot/sssp_hip.cpp:25-81 and 350-595,
//   jasper_oneshot_untested/hip_adds_sssp.cpp:1138-1301,
//   minplus_hip.cpp:122-173, minplus_sparse_hip.cpp:410-813.
// The solves themselves run in one persistent launch each; progress callbacks
// are called from the calling thread while the kernel runs (b2_progress).
#include "../../include/b200sssp/compat.hpp"

#include <chrono>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>

#include "../../include/b200sssp.h"

namespace {

void throw_status(b2_status s, const std::string& what) {
  if (s == B2_SUCCESS) return;
  const std::string msg = what + ": " + b2_status_string(s);
  switch (s) {
    case B2_INVALID_ARGUMENT:
    case B2_INVALID_INDEX:
    case B2_INVALID_ROWPTR:
    case B2_INVALID_WEIGHT:
      throw std::invalid_argument(msg);
    case B2_NOT_SUPPORTED:
      throw std::overflow_error(msg);
    default:
      throw std::runtime_error(msg);
  }
}

struct GraphGuard {
  b2_graph g = nullptr;
  ~GraphGuard() {
    if (g) b2_graph_destroy(g);
  }
};

template <typename T>
struct DevArray {
  T* p = nullptr;
  explicit DevArray(size_t n) {
    if (cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess)
      throw std::runtime_error("cudaMalloc failed");
  }
  ~DevArray() {
    if (p) cudaFree(p);
  }
};

std::vector<float> to_host(const float* d, size_t n, cudaStream_t st) {
  std::vector<float> h(n);
  if (cudaMemcpyAsync(h.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    throw std::runtime_error("copy distances to host failed");
  return h;
}

void check_shape(minplus_sparse::Offset rows, minplus_sparse::Offset cols, minplus_sparse::Offset nnz, int source) {
  if (rows <= 0) throw std::invalid_argument("CSR graph must contain at least one vertex");
  if (rows != cols) throw std::invalid_argument("SSSP expects a square CSR adjacency matrix");
  if (nnz < 0) throw std::invalid_argument("CSR nnz must be nonnegative");
  if (source < 0 || source >= rows) throw std::out_of_range("source vertex is outside CSR row range");
  if (rows > std::numeric_limits<int>::max())
    throw std::overflow_error("frontier vertices are stored as int; rows must fit in int");
}

b2_graph incoming_graph(const minplus_sparse::DeviceCsrF32& a, int source, cudaStream_t st) {
  check_shape(a.rows, a.cols, a.nnz, source);
  if (a.rowptr == nullptr) throw std::invalid_argument("device CSR rowptr is null");
  if (a.nnz > 0 && (a.colind == nullptr || a.values == nullptr))
    throw std::invalid_argument("device CSR colind/values are null for a nonempty graph");
  b2_csr csr = {a.rows, a.cols, a.nnz, a.rowptr, a.colind, a.values, 64, B2_W_F32, B2_INCOMING, 1};
  b2_graph g = nullptr;
  throw_status(b2_graph_create(&csr, st, &g), "invalid device CSR");
  return g;
}

b2_graph incoming_graph(const HostCsrF32& h, int source, cudaStream_t st) {
  check_shape(h.rows, h.cols, h.nnz, source);
  const size_t rows = (size_t)h.rows, nnz = (size_t)h.nnz;
  if (h.rowptr.size() != rows + 1) throw std::invalid_argument("rowptr.size() must equal rows + 1");
  if (h.colind.size() != nnz) throw std::invalid_argument("colind.size() must equal nnz");
  if (h.values.size() != nnz) throw std::invalid_argument("values.size() must equal nnz");
  b2_csr csr = {h.rows, h.cols, h.nnz, h.rowptr.data(), h.colind.data(), h.values.data(), 64, B2_W_F32,
                B2_INCOMING, 0};
  b2_graph g = nullptr;
  throw_status(b2_graph_create(&csr, st, &g), "invalid host CSR");
  return g;
}

// Live progress: the C ABI calls this bridge from the calling thread while
// the persistent kernel runs (one call per finished round / bucket, in
// order); it forwards each call in the reference's callback form.  Rounds
// the reference would still run after the kernel has converged (no-checks
// and var-checks loops) change nothing and are reported after the solve.
struct Bridge {
  enum Kind { kChecked, kNoChecks, kVarChecks, kDelta };
  BellmanFordCsrProgressCallback cb = nullptr;
  void* ud = nullptr;
  Kind kind = kChecked;
  int interval = 1;
  int max_iters = 0;
  int reported = 0;

  void emit(int iteration, bool changed) {
    BellmanFordCsrProgress q;
    q.iteration = iteration;
    q.max_iters = max_iters;
    switch (kind) {
      case kNoChecks:
        q.convergence_checked = false;
        q.changed = false;
        break;
      case kVarChecks:
        q.convergence_checked = (iteration % interval) == 0;
        q.changed = q.convergence_checked && changed;
        break;
      default:
        q.convergence_checked = true;
        q.changed = changed;
    }
    cb(q, ud);
    reported = iteration;
  }
  void finish(int total) {   // rounds after the kernel converged: nothing changes
    if (cb)
      while (reported < total) emit(reported + 1, false);
  }
};

extern "C" void compat_progress_bridge(const b2_progress* p, void* user) {
  static_cast<Bridge*>(user)->emit(p->iteration, p->changed != 0);
}

struct BfRun {
  std::vector<float> dist;
  b2_stats st{};
  int max_iters = 0;
  double kernel_ms = 0, init_ms = 0, copy_ms = 0;
  std::vector<double> round_end_ms;   // device time at the end of each round (traced solves)
};

BfRun run_bf(b2_graph g, int n, int source, int max_iters, cudaStream_t stream, Bridge* bridge, bool trace) {
  using clk = std::chrono::steady_clock;
  BfRun r;
  r.max_iters = max_iters < 0 ? n - 1 : max_iters;
  const auto t0 = clk::now();
  DevArray<float> d((size_t)n);
  const auto t1 = clk::now();
  b2_sssp_opts o;
  b2_sssp_opts_default(&o);
  o.max_iters = r.max_iters;
  o.trace = trace ? 1 : 0;
  if (bridge && bridge->cb) {
    bridge->max_iters = r.max_iters;
    o.progress = compat_progress_bridge;
    o.progress_user = bridge;
  }
  throw_status(b2_sssp_bf(g, (uint32_t)source, d.p, nullptr, &o, stream, &r.st), "bellman-ford");
  const auto t2 = clk::now();
  r.dist = to_host(d.p, (size_t)n, stream);
  const auto t3 = clk::now();
  r.init_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  r.kernel_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
  r.copy_ms = std::chrono::duration<double, std::milli>(t3 - t2).count();
  if (trace) {
    std::vector<b2_trace_entry> tr(4096);
    int32_t cnt = 0;
    if (b2_graph_trace(g, tr.data(), (int32_t)tr.size(), &cnt) == B2_SUCCESS) {
      // the phases of round i carry bucket == i; its end is its last phase's end
      for (int32_t k = 0; k < cnt; ++k) {
        const uint32_t round = tr[k].bucket;
        if (round == 0 || round > (uint32_t)r.max_iters) continue;
        if (r.round_end_ms.size() < round) r.round_end_ms.resize(round, 0.0);
        r.round_end_ms[round - 1] = std::max(r.round_end_ms[round - 1], (double)tr[k].t_ns * 1e-6);
      }
    }
  }
  return r;
}

// Round i changed something iff i precedes the first unchanged round.
bool round_changed(const b2_stats& st, int i) {
  return st.first_unchanged == 0 || (uint32_t)i < st.first_unchanged;
}

BellmanFordCsrResult bf_checked(b2_graph g, int n, int source, int max_iters, cudaStream_t stream,
                                BellmanFordCsrProgressCallback cb, void* ud) {
  Bridge br;
  br.cb = cb;
  br.ud = ud;
  br.kind = Bridge::kChecked;
  BfRun r = run_bf(g, n, source, max_iters, stream, &br, false);
  BellmanFordCsrResult res;
  res.dist = std::move(r.dist);
  res.iterations_used = r.st.iterations_used;
  res.converged = r.st.converged != 0;
  br.finish(res.iterations_used);
  return res;
}

BellmanFordCsrNoChecksResult bf_no_checks(b2_graph g, int n, int source, int max_iters, cudaStream_t stream,
                                          BellmanFordCsrProgressCallback cb, void* ud) {
  Bridge br;
  br.cb = cb;
  br.ud = ud;
  br.kind = Bridge::kNoChecks;
  BfRun r = run_bf(g, n, source, max_iters, stream, &br, false);
  BellmanFordCsrNoChecksResult res;
  res.dist = std::move(r.dist);
  res.iterations_used = r.max_iters;   // rounds after convergence change nothing
  br.finish(r.max_iters);
  return res;
}

BellmanFordCsrVarChecksResult bf_var_checks(b2_graph g, int n, int source, int max_iters, int check_interval,
                                            cudaStream_t stream, BellmanFordCsrProgressCallback cb, void* ud) {
  if (check_interval <= 0) throw std::invalid_argument("check_interval must be positive");
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  Bridge br;
  br.cb = cb;
  br.ud = ud;
  br.kind = Bridge::kVarChecks;
  br.interval = check_interval;
  BfRun r = run_bf(g, n, source, max_iters, stream, &br, true);
  BellmanFordCsrVarChecksResult res;
  res.dist = std::move(r.dist);
  res.check_interval = check_interval;
  // convergence is observed at the first checked round at or after the first
  // unchanged round (bf_var_checks.cpp:79-160)
  const long long k = r.st.first_unchanged ? (long long)r.st.first_unchanged : -1;
  long long seen = -1;
  if (k > 0) seen = ((k + check_interval - 1) / check_interval) * (long long)check_interval;
  if (seen > 0 && seen <= r.max_iters) {
    res.iterations_used = (int)seen;
    res.converged = true;
  } else {
    res.iterations_used = r.max_iters;
    res.converged = false;
  }
  res.checks_performed = res.iterations_used / check_interval;
  for (int i = check_interval; i <= res.iterations_used; i += check_interval) {
    if (round_changed(r.st, i)) ++res.changed_checks;
    else ++res.unchanged_checks;
  }
  res.initialization_ms = r.init_ms;
  res.relaxation_ms = r.st.kernel_ms;
  res.bellman_ford_loop_ms = r.kernel_ms;
  // checked / unchecked round time from the kernel's own per-phase clock
  // (bf_var_checks.cpp:70-186 times them on the host); rounds the kernel did
  // not run (after convergence) took no time
  double checked = 0.0, unchecked = 0.0, prev = 0.0;
  for (size_t i = 0; i < r.round_end_ms.size(); ++i) {
    const double end = std::max(prev, r.round_end_ms[i]);
    const double dur = end - prev;
    prev = end;
    if ((int)(i + 1) > res.iterations_used) break;
    if ((int)(i + 1) % check_interval == 0) checked += dur;
    else unchecked += dur;
  }
  if (r.round_end_ms.empty()) unchecked = r.st.kernel_ms;
  res.checked_iteration_ms = checked;
  res.unchecked_iteration_ms = unchecked;
  res.final_copy_ms = r.copy_ms;
  res.estimated_check_overhead_ms = 0.0;   // change detection is free on the device
  res.total_runtime_ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  br.finish(res.iterations_used);
  return res;
}

BellmanFordCsrResult var_to_plain(BellmanFordCsrVarChecksResult&& v) {
  BellmanFordCsrResult r;
  r.dist = std::move(v.dist);
  r.iterations_used = v.iterations_used;
  r.converged = v.converged;
  return r;
}

void validate_delta(float delta) {
  if (!(delta > 0.0f) || !std::isfinite(delta)) throw std::invalid_argument("delta must be a finite positive float");
}

DeltaSteppingCsrResult delta_run(b2_graph g, int n, int source, float delta, int max_iters, cudaStream_t stream,
                                 DeltaSteppingCsrProgressCallback cb, void* ud) {
  DevArray<float> d((size_t)n);
  b2_sssp_opts o;
  b2_sssp_opts_default(&o);
  o.delta = (double)delta;
  o.max_iters = max_iters;   // < 0: unbounded (delta_stepping_hip_CSR.cpp:666)
  o.light_heavy = 1;
  Bridge br;
  br.cb = cb;
  br.ud = ud;
  br.kind = Bridge::kDelta;
  br.max_iters = max_iters < 0 ? std::numeric_limits<int>::max() : max_iters;
  if (cb) {
    o.progress = compat_progress_bridge;
    o.progress_user = &br;
  }
  b2_stats st;
  const b2_status s = b2_sssp_delta(g, (uint32_t)source, d.p, nullptr, &o, stream, &st);
  if (s == B2_INVALID_WEIGHT)
    throw std::invalid_argument("invalid device CSR: rowptr/colind must be in range and weights finite nonnegative");
  throw_status(s, "delta-stepping");
  DeltaSteppingCsrResult res;
  res.dist = to_host(d.p, (size_t)n, stream);
  res.iterations_used = st.iterations_used;
  res.converged = st.converged != 0;
  return res;
}

// ---- oneshot helpers (sssp_hip.cpp:25-81)
void validate_graph(const CsrGraph& g, bool nonneg) {
  if (g.num_nodes <= 0) throw std::invalid_argument("graph must contain at least one node");
  if (g.num_edges < 0) throw std::invalid_argument("num_edges must be nonnegative");
  if ((int)g.row_offsets.size() != g.num_nodes + 1)
    throw std::invalid_argument("row_offsets must contain num_nodes + 1 entries");
  if (g.row_offsets.front() != 0 || g.row_offsets.back() != g.num_edges)
    throw std::invalid_argument("row_offsets must start at 0 and end at num_edges");
  if ((int)g.col_indices.size() != g.num_edges || (int)g.weights.size() != g.num_edges)
    throw std::invalid_argument("col_indices and weights must contain num_edges entries");
  for (int u = 0; u < g.num_nodes; ++u)
    if (g.row_offsets[u] > g.row_offsets[u + 1]) throw std::invalid_argument("row_offsets must be nondecreasing");
  for (int e = 0; e < g.num_edges; ++e) {
    if (g.col_indices[e] < 0 || g.col_indices[e] >= g.num_nodes)
      throw std::invalid_argument("col_indices contains a vertex outside graph");
    if (std::isnan(g.weights[e]) || (nonneg && !(g.weights[e] >= 0.0f)))
      throw std::invalid_argument("ADDS / delta-stepping requires non-negative, non-NaN weights");
  }
}

b2_graph outgoing_graph(const CsrGraph& g, int source, cudaStream_t st) {
  if (source < 0 || source >= g.num_nodes) throw std::invalid_argument("source is outside graph");
  // 32-bit offsets are read as uint32 (valid: validated nonnegative and monotone)
  b2_csr csr = {g.num_nodes, g.num_nodes, g.num_edges, g.row_offsets.data(), g.col_indices.data(),
                g.weights.data(), 32, B2_W_F32, B2_OUTGOING, 0};
  b2_graph h = nullptr;
  throw_status(b2_graph_create(&csr, st, &h), "invalid graph");
  return h;
}

cudaError_t to_cuda(b2_status s) {
  switch (s) {
    case B2_SUCCESS: return cudaSuccess;
    case B2_OUT_OF_MEMORY: return cudaErrorMemoryAllocation;
    case B2_CUDA_ERROR: return cudaErrorLaunchFailure;
    case B2_INVALID_ARGUMENT:
    case B2_INVALID_INDEX:
    case B2_INVALID_ROWPTR:
    case B2_INVALID_WEIGHT:
    case B2_NOT_SUPPORTED:
      return cudaErrorInvalidValue;
    default:
      return cudaErrorUnknown;
  }
}

}  // namespace

// ============================================================== min-plus
cudaError_t minplus_gemm_f32(const float* d_A, const float* d_B, float* d_C, int M, int N, int K, int lda, int ldb,
                             int ldc, cudaStream_t stream) {
  return to_cuda(b2_minplus_gemm_f32(d_A, d_B, d_C, M, N, K, lda, ldb, ldc, stream));
}

namespace minplus_sparse {

namespace {
cudaError_t spgemm(const DeviceCsrF32& A, const DeviceCsrF32& B, Offset** rp, Index** ci, float** v, Offset* nnz,
                   cudaStream_t stream) {
  if (!rp || !ci || !v || !nnz) return cudaErrorInvalidValue;
  b2_csr a = {A.rows, A.cols, A.nnz, A.rowptr, A.colind, A.values, 64, B2_W_F32, B2_OUTGOING, 1};
  b2_csr b = {B.rows, B.cols, B.nnz, B.rowptr, B.colind, B.values, 64, B2_W_F32, B2_OUTGOING, 1};
  int64_t* crp = nullptr;
  int32_t* cci = nullptr;
  float* cv = nullptr;
  int64_t cn = 0;
  const b2_status s = b2_minplus_spgemm_f32(&a, &b, &crp, &cci, &cv, &cn, stream);
  *rp = crp;
  *ci = cci;
  *v = cv;
  *nnz = cn;
  return to_cuda(s);
}
}  // namespace

cudaError_t minplus_spgemm_csr_f32(const DeviceCsrF32& A, const DeviceCsrF32& B, Offset** d_C_rowptr,
                                   Index** d_C_colind, float** d_C_values, Offset* h_C_nnz, cudaStream_t stream) {
  return spgemm(A, B, d_C_rowptr, d_C_colind, d_C_values, h_C_nnz, stream);
}

cudaError_t minplus_spgemm_csr_f32_large_rows(const DeviceCsrF32& A, const DeviceCsrF32& B, Offset** d_C_rowptr,
                                              Index** d_C_colind, float** d_C_values, Offset* h_C_nnz,
                                              cudaStream_t stream) {
  return spgemm(A, B, d_C_rowptr, d_C_colind, d_C_values, h_C_nnz, stream);
}

template <int HASH_CAP, int BLOCK_SIZE>
cudaError_t minplus_spgemm_csr_f32_tuned(const DeviceCsrF32& A, const DeviceCsrF32& B, Offset** d_C_rowptr,
                                         Index** d_C_colind, float** d_C_values, Offset* h_C_nnz,
                                         cudaStream_t stream) {
  static_assert(HASH_CAP > 0 && (HASH_CAP & (HASH_CAP - 1)) == 0, "HASH_CAP must be a power of two");
  static_assert(BLOCK_SIZE > 0, "BLOCK_SIZE must be positive");
  return spgemm(A, B, d_C_rowptr, d_C_colind, d_C_values, h_C_nnz, stream);
}

template cudaError_t minplus_spgemm_csr_f32_tuned<256, 64>(const DeviceCsrF32&, const DeviceCsrF32&, Offset**,
                                                           Index**, float**, Offset*, cudaStream_t);
template cudaError_t minplus_spgemm_csr_f32_tuned<512, 64>(const DeviceCsrF32&, const DeviceCsrF32&, Offset**,
                                                           Index**, float**, Offset*, cudaStream_t);
template cudaError_t minplus_spgemm_csr_f32_tuned<1024, 128>(const DeviceCsrF32&, const DeviceCsrF32&, Offset**,
                                                             Index**, float**, Offset*, cudaStream_t);
template cudaError_t minplus_spgemm_csr_f32_tuned<2048, 128>(const DeviceCsrF32&, const DeviceCsrF32&, Offset**,
                                                             Index**, float**, Offset*, cudaStream_t);
template cudaError_t minplus_spgemm_csr_f32_tuned<4096, 256>(const DeviceCsrF32&, const DeviceCsrF32&, Offset**,
                                                             Index**, float**, Offset*, cudaStream_t);

}  // namespace minplus_sparse

// ============================================================== CSR BF
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                  int max_iters, cudaStream_t stream,
                                                  BellmanFordCsrProgressCallback cb, void* ud) {
  GraphGuard g{incoming_graph(d_adjacency, source, stream)};
  return bf_checked(g.g, (int)d_adjacency.rows, source, max_iters, stream, cb, ud);
}
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                  cudaStream_t stream) {
  return bellman_ford_minplus_hip_csr(d_adjacency, source, (int)d_adjacency.rows - 1, stream, nullptr, nullptr);
}
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const HostCsrF32& adjacency, int source, int max_iters,
                                                  cudaStream_t stream, BellmanFordCsrProgressCallback cb, void* ud) {
  GraphGuard g{incoming_graph(adjacency, source, stream)};
  return bf_checked(g.g, (int)adjacency.rows, source, max_iters, stream, cb, ud);
}
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const HostCsrF32& adjacency, int source, cudaStream_t stream) {
  return bellman_ford_minplus_hip_csr(adjacency, source, (int)adjacency.rows - 1, stream, nullptr, nullptr);
}

BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(const minplus_sparse::DeviceCsrF32& d_adjacency,
                                                                    int source, int max_iters, cudaStream_t stream,
                                                                    BellmanFordCsrProgressCallback cb, void* ud) {
  GraphGuard g{incoming_graph(d_adjacency, source, stream)};
  return bf_no_checks(g.g, (int)d_adjacency.rows, source, max_iters, stream, cb, ud);
}
BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(const minplus_sparse::DeviceCsrF32& d_adjacency,
                                                                    int source, cudaStream_t stream) {
  return bellman_ford_minplus_hip_csr_no_checks(d_adjacency, source, (int)d_adjacency.rows - 1, stream, nullptr,
                                                nullptr);
}
BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(const HostCsrF32& adjacency, int source,
                                                                    int max_iters, cudaStream_t stream,
                                                                    BellmanFordCsrProgressCallback cb, void* ud) {
  GraphGuard g{incoming_graph(adjacency, source, stream)};
  return bf_no_checks(g.g, (int)adjacency.rows, source, max_iters, stream, cb, ud);
}
BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(const HostCsrF32& adjacency, int source,
                                                                    cudaStream_t stream) {
  return bellman_ford_minplus_hip_csr_no_checks(adjacency, source, (int)adjacency.rows - 1, stream, nullptr, nullptr);
}

BellmanFordCsrVarChecksResult bellman_ford_minplus_hip_csr_var_checks_with_stats(
    const minplus_sparse::DeviceCsrF32& d_adjacency, int source, int max_iters, int check_interval,
    cudaStream_t stream, BellmanFordCsrProgressCallback cb, void* ud) {
  if (check_interval <= 0) throw std::invalid_argument("check_interval must be positive");
  GraphGuard g{incoming_graph(d_adjacency, source, stream)};
  return bf_var_checks(g.g, (int)d_adjacency.rows, source, max_iters, check_interval, stream, cb, ud);
}
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const minplus_sparse::DeviceCsrF32& d_adjacency,
                                                             int source, int max_iters, int check_interval,
                                                             cudaStream_t stream, BellmanFordCsrProgressCallback cb,
                                                             void* ud) {
  return var_to_plain(bellman_ford_minplus_hip_csr_var_checks_with_stats(d_adjacency, source, max_iters,
                                                                         check_interval, stream, cb, ud));
}
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const minplus_sparse::DeviceCsrF32& d_adjacency,
                                                             int source, int check_interval, cudaStream_t stream) {
  return bellman_ford_minplus_hip_csr_var_checks(d_adjacency, source, (int)d_adjacency.rows - 1, check_interval,
                                                 stream, nullptr, nullptr);
}
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const HostCsrF32& adjacency, int source, int max_iters,
                                                             int check_interval, cudaStream_t stream,
                                                             BellmanFordCsrProgressCallback cb, void* ud) {
  if (check_interval <= 0) throw std::invalid_argument("check_interval must be positive");
  GraphGuard g{incoming_graph(adjacency, source, stream)};
  return var_to_plain(bf_var_checks(g.g, (int)adjacency.rows, source, max_iters, check_interval, stream, cb, ud));
}
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const HostCsrF32& adjacency, int source,
                                                             int check_interval, cudaStream_t stream) {
  return bellman_ford_minplus_hip_csr_var_checks(adjacency, source, (int)adjacency.rows - 1, check_interval, stream,
                                                 nullptr, nullptr);
}

// ============================================================== dense BF
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source, int max_iters,
                                           cudaStream_t stream) {
  if (d_adjacency == nullptr) throw std::invalid_argument("d_adjacency must not be null");
  if (n <= 0) throw std::invalid_argument("n must be positive");
  if (source < 0 || source >= n) throw std::invalid_argument("source is outside graph");
  if (max_iters < 0) max_iters = n - 1;
  DevArray<float> d((size_t)n);
  b2_sssp_opts o;
  b2_sssp_opts_default(&o);
  o.max_iters = max_iters;
  b2_stats st;
  throw_status(b2_sssp_bf_dense(d_adjacency, n, (uint32_t)source, d.p, &o, stream, &st), "dense bellman-ford");
  BellmanFordResult r;
  r.dist = to_host(d.p, (size_t)n, stream);
  r.iterations_used = st.iterations_used;
  r.converged = st.converged != 0;
  return r;
}
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source, cudaStream_t stream) {
  return bellman_ford_minplus_hip(d_adjacency, n, source, n - 1, stream);
}
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source, int max_iters) {
  return bellman_ford_minplus_hip(d_adjacency, n, source, max_iters, nullptr);
}
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source) {
  return bellman_ford_minplus_hip(d_adjacency, n, source, n - 1, nullptr);
}
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source, int max_iters,
                                           cudaStream_t stream) {
  if (n <= 0) throw std::invalid_argument("n must be positive");
  const size_t expected = (size_t)n * (size_t)n;
  if (adjacency.size() != expected) throw std::invalid_argument("adjacency must contain n*n row-major values");
  DevArray<float> d(expected);
  if (cudaMemcpyAsync(d.p, adjacency.data(), expected * sizeof(float), cudaMemcpyHostToDevice, stream) != cudaSuccess)
    throw std::runtime_error("copy adjacency to device failed");
  return bellman_ford_minplus_hip(d.p, n, source, max_iters, stream);
}
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source,
                                           cudaStream_t stream) {
  return bellman_ford_minplus_hip(adjacency, n, source, n - 1, stream);
}
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source, int max_iters) {
  return bellman_ford_minplus_hip(adjacency, n, source, max_iters, nullptr);
}
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source) {
  return bellman_ford_minplus_hip(adjacency, n, source, n - 1, nullptr);
}

// ============================================================== delta-stepping
DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                      float delta, int max_iters, cudaStream_t stream,
                                                      DeltaSteppingCsrProgressCallback cb, void* ud) {
  check_shape(d_adjacency.rows, d_adjacency.cols, d_adjacency.nnz, source);
  validate_delta(delta);
  GraphGuard g{incoming_graph(d_adjacency, source, stream)};
  return delta_run(g.g, (int)d_adjacency.rows, source, delta, max_iters, stream, cb, ud);
}
DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                      float delta, cudaStream_t stream) {
  return delta_stepping_minplus_hip_csr(d_adjacency, source, delta, -1, stream, nullptr, nullptr);
}
DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const HostCsrF32& adjacency, int source, float delta,
                                                      int max_iters, cudaStream_t stream,
                                                      DeltaSteppingCsrProgressCallback cb, void* ud) {
  check_shape(adjacency.rows, adjacency.cols, adjacency.nnz, source);
  validate_delta(delta);
  for (float w : adjacency.values)
    if (!std::isfinite(w) || w < 0.0f)
      throw std::invalid_argument("delta-stepping requires finite nonnegative edge weights");
  GraphGuard g{incoming_graph(adjacency, source, stream)};
  return delta_run(g.g, (int)adjacency.rows, source, delta, max_iters, stream, cb, ud);
}
DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const HostCsrF32& adjacency, int source, float delta,
                                                      cudaStream_t stream) {
  return delta_stepping_minplus_hip_csr(adjacency, source, delta, -1, stream, nullptr, nullptr);
}

// ============================================================== oneshot
CsrGraph dense_to_csr_outgoing(const std::vector<float>& adjacency, int n) {
  if (n <= 0) throw std::invalid_argument("n must be positive");
  if (adjacency.size() != (size_t)n * (size_t)n)
    throw std::invalid_argument("adjacency must contain n*n row-major values");
  CsrGraph g;
  g.num_nodes = n;
  g.row_offsets.assign((size_t)n + 1, 0);
  for (int u = 0; u < n; ++u) {
    for (int v = 0; v < n; ++v) {
      const float w = adjacency[(size_t)u * n + v];
      if (std::isfinite(w)) {
        g.col_indices.push_back(v);
        g.weights.push_back(w);
      }
    }
    g.row_offsets[(size_t)u + 1] = (int)g.col_indices.size();
  }
  g.num_edges = (int)g.col_indices.size();
  return g;
}

SSSPResult bellman_ford_sssp_hip(const CsrGraph& graph, int source, const SSSPOptions& options,
                                 cudaStream_t stream) {
  validate_graph(graph, false);
  GraphGuard g{outgoing_graph(graph, source, stream)};
  DevArray<float> d((size_t)graph.num_nodes);
  b2_sssp_opts o;
  b2_sssp_opts_default(&o);
  o.max_iters = options.max_iters <= 0 ? graph.num_nodes - 1 : options.max_iters;
  o.detect_negative_cycle = 1;   // bf_detect_negative_like_change_kernel (sssp_hip.cpp:204-220)
  b2_stats st;
  throw_status(b2_sssp_bf(g.g, (uint32_t)source, d.p, nullptr, &o, stream, &st), "bellman-ford");
  SSSPResult r;
  r.dist = to_host(d.p, (size_t)graph.num_nodes, stream);
  r.iterations_used = st.iterations_used;
  r.converged = st.converged != 0;
  r.has_negative_cycle = st.has_negative_cycle != 0;
  r.work_count = st.edges_scanned;
  r.milliseconds = st.kernel_ms;
  return r;
}

SSSPResult adds_sssp_hip(const CsrGraph& graph, int source, const SSSPOptions& options, cudaStream_t stream) {
  validate_graph(graph, true);
  GraphGuard g{outgoing_graph(graph, source, stream)};
  DevArray<float> d((size_t)graph.num_nodes);
  b2_sssp_opts o;
  b2_sssp_opts_default(&o);
  o.max_iters = options.max_iters <= 0 ? -1 : options.max_iters;
  o.delta = (options.initial_delta > 0.0f && std::isfinite(options.initial_delta)) ? options.initial_delta : 0.0;
  b2_stats st;
  const b2_status s = options.dynamic_delta ? b2_sssp_adds(g.g, (uint32_t)source, d.p, nullptr, &o, stream, &st)
                                            : b2_sssp_delta(g.g, (uint32_t)source, d.p, nullptr, &o, stream, &st);
  throw_status(s, "adds");
  SSSPResult r;
  r.dist = to_host(d.p, (size_t)graph.num_nodes, stream);
  r.iterations_used = st.iterations_used;
  r.converged = st.converged != 0;
  r.has_negative_cycle = false;
  r.work_count = st.edges_scanned;
  r.milliseconds = st.kernel_ms;
  r.final_delta = (float)st.delta_final;
  return r;
}

SSSPResult bellman_ford_sssp_hip(const std::vector<float>& adjacency, int n, int source, const SSSPOptions& options,
                                 cudaStream_t stream) {
  return bellman_ford_sssp_hip(dense_to_csr_outgoing(adjacency, n), source, options, stream);
}

SSSPResult adds_sssp_hip(const std::vector<float>& adjacency, int n, int source, const SSSPOptions& options,
                         cudaStream_t stream) {
  return adds_sssp_hip(dense_to_csr_outgoing(adjacency, n), source, options, stream);
}

// ============================================================== hip_adds
namespace hip_adds {

const char* status_string(Status status) {
  switch (status) {
    case Status::Success: return "success";
    case Status::InvalidArgument: return "invalid argument";
    case Status::HipError: return "CUDA runtime error";
    case Status::OutOfMemory: return "out of device memory";
    case Status::PoolExhausted: return "worklist pool exhausted";
    case Status::BucketOverflow: return "bucket overflow";
    case Status::DeviceError: return "device error";
    case Status::Timeout: return "bounded device wait timed out";
  }
  return "unknown status";
}

namespace {
Status map_status(b2_status s) {
  switch (s) {
    case B2_SUCCESS: return Status::Success;
    case B2_OUT_OF_MEMORY: return Status::OutOfMemory;
    case B2_POOL_EXHAUSTED: return Status::PoolExhausted;
    case B2_BUCKET_OVERFLOW: return Status::BucketOverflow;
    case B2_CUDA_ERROR: return Status::HipError;
    case B2_TIMEOUT: return Status::Timeout;
    case B2_DEVICE_ERROR: return Status::DeviceError;
    default: return Status::InvalidArgument;
  }
}

template <typename Weight>
Status run(const DeviceCsrGraph<Weight>& graph, uint32_t source, Weight* d_distances, RunStats* stats,
           const Options& options, cudaStream_t stream, int wt) {
  if (graph.num_vertices == 0 || source >= graph.num_vertices || d_distances == nullptr) return Status::InvalidArgument;
  if (!graph.row_offsets || (graph.num_edges && (!graph.col_indices || !graph.weights))) return Status::InvalidArgument;
  b2_csr csr = {graph.num_vertices, graph.num_vertices, graph.num_edges, graph.row_offsets,
                reinterpret_cast<const int32_t*>(graph.col_indices), graph.weights, 32, wt, B2_OUTGOING, 1};
  b2_graph g = nullptr;
  b2_status s = b2_graph_create(&csr, stream, &g);
  if (s != B2_SUCCESS) return map_status(s);
  b2_sssp_opts o;
  b2_sssp_opts_default(&o);
  if (options.initial_delta > 0.0) o.delta = options.initial_delta;
  o.delta_scale = options.initial_delta_scale;
  o.keep_distances = options.initialize_distances ? 0 : 1;   // warm start (hip_adds_sssp.hpp:64-66)
  o.adds_fixed_delta = options.dynamic_delta ? 0 : 1;
  o.active_buckets = options.initial_active_buckets;
  o.max_active_buckets = options.dynamic_active_buckets ? options.max_active_buckets
                                                        : std::max<uint32_t>(1u, options.initial_active_buckets);
  if (options.worker_blocks) o.grid_blocks = options.worker_blocks;
  // pool_words is the reference's whole worklist pool; here each of the
  // window queues and far piles holds an equal share
  if (options.pool_words) o.worklist_capacity = (uint32_t)std::min<size_t>(std::max<size_t>(options.pool_words / 34, 1),
                                                                            0xFFFFFFFFull);
  b2_stats st;
  s = b2_sssp_adds(g, source, d_distances, nullptr, &o, stream, &st);
  b2_graph_destroy(g);
  if (stats) {
    *stats = RunStats();
    stats->initial_delta = st.delta_used;
    stats->final_delta = st.delta_final;
    stats->worker_blocks = st.grid_blocks;
    stats->final_active_buckets = st.active_buckets_max;
    stats->device_error = st.device_error;
    stats->assigned_items = st.work_items;
    stats->processed_items = st.work_items;
    stats->enqueued_items = st.pushes + 1;   // + the source
    stats->edge_relaxations = st.edges_scanned;
    stats->successful_relaxations = st.improvements;
    stats->head_switches = (uint64_t)st.iterations_used;
    stats->delta_updates = st.delta_updates;
  }
  return map_status(s);
}
}  // namespace

Status sssp(const DeviceCsrGraph<float>& graph, uint32_t source, float* d_distances, RunStats* stats,
            const Options& options, cudaStream_t stream) {
  return run<float>(graph, source, d_distances, stats, options, stream, B2_W_F32);
}

Status sssp(const DeviceCsrGraph<uint32_t>& graph, uint32_t source, uint32_t* d_distances, RunStats* stats,
            const Options& options, cudaStream_t stream) {
  return run<uint32_t>(graph, source, d_distances, stats, options, stream, B2_W_U32);
}

}  // namespace hip_adds
