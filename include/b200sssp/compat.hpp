// Drop-in C++ surface: the reference's types and entry points, implemented
// by libb200sssp.so on the B200 (hipStream_t becomes cudaStream_t, hipError_t
// becomes cudaError_t; every other name, argument and result field is kept).
//
// Reference headers mirrored (charlottesylvie/rips2026-amd):
//   HIP_kernel/minplus_mm/src/minplus_sparse_hip.hpp:9-150
//   HIP_kernel/minplus_mm/src/minplus_hip.hpp:24-33
//   HIP_kernel/bellman_ford/src/bf_hip_CSR.hpp:9-66
//   HIP_kernel/bellman_ford/src/bf_hip_no_checks_CSR.hpp:9-42
//   HIP_kernel/bellman_ford/src/bf_var_checks.hpp:9-71
//   HIP_kernel/bellman_ford/src/bellman_ford_hip.hpp:8-60
//   HIP_kernel/delta_stepping/src/delta_stepping_hip_CSR.hpp:10-67
//   HIP_kernel/faster_GPU_algo/Charlotte_oneshot/sssp_hip.hpp:8-78
//   HIP_kernel/faster_GPU_algo/jasper_oneshot_untested/hip_adds_sssp.hpp:9-113
//
// Error conventions are the reference's: the Bellman-Ford, delta-stepping
// and oneshot functions throw std::invalid_argument / std::out_of_range /
// std::overflow_error / std::runtime_error; the min-plus functions return an
// error code; hip_adds::sssp returns a Status.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <vector>

// ---------------------------------------------------------------- min-plus
namespace minplus_sparse {

using Offset = std::int64_t;
using Index = int;

inline constexpr int kDefaultHashCapacity = 512;
inline constexpr int kDefaultBlockSize = 64;
inline constexpr int kLargeHashCapacity = 4096;
inline constexpr int kLargeBlockSize = 256;

struct DeviceCsrF32 {
  Offset rows;
  Offset cols;
  Offset nnz;
  const Offset* rowptr;
  const Index* colind;
  const float* values;
};

// C = A min-plus B.  Outputs are device allocations owned by the caller
// (cudaFree).  Columns within a row come out sorted; rows have no size limit
// (HASH_CAP / BLOCK_SIZE of the tuned variants are accepted for source
// compatibility and do not limit the result).
cudaError_t minplus_spgemm_csr_f32(const DeviceCsrF32& A, const DeviceCsrF32& B, Offset** d_C_rowptr,
                                   Index** d_C_colind, float** d_C_values, Offset* h_C_nnz,
                                   cudaStream_t stream = 0);
cudaError_t minplus_spgemm_csr_f32_large_rows(const DeviceCsrF32& A, const DeviceCsrF32& B, Offset** d_C_rowptr,
                                              Index** d_C_colind, float** d_C_values, Offset* h_C_nnz,
                                              cudaStream_t stream = 0);
template <int HASH_CAP, int BLOCK_SIZE>
cudaError_t minplus_spgemm_csr_f32_tuned(const DeviceCsrF32& A, const DeviceCsrF32& B, Offset** d_C_rowptr,
                                         Index** d_C_colind, float** d_C_values, Offset* h_C_nnz,
                                         cudaStream_t stream = 0);

extern template cudaError_t minplus_spgemm_csr_f32_tuned<256, 64>(const DeviceCsrF32&, const DeviceCsrF32&,
                                                                  Offset**, Index**, float**, Offset*, cudaStream_t);
extern template cudaError_t minplus_spgemm_csr_f32_tuned<512, 64>(const DeviceCsrF32&, const DeviceCsrF32&,
                                                                  Offset**, Index**, float**, Offset*, cudaStream_t);
extern template cudaError_t minplus_spgemm_csr_f32_tuned<1024, 128>(const DeviceCsrF32&, const DeviceCsrF32&,
                                                                    Offset**, Index**, float**, Offset*, cudaStream_t);
extern template cudaError_t minplus_spgemm_csr_f32_tuned<2048, 128>(const DeviceCsrF32&, const DeviceCsrF32&,
                                                                    Offset**, Index**, float**, Offset*, cudaStream_t);
extern template cudaError_t minplus_spgemm_csr_f32_tuned<4096, 256>(const DeviceCsrF32&, const DeviceCsrF32&,
                                                                    Offset**, Index**, float**, Offset*, cudaStream_t);

}  // namespace minplus_sparse

// C[i,j] = min_k A[i,k] + B[k,j], row-major; asynchronous on `stream`.
cudaError_t minplus_gemm_f32(const float* d_A, const float* d_B, float* d_C, int M, int N, int K, int lda, int ldb,
                             int ldc, cudaStream_t stream = nullptr);

// ---------------------------------------------------------------- CSR BF
struct BellmanFordCsrProgress {
  int iteration = 0;
  int max_iters = 0;
  bool convergence_checked = false;
  bool changed = false;
};

using BellmanFordCsrProgressCallback = void (*)(const BellmanFordCsrProgress& progress, void* user_data);

struct BellmanFordCsrResult {
  std::vector<float> dist;
  int iterations_used = 0;
  bool converged = false;
};

struct HostCsrF32 {
  minplus_sparse::Offset rows = 0;
  minplus_sparse::Offset cols = 0;
  minplus_sparse::Offset nnz = 0;
  std::vector<minplus_sparse::Offset> rowptr;
  std::vector<minplus_sparse::Index> colind;
  std::vector<float> values;
};

// Matrix convention: row v, column u = weight of edge u -> v (incoming).
// The whole solve runs in one persistent launch; the progress callback is
// called from the calling thread while it runs, once per iteration and in
// order, with the field values the reference's per-iteration loop reports
// (rounds the reference would run after convergence follow at the end).
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                  int max_iters, cudaStream_t stream = nullptr,
                                                  BellmanFordCsrProgressCallback progress_callback = nullptr,
                                                  void* progress_user_data = nullptr);
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                  cudaStream_t stream = nullptr);
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const HostCsrF32& adjacency, int source, int max_iters,
                                                  cudaStream_t stream = nullptr,
                                                  BellmanFordCsrProgressCallback progress_callback = nullptr,
                                                  void* progress_user_data = nullptr);
BellmanFordCsrResult bellman_ford_minplus_hip_csr(const HostCsrF32& adjacency, int source,
                                                  cudaStream_t stream = nullptr);

struct BellmanFordCsrNoChecksResult {
  std::vector<float> dist;
  int iterations_used = 0;
};

BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(
    const minplus_sparse::DeviceCsrF32& d_adjacency, int source, int max_iters, cudaStream_t stream = nullptr,
    BellmanFordCsrProgressCallback progress_callback = nullptr, void* progress_user_data = nullptr);
BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(const minplus_sparse::DeviceCsrF32& d_adjacency,
                                                                    int source, cudaStream_t stream = nullptr);
BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(
    const HostCsrF32& adjacency, int source, int max_iters, cudaStream_t stream = nullptr,
    BellmanFordCsrProgressCallback progress_callback = nullptr, void* progress_user_data = nullptr);
BellmanFordCsrNoChecksResult bellman_ford_minplus_hip_csr_no_checks(const HostCsrF32& adjacency, int source,
                                                                    cudaStream_t stream = nullptr);

struct BellmanFordCsrVarChecksResult {
  std::vector<float> dist;
  int iterations_used = 0;
  bool converged = false;
  int check_interval = 0;
  int checks_performed = 0;
  int changed_checks = 0;
  int unchanged_checks = 0;
  double initialization_ms = 0.0;
  double bellman_ford_loop_ms = 0.0;
  double relaxation_ms = 0.0;
  double checked_merge_ms = 0.0;
  double unchecked_merge_ms = 0.0;
  double checked_iteration_ms = 0.0;
  double unchecked_iteration_ms = 0.0;
  double final_copy_ms = 0.0;
  double total_runtime_ms = 0.0;
  double estimated_check_overhead_ms = 0.0;
};

BellmanFordCsrVarChecksResult bellman_ford_minplus_hip_csr_var_checks_with_stats(
    const minplus_sparse::DeviceCsrF32& d_adjacency, int source, int max_iters, int check_interval,
    cudaStream_t stream = nullptr, BellmanFordCsrProgressCallback progress_callback = nullptr,
    void* progress_user_data = nullptr);
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const minplus_sparse::DeviceCsrF32& d_adjacency,
                                                             int source, int max_iters, int check_interval,
                                                             cudaStream_t stream = nullptr,
                                                             BellmanFordCsrProgressCallback progress_callback = nullptr,
                                                             void* progress_user_data = nullptr);
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const minplus_sparse::DeviceCsrF32& d_adjacency,
                                                             int source, int check_interval,
                                                             cudaStream_t stream = nullptr);
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const HostCsrF32& adjacency, int source, int max_iters,
                                                             int check_interval, cudaStream_t stream = nullptr,
                                                             BellmanFordCsrProgressCallback progress_callback = nullptr,
                                                             void* progress_user_data = nullptr);
BellmanFordCsrResult bellman_ford_minplus_hip_csr_var_checks(const HostCsrF32& adjacency, int source,
                                                             int check_interval, cudaStream_t stream = nullptr);

// ---------------------------------------------------------------- dense BF
struct BellmanFordResult {
  std::vector<float> dist;
  int iterations_used = 0;
  bool converged = false;
};

// d_adjacency[v * n + u] = weight of u -> v, +inf = no edge.
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source, int max_iters,
                                           cudaStream_t stream);
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source, cudaStream_t stream);
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source, int max_iters);
BellmanFordResult bellman_ford_minplus_hip(const float* d_adjacency, int n, int source);
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source, int max_iters,
                                           cudaStream_t stream);
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source,
                                           cudaStream_t stream);
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source, int max_iters);
BellmanFordResult bellman_ford_minplus_hip(const std::vector<float>& adjacency, int n, int source);

// ---------------------------------------------------------------- delta-stepping
using DeltaSteppingCsrProgress = BellmanFordCsrProgress;
using DeltaSteppingCsrProgressCallback = BellmanFordCsrProgressCallback;
using DeltaSteppingCsrResult = BellmanFordCsrResult;

DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                      float delta, int max_iters, cudaStream_t stream = nullptr,
                                                      DeltaSteppingCsrProgressCallback progress_callback = nullptr,
                                                      void* progress_user_data = nullptr);
DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                      float delta, cudaStream_t stream = nullptr);
DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const HostCsrF32& adjacency, int source, float delta,
                                                      int max_iters, cudaStream_t stream = nullptr,
                                                      DeltaSteppingCsrProgressCallback progress_callback = nullptr,
                                                      void* progress_user_data = nullptr);
DeltaSteppingCsrResult delta_stepping_minplus_hip_csr(const HostCsrF32& adjacency, int source, float delta,
                                                      cudaStream_t stream = nullptr);

inline DeltaSteppingCsrResult delta_stepping_hip_csr(const minplus_sparse::DeviceCsrF32& d_adjacency, int source,
                                                     float delta, int max_iters, cudaStream_t stream = nullptr,
                                                     DeltaSteppingCsrProgressCallback progress_callback = nullptr,
                                                     void* progress_user_data = nullptr) {
  return delta_stepping_minplus_hip_csr(d_adjacency, source, delta, max_iters, stream, progress_callback,
                                        progress_user_data);
}
inline DeltaSteppingCsrResult delta_stepping_hip_csr(const HostCsrF32& adjacency, int source, float delta,
                                                     int max_iters, cudaStream_t stream = nullptr,
                                                     DeltaSteppingCsrProgressCallback progress_callback = nullptr,
                                                     void* progress_user_data = nullptr) {
  return delta_stepping_minplus_hip_csr(adjacency, source, delta, max_iters, stream, progress_callback,
                                        progress_user_data);
}

// ---------------------------------------------------------------- oneshot
// Outgoing CSR: edges of u in row_offsets[u] .. row_offsets[u+1]-1.
struct CsrGraph {
  int num_nodes = 0;
  int num_edges = 0;
  std::vector<int> row_offsets;
  std::vector<int> col_indices;
  std::vector<float> weights;
};

struct SSSPOptions {
  int max_iters = -1;
  int num_buckets = 32;
  int bucket_capacity_per_bucket = 0;
  float initial_delta = 0.0f;
  bool dynamic_delta = true;
  int target_low_work = 8192;
  int target_high_work = 262144;
};

struct SSSPResult {
  std::vector<float> dist;
  int iterations_used = 0;
  bool converged = false;
  bool has_negative_cycle = false;
  unsigned long long work_count = 0;
  float milliseconds = 0.0f;
  float final_delta = 0.0f;
};

SSSPResult bellman_ford_sssp_hip(const CsrGraph& graph, int source, const SSSPOptions& options = {},
                                 cudaStream_t stream = nullptr);
SSSPResult adds_sssp_hip(const CsrGraph& graph, int source, const SSSPOptions& options = {},
                         cudaStream_t stream = nullptr);
// adjacency[u * n + v] = weight of u -> v; infinity means no edge.
SSSPResult bellman_ford_sssp_hip(const std::vector<float>& adjacency, int n, int source,
                                 const SSSPOptions& options = {}, cudaStream_t stream = nullptr);
SSSPResult adds_sssp_hip(const std::vector<float>& adjacency, int n, int source, const SSSPOptions& options = {},
                         cudaStream_t stream = nullptr);
CsrGraph dense_to_csr_outgoing(const std::vector<float>& adjacency, int n);

// ---------------------------------------------------------------- hip_adds
namespace hip_adds {

static constexpr uint32_t kBucketCount = 32u;

template <typename Weight>
struct DeviceCsrGraph {
  uint32_t num_vertices = 0;
  uint32_t num_edges = 0;
  const uint32_t* row_offsets = nullptr;
  const uint32_t* col_indices = nullptr;
  const Weight* weights = nullptr;
};

struct Options {
  uint32_t worker_blocks = 0;
  uint32_t assignment_chunk = 256;
  uint32_t initial_active_buckets = 1;
  uint32_t max_active_buckets = kBucketCount;
  double initial_delta = 0.0;
  double initial_delta_scale = 16.0;
  double min_delta = 1.0e-3;
  double delta_growth = 1.5;
  double delta_shrink = 0.75;
  double clip_threshold = 0.65;
  double utilization_low = 0.35;
  double utilization_high = 0.85;
  uint32_t adjust_period_head_switches = 8;
  bool dynamic_delta = true;
  bool dynamic_active_buckets = true;
  size_t pool_words = 0;
  double memory_fraction = 0.45;
  bool initialize_distances = true;
};

struct RunStats {
  double initial_delta = 0.0;
  double final_delta = 0.0;
  double final_bucket_base = 0.0;
  uint32_t worker_blocks = 0;
  uint32_t final_active_buckets = 0;
  uint32_t pool_pages = 0;
  uint32_t device_error = 0;
  uint64_t assigned_items = 0;
  uint64_t processed_items = 0;
  uint64_t enqueued_items = 0;
  uint64_t edge_relaxations = 0;
  uint64_t successful_relaxations = 0;
  uint64_t head_switches = 0;
  uint64_t delta_updates = 0;
  uint64_t max_inflight_items = 0;
};

enum class Status : int {
  Success = 0,
  InvalidArgument,
  HipError,
  OutOfMemory,
  PoolExhausted,
  BucketOverflow,
  DeviceError,
  Timeout  // a bounded device wait gave up (the kernel exited cleanly)
};

const char* status_string(Status status);

Status sssp(const DeviceCsrGraph<float>& graph, uint32_t source, float* d_distances, RunStats* stats = nullptr,
            const Options& options = Options{}, cudaStream_t stream = nullptr);
Status sssp(const DeviceCsrGraph<uint32_t>& graph, uint32_t source, uint32_t* d_distances, RunStats* stats = nullptr,
            const Options& options = Options{}, cudaStream_t stream = nullptr);

}  // namespace hip_adds
