// Resident graph construction: validation, statistics, and the packed
// outgoing CSR every SSSP kernel reads.
//
// The reference transposes the incoming CSR to outgoing on every
// delta-stepping call (build_outgoing_csr_from_incoming,
// HIP_kernel/delta_stepping/src/delta_stepping_hip_CSR.cpp:558-605) and
// validates it every call (:546-556).  Here both happen once when the graph
// becomes resident; solves only read the packed arrays:
//   rowptr : uint64[n+1]        (8 B / vertex)
//   edges  : uint2[m] = {dst, weight bits}  (8 B / edge, one coalesced load)
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "b2_common.cuh"
#include "b2_internal.hpp"

namespace b2 {
namespace {

__device__ __forceinline__ int64_t load_rp(const void* rp, int bits, int64_t i) {
  return bits == 64 ? (int64_t)((const int64_t*)rp)[i] : (int64_t)((const uint32_t*)rp)[i];
}

// flags[0] bad rowptr, [1] bad column, [2] NaN weight, [3] negative weight
__global__ void k_validate(int64_t rows, int64_t cols, int64_t nnz, const void* rp, int bits,
                           const int32_t* colind, const void* vals, int wt, uint32_t* flags) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if (tid == 0) {
    if (load_rp(rp, bits, 0) != 0 || load_rp(rp, bits, rows) != nnz) atomicOr(&flags[0], 1u);
  }
  for (int64_t r = tid; r < rows; r += stride) {
    const int64_t a = load_rp(rp, bits, r), b = load_rp(rp, bits, r + 1);
    if (a < 0 || b < a || b > nnz) atomicOr(&flags[0], 1u);
  }
  for (int64_t e = tid; e < nnz; e += stride) {
    const int32_t c = colind[e];
    if (c < 0 || (int64_t)c >= cols) atomicOr(&flags[1], 1u);
    if (wt == B2_W_F32) {
      const float w = ((const float*)vals)[e];
      if (w != w) atomicOr(&flags[2], 1u);
      if (w < 0.0f) atomicOr(&flags[3], 1u);
    }
  }
}

__global__ void k_count_degree(int64_t nnz, const int32_t* colind, uint32_t* deg) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride)
    atomicAdd(&deg[colind[e]], 1u);
}

struct U32ToU64 {
  __host__ __device__ uint64_t operator()(uint32_t x) const { return (uint64_t)x; }
};

// Scatter incoming row r = destination into outgoing rows keyed by source;
// one warp per incoming row.
__global__ void k_transpose_fill(int64_t rows, const void* rp, int bits, const int32_t* colind,
                                 const uint32_t* vals, unsigned long long* cursor, uint2* out) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t r = warp; r < rows; r += nwarps) {
    const int64_t a = load_rp(rp, bits, r), b = load_rp(rp, bits, r + 1);
    for (int64_t e = a + lane; e < b; e += 32) {
      const uint32_t src = (uint32_t)colind[e];
      const unsigned long long pos = atomicAdd(&cursor[src], 1ull);
      out[pos] = make_uint2((uint32_t)r, vals[e]);
    }
  }
}

__global__ void k_pack_outgoing(int64_t rows, int64_t nnz, const void* rp, int bits,
                                const int32_t* colind, const uint32_t* vals, uint64_t* rowptr,
                                uint2* out) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = tid; r <= rows; r += stride) rowptr[r] = (uint64_t)load_rp(rp, bits, r);
  for (int64_t e = tid; e < nnz; e += stride) out[e] = make_uint2((uint32_t)colind[e], vals[e]);
}

// Deterministic statistics: block b owns a fixed contiguous edge range and
// reduces it in a fixed tree order; the host adds the partials in order.
constexpr int kStatBlocks = 512;
constexpr int kStatThreads = 256;
__global__ void k_weight_stats(int64_t m, const uint2* edges, int wt, double* part_sum,
                               unsigned long long* part_pos) {
  __shared__ double s_sum[kStatThreads];
  __shared__ unsigned long long s_cnt[kStatThreads];
  const int64_t chunk = (m + gridDim.x - 1) / gridDim.x;
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < m ? lo + chunk : m;
  double sum = 0.0;
  unsigned long long cnt = 0;
  for (int64_t e = lo + threadIdx.x; e < hi; e += blockDim.x) {
    const uint32_t wb = edges[e].y;
    double w;
    if (wt == B2_W_F32) {
      const float f = __uint_as_float(wb);
      w = (f > 0.0f && isfinite(f)) ? (double)f : 0.0;
    } else {
      w = (double)wb;
    }
    if (w > 0.0) { sum += w; ++cnt; }
  }
  s_sum[threadIdx.x] = sum;
  s_cnt[threadIdx.x] = cnt;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + s];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part_sum[blockIdx.x] = s_sum[0];
    part_pos[blockIdx.x] = s_cnt[0];
  }
}

__global__ void k_max_degree(int64_t n, const uint64_t* rowptr, uint32_t* out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  uint32_t mx = 0;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const uint64_t d = rowptr[v + 1] - rowptr[v];
    mx = d > mx ? (uint32_t)(d > 0xFFFFFFFFull ? 0xFFFFFFFFull : d) : mx;
  }
  atomicMax(out, mx);
}

__global__ void k_unpack(int64_t m, const uint2* e, uint32_t* key, uint32_t* dst) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint2 x = e[i];
    dst[i] = x.x;
    key[i] = x.y;
  }
}
__global__ void k_pack(int64_t m, const uint32_t* key, const uint32_t* dst, uint2* e) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    e[i] = make_uint2(dst[i], key[i]);
}

int grid_for(int64_t items, int threads) {
  int64_t b = (items + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t count) { return cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T)); }
  T* release() { T* q = p; p = nullptr; return q; }
};

b2_status finish_stats(b2_graph g, cudaStream_t st) {
  DevBuf<double> psum;
  DevBuf<unsigned long long> pcnt;
  DevBuf<uint32_t> dmax;
  B2_CUDA_TRY(psum.alloc(kStatBlocks));
  B2_CUDA_TRY(pcnt.alloc(kStatBlocks));
  B2_CUDA_TRY(dmax.alloc(1));
  B2_CUDA_TRY(cudaMemsetAsync(dmax.p, 0, sizeof(uint32_t), st));
  if (g->m > 0) {
    k_weight_stats<<<kStatBlocks, kStatThreads, 0, st>>>(g->m, g->edges, g->weight_type, psum.p, pcnt.p);
    B2_CUDA_TRY(cudaGetLastError());
  }
  k_max_degree<<<grid_for(g->n, 256), 256, 0, st>>>(g->n, g->rowptr, dmax.p);
  B2_CUDA_TRY(cudaGetLastError());
  std::vector<double> hs(kStatBlocks, 0.0);
  std::vector<unsigned long long> hc(kStatBlocks, 0);
  uint32_t hmax = 0;
  if (g->m > 0) {
    B2_CUDA_TRY(cudaMemcpyAsync(hs.data(), psum.p, kStatBlocks * sizeof(double), cudaMemcpyDeviceToHost, st));
    B2_CUDA_TRY(cudaMemcpyAsync(hc.data(), pcnt.p, kStatBlocks * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  }
  B2_CUDA_TRY(cudaMemcpyAsync(&hmax, dmax.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  B2_CUDA_TRY(cudaStreamSynchronize(st));
  double s = 0.0;
  unsigned long long c = 0;
  for (int i = 0; i < kStatBlocks; ++i) { s += hs[i]; c += hc[i]; }
  g->mean_weight = c ? s / (double)c : 1.0;
  g->mean_degree = g->n ? (double)g->m / (double)g->n : 0.0;
  g->max_degree = (int32_t)std::min<uint32_t>(hmax, 0x7fffffffu);
  return B2_SUCCESS;
}

// ---- degree order ---------------------------------------------------------
// On graphs with a few very high-degree vertices (RMAT, power-law) the
// random label loads and dedup atomics of a solve hit L2 far more often when
// the hot vertices sit next to each other: internal ids are assigned by
// out-degree, descending (stable).  rowptr / edges are rebuilt in that order
// with every destination renamed; solves and queries map the source id in
// and scatter their outputs back through perm.
__global__ void k_degrees(int64_t n, const uint64_t* rowptr, uint32_t* deg, uint32_t* ids) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const uint64_t d = rowptr[v + 1] - rowptr[v];
    deg[v] = (uint32_t)(d > 0xFFFFFFFFull ? 0xFFFFFFFFull : d);
    ids[v] = (uint32_t)v;
  }
}
__global__ void k_inverse(int64_t n, const uint32_t* perm, uint32_t* inv) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) inv[perm[i]] = (uint32_t)i;
}
// one warp per new row i: copy old row perm[i], renaming destinations
__global__ void k_relabel_rows(int64_t n, const uint32_t* perm, const uint32_t* inv, const uint64_t* old_rp,
                               const uint2* old_e, const uint64_t* new_rp, uint2* new_e) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < n; i += nwarps) {
    const uint64_t a = old_rp[perm[i]], len = old_rp[perm[i] + 1] - a, b = new_rp[i];
    for (uint64_t k = lane; k < len; k += 32) {
      const uint2 e = old_e[a + k];
      new_e[b + k] = make_uint2(inv[e.x], e.y);
    }
  }
}

b2_status reorder_by_degree(b2_graph g, cudaStream_t st) {
  if (g->perm || g->n < 2) return B2_SUCCESS;
  const int64_t n = g->n, m = g->m;
  DevBuf<uint32_t> deg, ids, sdeg;
  DevBuf<unsigned char> tmp;
  uint32_t *perm = nullptr, *inv = nullptr;
  uint64_t* rp = nullptr;
  uint2* ed = nullptr;
  auto fail = [&](cudaError_t e) {
    cudaFree(perm); cudaFree(inv); cudaFree(rp); cudaFree(ed);
    return from_cuda(e);
  };
  cudaError_t e = deg.alloc((size_t)n);
  if (e == cudaSuccess) e = ids.alloc((size_t)n);
  if (e == cudaSuccess) e = sdeg.alloc((size_t)n + 1);
  if (e == cudaSuccess) e = cudaMalloc((void**)&perm, (size_t)n * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&inv, (size_t)n * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&rp, (size_t)(n + 1) * 8);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ed, std::max<size_t>((size_t)m, 1) * sizeof(uint2));
  if (e != cudaSuccess) return fail(e);
  k_degrees<<<grid_for(n, 256), 256, 0, st>>>(n, g->rowptr, deg.p, ids.p);
  e = cudaGetLastError();
  size_t tb = 0;
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, deg.p, sdeg.p, ids.p, perm, (int)n, 0, 32, st);
  if (e == cudaSuccess) e = tmp.alloc(tb);
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, deg.p, sdeg.p, ids.p, perm, (int)n, 0, 32, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(sdeg.p + n, 0, 4, st);
  size_t tb2 = 0;
  DevBuf<unsigned char> tmp2;
  cub::TransformInputIterator<uint64_t, U32ToU64, const uint32_t*> it(sdeg.p, U32ToU64());
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb2, it, rp, n + 1, st);
  if (e == cudaSuccess) e = tmp2.alloc(tb2);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp2.p, tb2, it, rp, n + 1, st);
  if (e == cudaSuccess) {
    k_inverse<<<grid_for(n, 256), 256, 0, st>>>(n, perm, inv);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && m) {
    k_relabel_rows<<<grid_for(n * 32, 256), 256, 0, st>>>(n, perm, inv, g->rowptr, g->edges, rp, ed);
    e = cudaGetLastError();
  }
  std::vector<uint32_t> hinv;
  if (e == cudaSuccess) {
    hinv.resize((size_t)n);
    e = cudaMemcpyAsync(hinv.data(), inv, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(e);
  cudaFree(g->rowptr);
  cudaFree(g->edges);
  g->rowptr = rp;
  g->edges = ed;
  g->perm = perm;
  g->inv = inv;
  g->inv_host.swap(hinv);
  g->graph_bytes += (size_t)n * 8;
  return B2_SUCCESS;
}

// Degree order pays off on large graphs whose degree distribution is skewed.
bool wants_degree_order(b2_graph g) {
  return g->n >= ((int64_t)1 << 23) && g->max_degree >= 64.0 * std::max(1.0, g->mean_degree);
}

// Order every adjacency list by weight (stable: equal weights keep their
// order), so the edges with weight <= delta are a prefix of each row and a
// light pass reads exactly them.  Stable segmented radix sort, keys = weight.
b2_status sort_segments_by_weight(int64_t n, int64_t m, const uint64_t* rowptr, uint2* edges, int weight_type,
                                  cudaStream_t st, bool* sorted) {
  *sorted = false;
  if (m < 2) { *sorted = true; return B2_SUCCESS; }
  if (m > 0x7fffffffLL) return B2_SUCCESS;   // segmented sort item count is int; rows stay unsorted
  DevBuf<uint32_t> k0, k1, v0, v1;
  DevBuf<unsigned char> tmp;
  B2_CUDA_TRY(k0.alloc((size_t)m));
  B2_CUDA_TRY(k1.alloc((size_t)m));
  B2_CUDA_TRY(v0.alloc((size_t)m));
  B2_CUDA_TRY(v1.alloc((size_t)m));
  k_unpack<<<grid_for(m, 256), 256, 0, st>>>(m, edges, k0.p, v0.p);
  B2_CUDA_TRY(cudaGetLastError());
  size_t tb = 0;
  const int nseg = (int)n;
  if (weight_type == B2_W_F32) {
    B2_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb, (const float*)k0.p, (float*)k1.p, v0.p, v1.p,
                                                          (int)m, nseg, rowptr, rowptr + 1, st));
    B2_CUDA_TRY(tmp.alloc(tb));
    B2_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(tmp.p, tb, (const float*)k0.p, (float*)k1.p, v0.p, v1.p,
                                                          (int)m, nseg, rowptr, rowptr + 1, st));
  } else {
    B2_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb, (const uint32_t*)k0.p, k1.p, v0.p, v1.p,
                                                          (int)m, nseg, rowptr, rowptr + 1, st));
    B2_CUDA_TRY(tmp.alloc(tb));
    B2_CUDA_TRY(cub::DeviceSegmentedSort::StableSortPairs(tmp.p, tb, (const uint32_t*)k0.p, k1.p, v0.p, v1.p,
                                                          (int)m, nseg, rowptr, rowptr + 1, st));
  }
  k_pack<<<grid_for(m, 256), 256, 0, st>>>(m, k1.p, v1.p, edges);
  B2_CUDA_TRY(cudaGetLastError());
  B2_CUDA_TRY(cudaStreamSynchronize(st));
  *sorted = true;
  return B2_SUCCESS;
}

b2_status sort_rows_by_weight(b2_graph g, cudaStream_t st) {
  bool sorted = false;
  b2_status s = sort_segments_by_weight(g->n, g->m, g->rowptr, g->edges, g->weight_type, st, &sorted);
  if (s == B2_SUCCESS) g->rows_sorted = sorted;
  return s;
}

// ---- incoming CSR (pull direction) ----------------------------------------
__global__ void k_in_degree(int64_t m, const uint2* e, uint32_t* deg) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) atomicAdd(&deg[e[i].x], 1u);
}
// one warp per outgoing row u: every edge u -> v lands in row v as (u, w)
__global__ void k_in_fill(int64_t n, const uint64_t* rp, const uint2* e, unsigned long long* cursor, uint2* out) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t u = warp; u < n; u += nwarps)
    for (uint64_t k = rp[u] + lane; k < rp[u + 1]; k += 32) {
      const uint2 x = e[k];
      out[atomicAdd(&cursor[x.x], 1ull)] = make_uint2((uint32_t)u, x.y);
    }
}

}  // namespace

b2_status graph_from_device_outgoing(int64_t n, int64_t m, const uint64_t* rowptr, const uint2* edges,
                                     int weight_type, b2_graph* out) {
  b2_graph g = new b2_graph_s();
  g->n = n;
  g->m = m;
  g->weight_type = weight_type;
  cudaGetDevice(&g->device);
  cudaError_t e1 = cudaMalloc((void**)&g->rowptr, (size_t)(n + 1) * sizeof(uint64_t));
  cudaError_t e2 = cudaMalloc((void**)&g->edges, std::max<size_t>((size_t)m, 1) * sizeof(uint2));
  if (e1 != cudaSuccess || e2 != cudaSuccess) { b2_graph_destroy(g); return B2_OUT_OF_MEMORY; }
  cudaMemcpy(g->rowptr, rowptr, (size_t)(n + 1) * sizeof(uint64_t), cudaMemcpyDeviceToDevice);
  if (m) cudaMemcpy(g->edges, edges, (size_t)m * sizeof(uint2), cudaMemcpyDeviceToDevice);
  g->graph_bytes = (size_t)(n + 1) * 8 + (size_t)m * 8;
  b2_status s = finish_stats(g, 0);
  if (s == B2_SUCCESS && wants_degree_order(g)) s = reorder_by_degree(g, 0);
  if (s == B2_SUCCESS) s = sort_rows_by_weight(g, 0);
  if (s != B2_SUCCESS) { b2_graph_destroy(g); return s; }
  *out = g;
  return B2_SUCCESS;
}

// Incoming CSR in internal ids with weight-sorted rows; built once per graph
// (the order of equal weights inside a row is not fixed, which no result
// depends on: a pulled label is the minimum over the row).
b2_status ensure_incoming(b2_graph g, cudaStream_t st) {
  if (g->in_rowptr) return B2_SUCCESS;
  const int64_t n = g->n, m = g->m;
  DevBuf<uint32_t> deg;
  DevBuf<unsigned long long> cursor;
  DevBuf<unsigned char> tmp;
  uint64_t* rp = nullptr;
  uint2* ed = nullptr;
  cudaError_t e = deg.alloc((size_t)n + 1);
  if (e == cudaSuccess) e = cursor.alloc((size_t)n + 1);
  if (e == cudaSuccess) e = cudaMalloc((void**)&rp, (size_t)(n + 1) * 8);
  if (e == cudaSuccess) e = cudaMalloc((void**)&ed, std::max<size_t>((size_t)m, 1) * sizeof(uint2));
  if (e == cudaSuccess) e = cudaMemsetAsync(deg.p, 0, (size_t)(n + 1) * 4, st);
  if (e == cudaSuccess && m) {
    k_in_degree<<<grid_for(m, 256), 256, 0, st>>>(m, g->edges, deg.p);
    e = cudaGetLastError();
  }
  size_t tb = 0;
  cub::TransformInputIterator<uint64_t, U32ToU64, const uint32_t*> it(deg.p, U32ToU64());
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, it, rp, n + 1, st);
  if (e == cudaSuccess) e = tmp.alloc(tb);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp.p, tb, it, rp, n + 1, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cursor.p, rp, (size_t)(n + 1) * 8, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && m) {
    k_in_fill<<<grid_for(n * 32, 256), 256, 0, st>>>(n, g->rowptr, g->edges, cursor.p, ed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  b2_status s = from_cuda(e);
  bool sorted = false;
  if (s == B2_SUCCESS) s = sort_segments_by_weight(n, m, rp, ed, g->weight_type, st, &sorted);
  if (s == B2_SUCCESS && !sorted && m >= 2) s = B2_NOT_SUPPORTED;   // pull needs weight-sorted rows
  if (s != B2_SUCCESS) {
    cudaFree(rp);
    cudaFree(ed);
    return s;
  }
  g->in_rowptr = rp;
  g->in_edges = ed;
  g->graph_bytes += (size_t)(n + 1) * 8 + (size_t)m * 8;
  return B2_SUCCESS;
}

b2_status ensure_workspace(b2_graph g, bool pred) {
  Workspace& w = g->ws;
  const size_t n = (size_t)g->n;
  if (w.ctl && w.n == n && (w.pred || !pred)) return B2_SUCCESS;
  // (Re)allocate.
  auto fr = [](void* p) { if (p) cudaFree(p); };
  fr(w.dist_a); fr(w.dist_b); fr(w.pstamp); fr(w.bstamp); fr(w.farflag); fr(w.queues); fr(w.hubs);
  fr(w.hstamp); fr(w.lightcnt); fr(w.in_lightcnt); fr(w.trace);
  fr(w.ctl); fr(w.reach);
  if (w.h_ctl) cudaFreeHost(w.h_ctl);
  free_adds_workspace(w);
  if (w.board_h) cudaFreeHost(w.board_h);
  w = Workspace();
  const size_t word = pred ? 8 : 4;
  w.n = n;
  w.pred = pred;
  size_t bytes = 0;
  auto al = [&](void** p, size_t b) -> cudaError_t {
    bytes += b;
    return cudaMalloc(p, std::max<size_t>(b, 16));
  };
  // chunks per phase <= sum over hub vertices of ceil(range / 256), and a hub
  // range has >= 32 edges: at most m / 256 + m / 32 chunks.
  w.hub_cap = std::min<size_t>((size_t)g->m / kHubChunk + (size_t)g->m / 32 + 2, 0xFFFFFFF0ull);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = al(&w.dist_a, n * word);
  if (e == cudaSuccess) e = al(&w.dist_b, n * word);
  if (e == cudaSuccess) e = al((void**)&w.pstamp, n * 4);
  if (e == cudaSuccess) e = al((void**)&w.bstamp, n * 4);
  if (e == cudaSuccess) e = al((void**)&w.farflag, n * 4);
  if (e == cudaSuccess) e = al((void**)&w.hstamp, n * 4);
  if (e == cudaSuccess) e = al((void**)&w.lightcnt, n * 4);
  if (e == cudaSuccess) e = al((void**)&w.in_lightcnt, n * 4);
  if (e == cudaSuccess) e = al((void**)&w.trace, kTraceCap * sizeof(TraceEntry));
  if (e == cudaSuccess) e = al((void**)&w.queues, (5 + (size_t)kRing) * n * 4);
  if (e == cudaSuccess) e = al((void**)&w.hubs, 2 * w.hub_cap * sizeof(HubEntry));
  if (e == cudaSuccess) e = al((void**)&w.ctl, sizeof(Control));
  if (e == cudaSuccess) e = al((void**)&w.reach, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&w.h_ctl, sizeof(Control));
  if (e != cudaSuccess) {
    fr(w.dist_a); fr(w.dist_b); fr(w.pstamp); fr(w.bstamp); fr(w.farflag); fr(w.queues); fr(w.hubs);
    fr(w.hstamp); fr(w.lightcnt); fr(w.in_lightcnt); fr(w.trace);
    fr(w.ctl); fr(w.reach);
    if (w.h_ctl) cudaFreeHost(w.h_ctl);
    w = Workspace();
    return from_cuda(e);
  }
  // Stamps start at zero; phase ids handed out by solves start at 1.
  cudaMemset(w.pstamp, 0, n * 4);
  cudaMemset(w.hstamp, 0, n * 4);
  w.phase_epoch = 1;
  w.bytes = bytes;
  return B2_SUCCESS;
}

}  // namespace b2

using namespace b2;

extern "C" b2_status b2_graph_create(const b2_csr* csr, b2_stream stream, b2_graph* out) {
  if (!csr || !out) return B2_INVALID_ARGUMENT;
  *out = nullptr;
  if (csr->rows <= 0 || csr->rows != csr->cols || csr->nnz < 0) return B2_INVALID_ARGUMENT;
  if (csr->rowptr_bits != 32 && csr->rowptr_bits != 64) return B2_INVALID_ARGUMENT;
  if (csr->weight_type != B2_W_U32 && csr->weight_type != B2_W_F32) return B2_INVALID_ARGUMENT;
  if (csr->orientation != B2_INCOMING && csr->orientation != B2_OUTGOING) return B2_INVALID_ARGUMENT;
  if (!csr->rowptr || (csr->nnz > 0 && (!csr->colind || !csr->values))) return B2_INVALID_ARGUMENT;
  if (csr->rows >= (int64_t)1 << 31) return B2_NOT_SUPPORTED;        // vertex ids are 32-bit
  if (csr->rowptr_bits == 32 && csr->nnz >= ((int64_t)1 << 32)) return B2_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = csr->rows, m = csr->nnz;
  const int bits = csr->rowptr_bits;
  const size_t rp_bytes = (size_t)(n + 1) * (bits / 8);

  // Stage host arrays on the device.
  DevBuf<unsigned char> t_rp, t_ci, t_v;
  const void* rp = csr->rowptr;
  const int32_t* ci = csr->colind;
  const void* vals = csr->values;
  if (!csr->on_device) {
    B2_CUDA_TRY(t_rp.alloc(rp_bytes));
    B2_CUDA_TRY(t_ci.alloc((size_t)m * 4));
    B2_CUDA_TRY(t_v.alloc((size_t)m * 4));
    B2_CUDA_TRY(cudaMemcpyAsync(t_rp.p, csr->rowptr, rp_bytes, cudaMemcpyHostToDevice, st));
    if (m) {
      B2_CUDA_TRY(cudaMemcpyAsync(t_ci.p, csr->colind, (size_t)m * 4, cudaMemcpyHostToDevice, st));
      B2_CUDA_TRY(cudaMemcpyAsync(t_v.p, csr->values, (size_t)m * 4, cudaMemcpyHostToDevice, st));
    }
    rp = t_rp.p;
    ci = (const int32_t*)t_ci.p;
    vals = t_v.p;
  }

  DevBuf<uint32_t> flags;
  B2_CUDA_TRY(flags.alloc(4));
  B2_CUDA_TRY(cudaMemsetAsync(flags.p, 0, 16, st));
  k_validate<<<grid_for(std::max(n, m), 256), 256, 0, st>>>(n, n, m, rp, bits, ci, vals, csr->weight_type,
                                                           flags.p);
  B2_CUDA_TRY(cudaGetLastError());
  uint32_t hf[4];
  B2_CUDA_TRY(cudaMemcpyAsync(hf, flags.p, 16, cudaMemcpyDeviceToHost, st));
  B2_CUDA_TRY(cudaStreamSynchronize(st));
  if (hf[0]) return B2_INVALID_ROWPTR;
  if (hf[1]) return B2_INVALID_INDEX;
  if (hf[2]) return B2_INVALID_WEIGHT;

  b2_graph g = new b2_graph_s();
  g->n = n;
  g->m = m;
  g->weight_type = csr->weight_type;
  g->has_negative = hf[3] != 0;
  cudaGetDevice(&g->device);
  cudaError_t e = cudaMalloc((void**)&g->rowptr, (size_t)(n + 1) * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc((void**)&g->edges, std::max<size_t>((size_t)m, 1) * sizeof(uint2));
  if (e != cudaSuccess) { b2_graph_destroy(g); return from_cuda(e); }
  g->graph_bytes = (size_t)(n + 1) * 8 + (size_t)m * 8;

  if (csr->orientation == B2_OUTGOING) {
    k_pack_outgoing<<<grid_for(std::max(n + 1, m), 256), 256, 0, st>>>(n, m, rp, bits, ci,
                                                                       (const uint32_t*)vals, g->rowptr,
                                                                       g->edges);
    e = cudaGetLastError();
  } else {
    DevBuf<uint32_t> deg;
    DevBuf<unsigned long long> cursor;
    DevBuf<unsigned char> tmp;
    e = deg.alloc((size_t)n + 1);
    if (e == cudaSuccess) e = cursor.alloc((size_t)n + 1);
    if (e == cudaSuccess) e = cudaMemsetAsync(deg.p, 0, (size_t)(n + 1) * 4, st);
    if (e == cudaSuccess && m) {
      k_count_degree<<<grid_for(m, 256), 256, 0, st>>>(m, ci, deg.p);
      e = cudaGetLastError();
    }
    size_t tmp_bytes = 0;
    cub::TransformInputIterator<uint64_t, U32ToU64, const uint32_t*> it(deg.p, U32ToU64());
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, it, g->rowptr, n + 1, st);
    if (e == cudaSuccess) e = tmp.alloc(tmp_bytes);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, it, g->rowptr, n + 1, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(cursor.p, g->rowptr, (size_t)(n + 1) * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && m) {
      k_transpose_fill<<<grid_for(n * 32, 256), 256, 0, st>>>(n, rp, bits, ci, (const uint32_t*)vals,
                                                              cursor.p, g->edges);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess) { b2_graph_destroy(g); return from_cuda(e); }
  b2_status s = finish_stats(g, st);
  if (s == B2_SUCCESS && wants_degree_order(g)) s = reorder_by_degree(g, st);
  if (s == B2_SUCCESS) s = sort_rows_by_weight(g, st);
  if (s != B2_SUCCESS) { b2_graph_destroy(g); return s; }
  *out = g;
  return B2_SUCCESS;
}

extern "C" b2_status b2_graph_destroy(b2_graph g) {
  if (!g) return B2_INVALID_ARGUMENT;
  Workspace& w = g->ws;
  auto fr = [](void* p) { if (p) cudaFree(p); };
  fr(g->rowptr); fr(g->edges); fr(g->in_rowptr32); fr(g->perm); fr(g->inv); fr(g->in_rowptr); fr(g->in_edges);
  fr(w.dist_a); fr(w.dist_b); fr(w.pstamp); fr(w.bstamp); fr(w.farflag); fr(w.queues); fr(w.hubs);
  fr(w.hstamp); fr(w.lightcnt); fr(w.in_lightcnt); fr(w.trace);
  fr(w.ctl); fr(w.reach);
  if (w.h_ctl) cudaFreeHost(w.h_ctl);
  free_adds_workspace(w);
  if (w.board_h) cudaFreeHost(w.board_h);
  delete g;
  return B2_SUCCESS;
}

extern "C" b2_status b2_graph_set_degree_order(b2_graph g, b2_stream stream) {
  if (!g) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g->mu);
  const bool sorted = g->rows_sorted;
  b2_status s = reorder_by_degree(g, (cudaStream_t)stream);
  // relabelled rows keep each row's order, so weight-sorted rows stay sorted
  g->rows_sorted = sorted;
  g->ws.light_key_valid = 0;
  if (s == B2_SUCCESS && g->in_rowptr) {   // the incoming CSR was built in the old ids
    cudaFree(g->in_rowptr);
    cudaFree(g->in_edges);
    g->graph_bytes -= (size_t)(g->n + 1) * 8 + (size_t)g->m * 8;
    g->in_rowptr = nullptr;
    g->in_edges = nullptr;
  }
  g->ws.in_light_key_valid = 0;
  g->features_valid = false;
  g->pol_version = 0;
  return s;
}

extern "C" int32_t b2_graph_degree_ordered(b2_graph g) { return (g && g->perm) ? 1 : 0; }

extern "C" b2_status b2_graph_info_get(b2_graph g, b2_graph_info* info) {
  if (!g || !info) return B2_INVALID_ARGUMENT;
  info->n = g->n;
  info->m = g->m;
  info->weight_type = g->weight_type;
  info->max_out_degree = g->max_degree;
  info->mean_weight = g->mean_weight;
  info->mean_degree = g->mean_degree;
  info->device_bytes = g->graph_bytes + g->ws.bytes;
  return B2_SUCCESS;
}

// Near-Far heuristic (choose_initial_delta, Charlotte_oneshot/sssp_hip.cpp:59-81):
//   delta = C * mean(w > 0) / max(1, m / n), at least 1e-6; uint32 graphs use
//   an integral delta >= 1 (estimate_initial_delta, hip_adds_sssp.cpp:1118).
extern "C" b2_status b2_delta_heuristic(b2_graph g, double scale, double* delta_out) {
  if (!g || !delta_out) return B2_INVALID_ARGUMENT;
  if (!(scale > 0.0)) scale = 16.0;
  double d = scale * g->mean_weight / std::max(1.0, g->mean_degree);
  d = std::max(1.0e-6, d);
  if (g->weight_type == B2_W_U32) d = std::max(1.0, std::floor(d));
  *delta_out = d;
  return B2_SUCCESS;
}
