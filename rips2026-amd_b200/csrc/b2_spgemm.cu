// CSR x CSR min-plus product  C = A (min,+) B  (fp32 and int32).
//
// Semantics follow minplus_sparse::minplus_spgemm_csr_f32
// (HIP_kernel/minplus_mm/src/minplus_sparse_hip.hpp:64-150,
// minplus_sparse_hip.cpp:93-99, 170-398): absent entries are +inf; explicit
// +inf and NaN entries of A, and +inf / NaN candidates a + b, are skipped;
// duplicate columns are min-reduced; a bad row pointer or column index makes
// the call fail.  Outputs are allocated here and owned by the caller.
// Unlike the reference (per-row shared-memory hash with a fixed capacity and
// unsorted output) rows have no size limit and output columns are sorted.
//
// Expand-sort-compress:
//   1. k_row_bound   : candidates per row = sum of |B row k| over A's row;
//                      validates A's and B's row pointers and A's columns;
//   2. scan          : candidate offsets (CUB);
//   3. k_expand      : one warp per row writes (column, value) candidates,
//                      B rows read as contiguous lane-strided runs;
//   4. segmented sort: candidates of each row by column (CUB, stable);
//   5. k_count / scan / k_compress: one warp per row min-reduces runs of
//                      equal columns and writes the exact-size output.
// The int32 twin treats values >= INT32_MAX/2 as absent and drops sums that
// reach it.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "b2_common.cuh"
#include "b2_internal.hpp"

namespace b2 {
namespace {

constexpr int32_t kMiss32 = 1073741823;
constexpr int32_t kDropCol = 0x7fffffff;   // sorts after every real column

enum SpStatus : uint32_t { kSpOk = 0, kSpBadIndex = 1, kSpBadRowptr = 2 };

template <typename T>
struct SpVal;
template <>
struct SpVal<float> {
  __device__ __forceinline__ static bool present(float a) { return a == a && a != __int_as_float(0x7f800000); }
  __device__ __forceinline__ static bool combine(float a, float b, float& out) {
    out = a + b;
    return present(out);
  }
  __device__ __forceinline__ static float vmin(float x, float y) { return y < x ? y : x; }
};
template <>
struct SpVal<int32_t> {
  __device__ __forceinline__ static bool present(int32_t a) { return a < kMiss32; }
  __device__ __forceinline__ static bool combine(int32_t a, int32_t b, int32_t& out) {
    if (b >= kMiss32) return false;
    const long long s = (long long)a + (long long)b;
    out = (int32_t)s;
    return s < kMiss32;
  }
  __device__ __forceinline__ static int32_t vmin(int32_t x, int32_t y) { return y < x ? y : x; }
};

__global__ void k_row_bound(int64_t M, int64_t K, int64_t annz, int64_t bnnz, const int64_t* __restrict__ arp,
                            const int32_t* __restrict__ aci, const int64_t* __restrict__ brp,
                            unsigned long long* __restrict__ ub, uint32_t* status) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < M; i += nwarps) {
    const int64_t a0 = arp[i], a1 = arp[i + 1];
    unsigned long long s = 0;
    if (a0 < 0 || a1 < a0 || a1 > annz) {
      if (lane == 0) atomicCAS(status, kSpOk, (uint32_t)kSpBadRowptr);
    } else {
      for (int64_t p = a0 + lane; p < a1; p += 32) {
        const int32_t k = aci[p];
        if (k < 0 || (int64_t)k >= K) {
          atomicCAS(status, kSpOk, (uint32_t)kSpBadIndex);
          continue;
        }
        const int64_t b0 = brp[k], b1 = brp[k + 1];
        if (b0 < 0 || b1 < b0 || b1 > bnnz) {
          atomicCAS(status, kSpOk, (uint32_t)kSpBadRowptr);
          continue;
        }
        s += (unsigned long long)(b1 - b0);
      }
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) ub[i] = s;
  }
}

template <typename T>
__global__ void k_expand(int64_t M, int64_t N, const int64_t* __restrict__ arp, const int32_t* __restrict__ aci,
                         const T* __restrict__ av, const int64_t* __restrict__ brp,
                         const int32_t* __restrict__ bci, const T* __restrict__ bv,
                         const unsigned long long* __restrict__ off, int32_t* __restrict__ ccol,
                         T* __restrict__ cval, uint32_t* status) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < M; i += nwarps) {
    unsigned long long pos = off[i];
    for (int64_t p = arp[i]; p < arp[i + 1]; ++p) {
      const int32_t k = aci[p];
      const T a = av[p];
      const int64_t b0 = brp[k], b1 = brp[k + 1];
      const bool use = SpVal<T>::present(a);
      for (int64_t q = b0 + lane; q < b1; q += 32) {
        const int32_t j = bci[q];
        T c = T(0);
        bool ok = use && SpVal<T>::combine(a, bv[q], c);
        if (j < 0 || (int64_t)j >= N) {
          atomicCAS(status, kSpOk, (uint32_t)kSpBadIndex);
          ok = false;
        }
        const unsigned long long w = pos + (unsigned long long)(q - b0);
        ccol[w] = ok ? j : kDropCol;
        cval[w] = c;
      }
      pos += (unsigned long long)(b1 - b0);
    }
  }
}

// distinct kept columns per row (runs of equal columns in the sorted segment)
__global__ void k_count(int64_t M, const unsigned long long* __restrict__ off, const int32_t* __restrict__ scol,
                        int64_t* __restrict__ cnt) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < M; i += nwarps) {
    const unsigned long long b = off[i], e = off[i + 1];
    long long c = 0;
    for (unsigned long long q = b + lane; q < e; q += 32) {
      const int32_t j = scol[q];
      if (j != kDropCol && (q == b || scol[q - 1] != j)) ++c;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[i] = c;
  }
}

template <typename T>
__global__ void k_compress(int64_t M, const unsigned long long* __restrict__ off, const int32_t* __restrict__ scol,
                           const T* __restrict__ sval, const int64_t* __restrict__ crp, int32_t* __restrict__ cci,
                           T* __restrict__ cv) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < M; i += nwarps) {
    const unsigned long long b = off[i], e = off[i + 1];
    int64_t outpos = crp[i];
    for (unsigned long long base = b; base < e; base += 32) {
      const unsigned long long q = base + lane;
      const bool in = q < e;
      const int32_t j = in ? scol[q] : kDropCol;
      const bool head = in && j != kDropCol && (q == b || scol[q - 1] != j);
      const uint32_t hm = __ballot_sync(0xffffffffu, head);
      if (head) {
        // min over the run of column j (runs may cross the 32-entry window)
        T m = sval[q];
        for (unsigned long long r = q + 1; r < e && scol[r] == j; ++r) m = SpVal<T>::vmin(m, sval[r]);
        const int64_t w = outpos + __popc(hm & ((1u << lane) - 1u));
        cci[w] = j;
        cv[w] = m;
      }
      outpos += __popc(hm);
    }
  }
}

int grid_rows(int64_t rows) {
  int64_t b = (rows * 32 + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

template <typename T>
struct DBuf {
  T* p = nullptr;
  ~DBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t n) { return cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

template <typename T>
b2_status spgemm(const b2_csr* A, const b2_csr* B, int64_t** dC_rowptr, int32_t** dC_colind, T** dC_values,
                 int64_t* hC_nnz, cudaStream_t st) {
  if (!A || !B || !dC_rowptr || !dC_colind || !dC_values || !hC_nnz) return B2_INVALID_ARGUMENT;
  *dC_rowptr = nullptr;
  *dC_colind = nullptr;
  *dC_values = nullptr;
  *hC_nnz = 0;
  if (A->rows < 0 || A->cols < 0 || A->nnz < 0 || B->rows < 0 || B->cols < 0 || B->nnz < 0) return B2_INVALID_ARGUMENT;
  if (A->cols != B->rows) return B2_INVALID_ARGUMENT;
  if (A->cols > 0x7fffffffLL || B->cols > 0x7fffffffLL) return B2_INVALID_ARGUMENT;
  if (A->rowptr_bits != 64 || B->rowptr_bits != 64 || !A->on_device || !B->on_device) return B2_INVALID_ARGUMENT;
  if (!A->rowptr || !B->rowptr) return B2_INVALID_ARGUMENT;
  if ((A->nnz > 0 && (!A->colind || !A->values)) || (B->nnz > 0 && (!B->colind || !B->values)))
    return B2_INVALID_ARGUMENT;
  const int64_t M = A->rows, K = A->cols, N = B->cols;
  const int64_t* arp = (const int64_t*)A->rowptr;
  const int64_t* brp = (const int64_t*)B->rowptr;
  int64_t* crp = nullptr;
  B2_CUDA_TRY(cudaMalloc((void**)&crp, (size_t)(M + 1) * sizeof(int64_t)));
  auto fail = [&](b2_status s) {
    cudaFree(crp);
    return s;
  };
  if (M == 0 || K == 0 || A->nnz == 0 || B->nnz == 0) {
    if (cudaMemsetAsync(crp, 0, (size_t)(M + 1) * sizeof(int64_t), st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return fail(B2_CUDA_ERROR);
    *dC_rowptr = crp;
    return B2_SUCCESS;
  }
  DBuf<unsigned long long> ub, off;
  DBuf<uint32_t> status;
  DBuf<unsigned char> tmp;
  if (ub.alloc((size_t)M + 1) != cudaSuccess || off.alloc((size_t)M + 1) != cudaSuccess ||
      status.alloc(1) != cudaSuccess)
    return fail(B2_OUT_OF_MEMORY);
  cudaError_t e = cudaMemsetAsync(status.p, 0, 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ub.p + M, 0, 8, st);
  k_row_bound<<<grid_rows(M), 256, 0, st>>>(M, K, A->nnz, B->nnz, arp, A->colind, brp, ub.p, status.p);
  if (e == cudaSuccess) e = cudaGetLastError();
  size_t tb = 0;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, ub.p, off.p, M + 1, st);
  if (e == cudaSuccess) e = tmp.alloc(tb);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp.p, tb, ub.p, off.p, M + 1, st);
  unsigned long long U = 0;
  uint32_t hs = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&U, off.p + M, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hs, status.p, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(from_cuda(e));
  if (hs == kSpBadIndex) return fail(B2_INVALID_INDEX);
  if (hs == kSpBadRowptr) return fail(B2_INVALID_ROWPTR);
  if (U > 0x7fffffffull) return fail(B2_NOT_SUPPORTED);   // segmented sort item count is int
  DBuf<int32_t> col0, col1;
  DBuf<T> val0, val1;
  DBuf<int64_t> cnt;
  if (col0.alloc(U) != cudaSuccess || col1.alloc(U) != cudaSuccess || val0.alloc(U) != cudaSuccess ||
      val1.alloc(U) != cudaSuccess || cnt.alloc((size_t)M + 1) != cudaSuccess)
    return fail(B2_OUT_OF_MEMORY);
  if (U > 0) {
    k_expand<T><<<grid_rows(M), 256, 0, st>>>(M, N, arp, A->colind, (const T*)A->values, brp, B->colind,
                                              (const T*)B->values, off.p, col0.p, val0.p, status.p);
    e = cudaGetLastError();
    size_t tb2 = 0;
    DBuf<unsigned char> tmp2;
    if (e == cudaSuccess)
      e = cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb2, col0.p, col1.p, val0.p, val1.p, (int)U, (int)M,
                                                    off.p, off.p + 1, st);
    if (e == cudaSuccess) e = tmp2.alloc(tb2);
    if (e == cudaSuccess)
      e = cub::DeviceSegmentedSort::StableSortPairs(tmp2.p, tb2, col0.p, col1.p, val0.p, val1.p, (int)U, (int)M,
                                                    off.p, off.p + 1, st);
    if (e == cudaSuccess) {
      k_count<<<grid_rows(M), 256, 0, st>>>(M, off.p, col1.p, cnt.p);
      e = cudaGetLastError();
    }
  } else {
    e = cudaMemsetAsync(cnt.p, 0, (size_t)M * sizeof(int64_t), st);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(cnt.p + M, 0, 8, st);
  size_t tb3 = 0;
  DBuf<unsigned char> tmp3;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb3, cnt.p, crp, M + 1, st);
  if (e == cudaSuccess) e = tmp3.alloc(tb3);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp3.p, tb3, cnt.p, crp, M + 1, st);
  int64_t nnz = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nnz, crp + M, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hs, status.p, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(from_cuda(e));
  if (hs == kSpBadIndex) return fail(B2_INVALID_INDEX);
  if (hs == kSpBadRowptr) return fail(B2_INVALID_ROWPTR);
  int32_t* cci = nullptr;
  T* cv = nullptr;
  if (nnz > 0) {
    if (cudaMalloc((void**)&cci, (size_t)nnz * sizeof(int32_t)) != cudaSuccess) return fail(B2_OUT_OF_MEMORY);
    if (cudaMalloc((void**)&cv, (size_t)nnz * sizeof(T)) != cudaSuccess) {
      cudaFree(cci);
      return fail(B2_OUT_OF_MEMORY);
    }
    k_compress<T><<<grid_rows(M), 256, 0, st>>>(M, off.p, col1.p, val1.p, crp, cci, cv);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      cudaFree(cci);
      cudaFree(cv);
      return fail(from_cuda(e));
    }
  }
  *dC_rowptr = crp;
  *dC_colind = cci;
  *dC_values = cv;
  *hC_nnz = nnz;
  return B2_SUCCESS;
}

}  // namespace
}  // namespace b2

extern "C" b2_status b2_minplus_spgemm_f32(const b2_csr* A, const b2_csr* B, int64_t** dC_rowptr,
                                           int32_t** dC_colind, float** dC_values, int64_t* hC_nnz,
                                           b2_stream stream) {
  if (A && A->weight_type != B2_W_F32) return B2_INVALID_ARGUMENT;
  if (B && B->weight_type != B2_W_F32) return B2_INVALID_ARGUMENT;
  return b2::spgemm<float>(A, B, dC_rowptr, dC_colind, dC_values, hC_nnz, (cudaStream_t)stream);
}

extern "C" b2_status b2_minplus_spgemm_i32(const b2_csr* A, const b2_csr* B, int64_t** dC_rowptr,
                                           int32_t** dC_colind, int32_t** dC_values, int64_t* hC_nnz,
                                           b2_stream stream) {
  return b2::spgemm<int32_t>(A, B, dC_rowptr, dC_colind, dC_values, hC_nnz, (cudaStream_t)stream);
}
