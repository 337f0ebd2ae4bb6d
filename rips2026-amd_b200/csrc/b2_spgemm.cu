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
// Plan (one pass over the expansion for ordinary rows):
//   1. k_row_bound : candidates per row (sum of |B row k| over A's row);
//                    validates A's and B's row pointers and A's columns and
//                    lists the rows with more than kWarpRowMax candidates;
//   2. scan        : candidate offsets (CUB) = each row's slot in a scratch
//                    array sized by the bound;
//   3. k_rows_warp : one warp per ordinary row gathers its candidates into
//                    shared memory as 64-bit keys (column << 32 | order-
//                    preserving value bits), sorts them in registers with a
//                    bitonic network (32 x P keys, P = 1..16), and writes the
//                    first key of every column run (= the run's minimum) to
//                    the row's scratch slot with its count;
//   4. long rows   : expand-sort-compress over the listed rows only
//                    (k_expand, CUB segmented sort, k_compress into the same
//                    scratch slots);
//   5. scan of the counts (CUB) -> C.rowptr, then k_compact copies every row
//      from its scratch slot to the exact-size outputs: memory this call
//      allocates (the reference's one-call form), or the caller's own buffers
//      (b2_minplus_spgemm_plan / _fill, which need no output allocation here).
// Scratch arrays come from a library-owned stream-ordered memory pool that
// keeps up to 4 GiB cached between calls (no cudaMalloc / cudaFree on the
// critical path after the first call).
// The int32 twin treats values >= INT32_MAX/2 as absent and drops sums that
// reach it.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "b2_common.cuh"
#include "b2_internal.hpp"

namespace b2 {
namespace {

constexpr int32_t kMiss32 = 1073741823;
constexpr int32_t kDropCol = 0x7fffffff;   // sorts after every real column
constexpr int kWarpRowMax = 512;           // candidates of a row sorted in one warp's registers
constexpr int kRowWarps = 8;               // warps per block of k_rows_warp
constexpr int kPairMax = 64;                // candidates of a row sorted by half a warp (k_rows_pair)
constexpr unsigned long long kNoKey = ~0ull;

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

// Order-preserving 32-bit encodings of the values (sorting (column, key)
// pairs puts each column's minimum first).
template <typename T>
struct VKey;
template <>
struct VKey<float> {
  __device__ __forceinline__ static uint32_t enc(float v) { return f32_to_key(v); }
  __device__ __forceinline__ static float dec(uint32_t k) { return key_to_f32(k); }
};
template <>
struct VKey<int32_t> {
  __device__ __forceinline__ static uint32_t enc(int32_t v) { return (uint32_t)v ^ 0x80000000u; }
  __device__ __forceinline__ static int32_t dec(uint32_t k) { return (int32_t)(k ^ 0x80000000u); }
};

__global__ void k_row_bound(int64_t M, int64_t K, int64_t annz, int64_t bnnz, const int64_t* __restrict__ arp,
                            const int32_t* __restrict__ aci, const int64_t* __restrict__ brp,
                            unsigned long long* __restrict__ ub, uint32_t* status, int64_t* __restrict__ long_rows,
                            unsigned long long* __restrict__ long_count) {
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
    if (lane == 0) {
      ub[i] = s;
      if (s > (unsigned long long)kWarpRowMax) long_rows[atomicAdd(long_count, 1ull)] = i;
    }
  }
}

// ---- ordinary rows: one warp, registers -----------------------------------
__device__ __forceinline__ unsigned long long shfl_xor64(unsigned long long x, int m) {
  const uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)x, m);
  const uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(x >> 32), m);
  return ((unsigned long long)hi << 32) | lo;
}

// Sort the row's n <= 32 P staged keys (element e = r * 32 + lane holds
// key[r]; padding is kNoKey), then write the head of every column run.
template <typename T, int P>
__device__ __forceinline__ uint32_t sort_and_emit(const unsigned long long* __restrict__ sk, uint32_t n,
                                                  int32_t* __restrict__ tcol, T* __restrict__ tval) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long key[P];
#pragma unroll
  for (int r = 0; r < P; ++r) {
    const uint32_t e = (uint32_t)r * 32u + lane;
    key[r] = e < n ? sk[e] : kNoKey;
  }
  // bitonic network over 32 P elements, ascending
#pragma unroll
  for (int k = 2; k <= 32 * P; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
#pragma unroll
        for (int r = 0; r < P; ++r) {
          const int rp = r ^ (j >> 5);
          if (rp > r) {
            const bool up = ((r * 32) & k) == 0;
            const unsigned long long x = key[r], y = key[rp];
            if ((x > y) == up) {
              key[r] = y;
              key[rp] = x;
            }
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < P; ++r) {
          const uint32_t e = (uint32_t)r * 32u + lane;
          const bool up = (e & (uint32_t)k) == 0;
          const unsigned long long o = shfl_xor64(key[r], j);
          const bool lower = (lane & (uint32_t)j) == 0;
          const bool take_min = lower == up;
          key[r] = take_min ? (o < key[r] ? o : key[r]) : (o > key[r] ? o : key[r]);
        }
      }
    }
  }
  // heads of column runs, in order
  uint32_t cnt = 0;
  uint32_t carry = 0xFFFFFFFFu;   // column of element r * 32 - 1
#pragma unroll
  for (int r = 0; r < P; ++r) {
    const uint32_t col = (uint32_t)(key[r] >> 32);
    uint32_t pc = __shfl_up_sync(0xffffffffu, col, 1);
    if (lane == 0) pc = carry;
    const bool head = key[r] != kNoKey && col != pc;
    const uint32_t b = __ballot_sync(0xffffffffu, head);
    if (head) {
      const uint32_t pos = cnt + __popc(b & ((1u << lane) - 1u));
      tcol[pos] = (int32_t)col;
      tval[pos] = VKey<T>::dec((uint32_t)key[r]);
    }
    cnt += __popc(b);
    carry = __shfl_sync(0xffffffffu, col, 31);
  }
  return cnt;
}

template <typename T>
__global__ void __launch_bounds__(kRowWarps * 32, 4)
    k_rows_warp(int64_t M, int64_t N, const int64_t* __restrict__ arp, const int32_t* __restrict__ aci,
                const T* __restrict__ av, const int64_t* __restrict__ brp, const int32_t* __restrict__ bci,
                const T* __restrict__ bv, const unsigned long long* __restrict__ off, int32_t* __restrict__ tcol,
                T* __restrict__ tval, int64_t* __restrict__ cnt, uint32_t* status) {
  __shared__ unsigned long long s_keys[kRowWarps][kWarpRowMax];
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long* sk = s_keys[threadIdx.x >> 5];
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = warp; i < M; i += nwarps) {
    const unsigned long long o0 = off[i], ub = off[i + 1] - o0;
    if (ub > (unsigned long long)kWarpRowMax) continue;   // long row: expand-sort-compress
    if (ub <= (unsigned long long)kPairMax) continue;      // small row: k_rows_pair
    // gather: up to 32 A entries at a time; lane t holds entry t's B range
    uint32_t n = 0;
    const int64_t a0 = arp[i], a1 = arp[i + 1];
    for (int64_t pa = a0; pa < a1; pa += 32) {
      const int64_t p = pa + lane;
      T a = T(0);
      int64_t b0 = 0;
      uint32_t len = 0;
      if (p < a1) {
        const int32_t k = aci[p];
        a = av[p];
        if (SpVal<T>::present(a)) {
          b0 = brp[k];
          len = (uint32_t)(brp[k + 1] - b0);
        }
      }
      const uint32_t incl = warp_incl_scan(len);
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      const uint32_t excl = incl - len;
      for (uint32_t s0 = 0; s0 < total; s0 += 32) {
        const uint32_t sl = s0 + lane;
        // owner: the last lane whose range starts at or before slot sl
        uint32_t t = 0;
#pragma unroll
        for (uint32_t step = 16; step >= 1; step >>= 1) {
          const uint32_t e = __shfl_sync(0xffffffffu, excl, t + step);
          if (e <= sl) t += step;
        }
        const uint32_t ex_t = __shfl_sync(0xffffffffu, excl, t);
        const long long b0_t = __shfl_sync(0xffffffffu, (long long)b0, t);
        const T a_t = __shfl_sync(0xffffffffu, a, t);
        if (sl < total) {
          const int64_t q = b0_t + (int64_t)(sl - ex_t);
          const int32_t j = bci[q];
          T c = T(0);
          bool ok = SpVal<T>::combine(a_t, bv[q], c);
          if (j < 0 || (int64_t)j >= N) {
            atomicCAS(status, kSpOk, (uint32_t)kSpBadIndex);
            ok = false;
          }
          sk[n + sl] = ok ? (((unsigned long long)(uint32_t)j << 32) | VKey<T>::enc(c)) : kNoKey;
        }
      }
      n += total;
    }
    __syncwarp();
    uint32_t kept;
    if (n <= 32) kept = sort_and_emit<T, 1>(sk, n, tcol + o0, tval + o0);
    else if (n <= 64) kept = sort_and_emit<T, 2>(sk, n, tcol + o0, tval + o0);
    else if (n <= 128) kept = sort_and_emit<T, 4>(sk, n, tcol + o0, tval + o0);
    else if (n <= 256) kept = sort_and_emit<T, 8>(sk, n, tcol + o0, tval + o0);
    else kept = sort_and_emit<T, 16>(sk, n, tcol + o0, tval + o0);
    if (lane == 0) cnt[i] = kept;
    __syncwarp();
  }
}

// ---- long rows: expand-sort-compress over a row list -----------------------
// ---- small rows: two rows per warp, one per half-warp ----------------------
// Rows with at most kPairMax candidates (every row of a sparse random graph)
// take half a warp each, so a warp keeps two rows' dependent gathers in
// flight.  Same steps as k_rows_warp inside 16 lanes: gather the row's
// candidates as keys into shared memory, bitonic-sort 16 x 4 keys in
// registers (shuffles never cross the half), emit the head of every column
// run.  Loop trip counts are the larger half's, so every shuffle runs on the
// full warp.

template <typename T>
__global__ void __launch_bounds__(kRowWarps * 32)
    k_rows_pair(int64_t M, int64_t N, const int64_t* __restrict__ arp, const int32_t* __restrict__ aci,
                const T* __restrict__ av, const int64_t* __restrict__ brp, const int32_t* __restrict__ bci,
                const T* __restrict__ bv, const unsigned long long* __restrict__ off, int32_t* __restrict__ tcol,
                T* __restrict__ tval, int64_t* __restrict__ cnt, uint32_t* status) {
  __shared__ unsigned long long s_keys[kRowWarps][2][kPairMax];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t half = lane >> 4, hl = lane & 15u;
  unsigned long long* sk = s_keys[threadIdx.x >> 5][half];
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i0 = warp * 2; i0 < M; i0 += nwarps * 2) {
    const int64_t i = i0 + half;
    unsigned long long o0 = 0, ub = 0;
    if (i < M) {
      o0 = off[i];
      ub = off[i + 1] - o0;
    }
    const bool mine = i < M && ub <= (unsigned long long)kPairMax;   // other rows: k_rows_warp
    int64_t a0 = 0, a1 = 0;
    if (mine && ub > 0) {
      a0 = arp[i];
      a1 = arp[i + 1];
    }
    // gather, 16 A entries per pass
    const int64_t alen = a1 - a0;
    const int64_t alen_max = max(alen, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)alen, 16));
    uint32_t n = 0;
    for (int64_t pa = 0; pa < alen_max; pa += 16) {
      const int64_t p = a0 + pa + hl;
      T a = T(0);
      int64_t b0 = 0;
      uint32_t len = 0;
      if (pa + hl < alen) {
        const int32_t k = aci[p];
        a = av[p];
        if (SpVal<T>::present(a)) {
          b0 = brp[k];
          len = (uint32_t)(brp[k + 1] - b0);
        }
      }
      uint32_t incl = len;
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o, 16);
        if (hl >= (uint32_t)o) incl += y;
      }
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 15, 16);
      const uint32_t excl = incl - len;
      const uint32_t total_max = max(total, __shfl_xor_sync(0xffffffffu, total, 16));
      for (uint32_t s0 = 0; s0 < total_max; s0 += 16) {
        const uint32_t sl = s0 + hl;
        uint32_t t = 0;   // owner: the last lane of the half whose range starts at or before slot sl
#pragma unroll
        for (uint32_t step = 8; step >= 1; step >>= 1) {
          const uint32_t e = __shfl_sync(0xffffffffu, excl, t + step, 16);
          if (e <= sl) t += step;
        }
        const uint32_t ex_t = __shfl_sync(0xffffffffu, excl, t, 16);
        const long long b0_t = __shfl_sync(0xffffffffu, (long long)b0, t, 16);
        const T a_t = __shfl_sync(0xffffffffu, a, t, 16);
        if (sl < total) {
          const int64_t q = b0_t + (int64_t)(sl - ex_t);
          const int32_t j = bci[q];
          T c = T(0);
          bool ok = SpVal<T>::combine(a_t, bv[q], c);
          if (j < 0 || (int64_t)j >= N) {
            atomicCAS(status, kSpOk, (uint32_t)kSpBadIndex);
            ok = false;
          }
          sk[n + sl] = ok ? (((unsigned long long)(uint32_t)j << 32) | VKey<T>::enc(c)) : kNoKey;
        }
      }
      n += total;
    }
    __syncwarp();
    // sort 64 keys per half: element e = r * 16 + hl
    constexpr int P = kPairMax / 16;
    unsigned long long key[P];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const uint32_t e = (uint32_t)r * 16u + hl;
      key[r] = (mine && e < n) ? sk[e] : kNoKey;
    }
#pragma unroll
    for (int k = 2; k <= kPairMax; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        if (j >= 16) {
#pragma unroll
          for (int r = 0; r < P; ++r) {
            const int rp = r ^ (j >> 4);
            if (rp > r) {
              const bool up = ((r * 16) & k) == 0;
              const unsigned long long x = key[r], y = key[rp];
              if ((x > y) == up) {
                key[r] = y;
                key[rp] = x;
              }
            }
          }
        } else {
#pragma unroll
          for (int r = 0; r < P; ++r) {
            const uint32_t e = (uint32_t)r * 16u + hl;
            const bool up = (e & (uint32_t)k) == 0;
            const unsigned long long o = shfl_xor64(key[r], j);
            const bool lower = (hl & (uint32_t)j) == 0;
            const bool take_min = lower == up;
            key[r] = take_min ? (o < key[r] ? o : key[r]) : (o > key[r] ? o : key[r]);
          }
        }
      }
    }
    // heads of column runs, in order
    uint32_t kept = 0;
    uint32_t carry = 0xFFFFFFFFu;
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const uint32_t col = (uint32_t)(key[r] >> 32);
      uint32_t pc = __shfl_up_sync(0xffffffffu, col, 1, 16);
      if (hl == 0) pc = carry;
      const bool head = mine && key[r] != kNoKey && col != pc;
      const uint32_t b = __ballot_sync(0xffffffffu, head) & (half ? 0xFFFF0000u : 0x0000FFFFu);
      if (head) {
        const uint32_t pos = kept + __popc(b & ((1u << lane) - 1u));
        tcol[o0 + pos] = (int32_t)col;
        tval[o0 + pos] = VKey<T>::dec((uint32_t)key[r]);
      }
      kept += __popc(b);
      carry = __shfl_sync(0xffffffffu, col, 15, 16);
    }
    if (mine && hl == 0) cnt[i] = kept;
    __syncwarp();
  }
}

template <typename T>
__global__ void k_expand(int64_t L, const int64_t* __restrict__ rows, int64_t N, const int64_t* __restrict__ arp,
                         const int32_t* __restrict__ aci, const T* __restrict__ av, const int64_t* __restrict__ brp,
                         const int32_t* __restrict__ bci, const T* __restrict__ bv,
                         const unsigned long long* __restrict__ off, int32_t* __restrict__ ccol,
                         T* __restrict__ cval, uint32_t* status) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t r = warp; r < L; r += nwarps) {
    const int64_t i = rows[r];
    unsigned long long pos = off[r];
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

// Heads of column runs of each listed row's sorted segment -> the row's
// scratch slot (tcol / tval at slot[row]) and its count.
template <typename T>
__global__ void k_compress(int64_t L, const int64_t* __restrict__ rows, const unsigned long long* __restrict__ off,
                           const int32_t* __restrict__ scol, const T* __restrict__ sval,
                           const unsigned long long* __restrict__ slot, int32_t* __restrict__ tcol,
                           T* __restrict__ tval, int64_t* __restrict__ cnt) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t rr = warp; rr < L; rr += nwarps) {
    const int64_t i = rows[rr];
    const unsigned long long b = off[rr], e = off[rr + 1];
    const unsigned long long dst = slot[i];
    int64_t outpos = 0;
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
        tcol[dst + w] = j;
        tval[dst + w] = m;
      }
      outpos += __popc(hm);
    }
    if (lane == 0) cnt[i] = outpos;
  }
}

__global__ void k_long_bounds(int64_t L, const int64_t* __restrict__ rows, const unsigned long long* __restrict__ off,
                              unsigned long long* __restrict__ lub) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < L; r += (int64_t)gridDim.x * blockDim.x)
    lub[r] = off[rows[r] + 1] - off[rows[r]];
}

// scratch slots -> exact-size outputs (one warp per row)
template <typename T>
__global__ void k_compact(int64_t M, const unsigned long long* __restrict__ slot, const int64_t* __restrict__ crp,
                          const int32_t* __restrict__ tcol, const T* __restrict__ tval, int32_t* __restrict__ cci,
                          T* __restrict__ cv) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (int64_t i = warp; i < M; i += nwarps) {
    const unsigned long long s0 = slot[i];
    const int64_t c0 = crp[i], c = crp[i + 1] - c0;
    for (int64_t q = lane; q < c; q += 32) {
      cci[c0 + q] = tcol[s0 + q];
      cv[c0 + q] = tval[s0 + q];
    }
  }
}

int grid_rows(int64_t rows) {
  int64_t b = (rows * 32 + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

// Library-owned stream-ordered pool for scratch arrays, one per device; it
// keeps up to kPoolKeep bytes cached after a call returns.
constexpr uint64_t kPoolKeep = 4ull << 30;
cudaError_t scratch_pool(cudaMemPool_t* out) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t p;
  e = cudaMemPoolCreate(&p, &props);
  if (e != cudaSuccess) return e;
  uint64_t keep = kPoolKeep;
  cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[dev] = p;
  *out = p;
  return cudaSuccess;
}

// Scratch array from the pool, released (stream-ordered) on scope exit.
template <typename T>
struct DBuf {
  T* p = nullptr;
  cudaStream_t st = nullptr;
  ~DBuf() { if (p) cudaFreeAsync(p, st); }
  cudaError_t alloc(size_t n, cudaStream_t s) {
    st = s;
    cudaMemPool_t pool;
    cudaError_t e = scratch_pool(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync((void**)&p, std::max<size_t>(n, 1) * sizeof(T), pool, s);
  }
  T* release() {
    T* q = p;
    p = nullptr;
    return q;
  }
};

}  // namespace

// A computed product waiting for its outputs: every row's result sits in a
// scratch slot (off[i] .. off[i] + cnt[i]) and crp holds C's row pointers.
struct SpPlan {
  int64_t M = 0;
  int64_t nnz = 0;
  int wt = B2_W_F32;
  int64_t* crp = nullptr;            // pool memory
  unsigned long long* off = nullptr; // pool memory
  int32_t* tcol = nullptr;           // pool memory
  void* tval = nullptr;              // pool memory
  cudaStream_t st = nullptr;
  void release() {
    if (crp) cudaFreeAsync(crp, st);
    if (off) cudaFreeAsync(off, st);
    if (tcol) cudaFreeAsync(tcol, st);
    if (tval) cudaFreeAsync(tval, st);
    crp = nullptr;
    off = nullptr;
    tcol = nullptr;
    tval = nullptr;
  }
};

namespace {

// Steps 1-5 up to C's row pointers; one host synchronization for the scratch
// size (two when long rows exist) and one for nnz(C).
template <typename T>
b2_status compute(const b2_csr* A, const b2_csr* B, cudaStream_t st, SpPlan& plan) {
  if (!A || !B) return B2_INVALID_ARGUMENT;
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
  plan.M = M;
  plan.st = st;
  DBuf<int64_t> crp;
  if (crp.alloc((size_t)M + 1, st) != cudaSuccess) return B2_OUT_OF_MEMORY;
  if (M == 0 || K == 0 || A->nnz == 0 || B->nnz == 0) {
    B2_CUDA_TRY(cudaMemsetAsync(crp.p, 0, (size_t)(M + 1) * sizeof(int64_t), st));
    plan.crp = crp.release();
    plan.nnz = 0;
    return B2_SUCCESS;
  }
  DBuf<unsigned long long> ub, off, lcount;
  DBuf<int64_t> lrows;
  DBuf<uint32_t> status;
  DBuf<unsigned char> tmp;
  if (ub.alloc((size_t)M + 1, st) != cudaSuccess || off.alloc((size_t)M + 1, st) != cudaSuccess ||
      status.alloc(1, st) != cudaSuccess || lrows.alloc((size_t)M, st) != cudaSuccess ||
      lcount.alloc(1, st) != cudaSuccess)
    return B2_OUT_OF_MEMORY;
  cudaError_t e = cudaMemsetAsync(status.p, 0, 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ub.p + M, 0, 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(lcount.p, 0, 8, st);
  if (e == cudaSuccess) {
    k_row_bound<<<grid_rows(M), 256, 0, st>>>(M, K, A->nnz, B->nnz, arp, A->colind, brp, ub.p, status.p, lrows.p,
                                              lcount.p);
    e = cudaGetLastError();
  }
  size_t tb = 0;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, ub.p, off.p, M + 1, st);
  if (e == cudaSuccess) e = tmp.alloc(tb, st);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp.p, tb, ub.p, off.p, M + 1, st);
  unsigned long long hv[2] = {0, 0};   // total candidates, long rows
  uint32_t hs = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hv[0], off.p + M, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hv[1], lcount.p, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hs, status.p, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return from_cuda(e);
  if (hs == kSpBadIndex) return B2_INVALID_INDEX;
  if (hs == kSpBadRowptr) return B2_INVALID_ROWPTR;
  const unsigned long long U = hv[0];
  const int64_t L = (int64_t)hv[1];
  DBuf<int32_t> tcol;
  DBuf<T> tval;
  DBuf<int64_t> cnt;
  if (tcol.alloc(U, st) != cudaSuccess || tval.alloc(U, st) != cudaSuccess ||
      cnt.alloc((size_t)M + 1, st) != cudaSuccess)
    return B2_OUT_OF_MEMORY;
  if (U > 0) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (M + kRowWarps - 1) / kRowWarps;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 6));
    const int pair_blocks =
        (int)std::max<int64_t>(1, std::min<int64_t>((M + 2 * kRowWarps - 1) / (2 * kRowWarps), (int64_t)sms * 16));
    k_rows_pair<T><<<pair_blocks, kRowWarps * 32, 0, st>>>(M, N, arp, A->colind, (const T*)A->values, brp,
                                                         B->colind, (const T*)B->values, off.p, tcol.p, tval.p,
                                                         cnt.p, status.p);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      k_rows_warp<T><<<blocks, kRowWarps * 32, 0, st>>>(M, N, arp, A->colind, (const T*)A->values, brp, B->colind,
                                                      (const T*)B->values, off.p, tcol.p, tval.p, cnt.p, status.p);
      e = cudaGetLastError();
    }
  } else {
    e = cudaMemsetAsync(cnt.p, 0, (size_t)M * sizeof(int64_t), st);
  }
  // long rows: expand, segmented sort, compress into their scratch slots
  DBuf<unsigned long long> lub, loff;
  DBuf<int32_t> col0, col1;
  DBuf<T> val0, val1;
  DBuf<unsigned char> tmp2, tmp3;
  if (e == cudaSuccess && L > 0) {
    if (lub.alloc((size_t)L + 1, st) != cudaSuccess || loff.alloc((size_t)L + 1, st) != cudaSuccess)
      return B2_OUT_OF_MEMORY;
    e = cudaMemsetAsync(lub.p + L, 0, 8, st);
    if (e == cudaSuccess) {
      k_long_bounds<<<(int)std::min<int64_t>((L + 255) / 256, 1184), 256, 0, st>>>(L, lrows.p, off.p, lub.p);
      e = cudaGetLastError();
    }
    size_t tb1 = 0;
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb1, lub.p, loff.p, L + 1, st);
    if (e == cudaSuccess) e = tmp2.alloc(tb1, st);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp2.p, tb1, lub.p, loff.p, L + 1, st);
    unsigned long long LU = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&LU, loff.p + L, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return from_cuda(e);
    if (LU > 0x7fffffffull) return B2_NOT_SUPPORTED;   // segmented sort item count is int
    if (col0.alloc(LU, st) != cudaSuccess || col1.alloc(LU, st) != cudaSuccess || val0.alloc(LU, st) != cudaSuccess ||
        val1.alloc(LU, st) != cudaSuccess)
      return B2_OUT_OF_MEMORY;
    k_expand<T><<<grid_rows(L), 256, 0, st>>>(L, lrows.p, N, arp, A->colind, (const T*)A->values, brp, B->colind,
                                              (const T*)B->values, loff.p, col0.p, val0.p, status.p);
    e = cudaGetLastError();
    size_t tbs = 0;
    if (e == cudaSuccess)
      e = cub::DeviceSegmentedSort::StableSortPairs(nullptr, tbs, col0.p, col1.p, val0.p, val1.p, (int)LU, (int)L,
                                                    loff.p, loff.p + 1, st);
    if (e == cudaSuccess) e = tmp3.alloc(tbs, st);
    if (e == cudaSuccess)
      e = cub::DeviceSegmentedSort::StableSortPairs(tmp3.p, tbs, col0.p, col1.p, val0.p, val1.p, (int)LU, (int)L,
                                                    loff.p, loff.p + 1, st);
    if (e == cudaSuccess) {
      k_compress<T><<<grid_rows(L), 256, 0, st>>>(L, lrows.p, loff.p, col1.p, val1.p, off.p, tcol.p, tval.p, cnt.p);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(cnt.p + M, 0, 8, st);
  size_t tb4 = 0;
  DBuf<unsigned char> tmp4;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb4, cnt.p, crp.p, M + 1, st);
  if (e == cudaSuccess) e = tmp4.alloc(tb4, st);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp4.p, tb4, cnt.p, crp.p, M + 1, st);
  int64_t nnz = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nnz, crp.p + M, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hs, status.p, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return from_cuda(e);
  if (hs == kSpBadIndex) return B2_INVALID_INDEX;
  if (hs == kSpBadRowptr) return B2_INVALID_ROWPTR;
  plan.nnz = nnz;
  plan.crp = crp.release();
  plan.off = off.release();
  plan.tcol = tcol.release();
  plan.tval = tval.release();
  return B2_SUCCESS;
}

// Scratch slots -> caller-visible outputs (stream-ordered).
template <typename T>
cudaError_t fill(const SpPlan& plan, int64_t* crp, int32_t* cci, T* cv, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(crp, plan.crp, (size_t)(plan.M + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && plan.nnz > 0) {
    k_compact<T><<<grid_rows(plan.M), 256, 0, st>>>(plan.M, plan.off, plan.crp, plan.tcol, (const T*)plan.tval,
                                                    cci, cv);
    e = cudaGetLastError();
  }
  return e;
}

// The reference's one-call form: outputs cudaMalloc'd here, freed by the caller.
template <typename T>
b2_status spgemm(const b2_csr* A, const b2_csr* B, int64_t** dC_rowptr, int32_t** dC_colind, T** dC_values,
                 int64_t* hC_nnz, cudaStream_t st) {
  if (!dC_rowptr || !dC_colind || !dC_values || !hC_nnz) return B2_INVALID_ARGUMENT;
  *dC_rowptr = nullptr;
  *dC_colind = nullptr;
  *dC_values = nullptr;
  *hC_nnz = 0;
  SpPlan plan;
  b2_status s = compute<T>(A, B, st, plan);
  if (s != B2_SUCCESS) {
    plan.release();
    return s;
  }
  int64_t* crp = nullptr;
  int32_t* cci = nullptr;
  T* cv = nullptr;
  cudaError_t e = cudaMalloc((void**)&crp, (size_t)(plan.M + 1) * sizeof(int64_t));
  if (e == cudaSuccess && plan.nnz > 0) e = cudaMalloc((void**)&cci, (size_t)plan.nnz * sizeof(int32_t));
  if (e == cudaSuccess && plan.nnz > 0) e = cudaMalloc((void**)&cv, (size_t)plan.nnz * sizeof(T));
  if (e == cudaSuccess) e = fill<T>(plan, crp, cci, cv, st);
  plan.release();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(crp);
    cudaFree(cci);
    cudaFree(cv);
    return e == cudaErrorMemoryAllocation ? B2_OUT_OF_MEMORY : from_cuda(e);
  }
  *dC_rowptr = crp;
  *dC_colind = cci;
  *dC_values = cv;
  *hC_nnz = plan.nnz;
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

extern "C" b2_status b2_minplus_spgemm_plan(const b2_csr* A, const b2_csr* B, b2_stream stream,
                                            b2_spgemm_plan* plan, int64_t* hC_nnz) {
  if (!A || !B || !plan || !hC_nnz) return B2_INVALID_ARGUMENT;
  *plan = nullptr;
  *hC_nnz = 0;
  if (A->weight_type != B->weight_type) return B2_INVALID_ARGUMENT;
  b2::SpPlan* p = new b2::SpPlan();
  p->wt = A->weight_type;
  const b2_status s = A->weight_type == B2_W_F32 ? b2::compute<float>(A, B, (cudaStream_t)stream, *p)
                                                  : b2::compute<int32_t>(A, B, (cudaStream_t)stream, *p);
  if (s != B2_SUCCESS) {
    p->release();
    delete p;
    return s;
  }
  *plan = reinterpret_cast<b2_spgemm_plan>(p);
  *hC_nnz = p->nnz;
  return B2_SUCCESS;
}

extern "C" b2_status b2_minplus_spgemm_fill(b2_spgemm_plan plan, int64_t* dC_rowptr, int32_t* dC_colind,
                                            void* dC_values, b2_stream stream) {
  b2::SpPlan* p = reinterpret_cast<b2::SpPlan*>(plan);
  if (!p || !dC_rowptr || (p->nnz > 0 && (!dC_colind || !dC_values))) return B2_INVALID_ARGUMENT;
  const cudaStream_t st = (cudaStream_t)stream;
  p->st = st;   // scratch is released in the order of this stream
  const cudaError_t e = p->wt == B2_W_F32 ? b2::fill<float>(*p, dC_rowptr, dC_colind, (float*)dC_values, st)
                                          : b2::fill<int32_t>(*p, dC_rowptr, dC_colind, (int32_t*)dC_values, st);
  p->release();
  delete p;
  return b2::from_cuda(e);
}

extern "C" b2_status b2_minplus_spgemm_plan_free(b2_spgemm_plan plan) {
  b2::SpPlan* p = reinterpret_cast<b2::SpPlan*>(plan);
  if (!p) return B2_INVALID_ARGUMENT;
  p->release();
  delete p;
  return B2_SUCCESS;
}
