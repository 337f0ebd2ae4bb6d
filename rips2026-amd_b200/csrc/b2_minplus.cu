// Dense min-plus (tropical) GEMM  C[i,j] = min_k A[i,k] + B[k,j]  and the
// APSP repeated-squaring driver.
//
// Tensor cores cannot evaluate (min,+), so the math runs on the CUDA cores:
//   int32 : one DPX __viaddmin_s32 (add + min fused) per (i,j,k) pair;
//   fp32  : FADD per pair and a three-input min.f32 per two pairs.
// Data movement is TMA: each k-tile of A (128 rows x 32 k, 128-byte swizzle)
// and B (32 k x 128 cols) lands in shared memory through
// cp.async.bulk.tensor with an mbarrier transaction count, three stages deep,
// issued by one thread; 256 threads each own an 8 x 8 block of C and read
// their A fragments as float4 along k (swizzle makes the two row groups of a
// warp hit different banks) and B fragments as float4 along n.
//
// Semantics follow minplus_kernel_f32 (HIP_kernel/minplus_mm/src/minplus_hip.cpp:13-118):
// accumulators start at +inf and a NaN candidate never replaces the
// accumulator.  The int32 twin (no reference counterpart) starts at
// INT32_MAX/2 = 1073741823 (the "missing" sentinel), so results are clamped to
// it; inputs must lie in [-2^30, 2^30-1] so no sum overflows.
// Partial k-tiles are bounded by a uniform loop limit, so TMA's out-of-range
// fill value never enters a minimum.  Operands that TMA cannot describe
// (unaligned base or leading dimension) take a plain-load kernel with the same
// tiling.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <type_traits>

#include "b2_common.cuh"
#include "b2_internal.hpp"

namespace b2 {
namespace {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, NT = 256;
constexpr int A_TILE = BM * BK;   // elements
constexpr int B_TILE = BK * BN;
constexpr int kMissing = 1073741823;

// Set by a bounded mbarrier wait that gave up.  One word per device: every
// product clears it in stream order before its launch (clear_mp_error), APSP
// reads it back after its last product, and b2_minplus_status reads it for
// the asynchronous GEMM.  Products that overlap on different streams of one
// device share the word.
__device__ uint32_t g_mp_error;

template <typename T>
struct MP;
template <>
struct MP<float> {
  __device__ __forceinline__ static float init() { return __int_as_float(0x7f800000); }
  // acc = min(acc, a + b0, a + b1)
  __device__ __forceinline__ static float step2(float acc, float a0, float b0, float a1, float b1) {
    const float x = a0 + b0, y = a1 + b1;
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(acc), "f"(x), "f"(y));
    return r;
  }
  __device__ __forceinline__ static float step1(float acc, float a, float b) { return fminf(acc, a + b); }
  static constexpr bool kTwoPerMin = true;   // one 3-input min per two pairs
};
template <>
struct MP<int> {
  __device__ __forceinline__ static int init() { return kMissing; }
  __device__ __forceinline__ static int step2(int acc, int a0, int b0, int a1, int b1) {
    return __viaddmin_s32(a1, b1, __viaddmin_s32(a0, b0, acc));
  }
  __device__ __forceinline__ static int step1(int acc, int a, int b) { return __viaddmin_s32(a, b, acc); }
  static constexpr bool kTwoPerMin = false;  // one fused add+min per pair
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after ~2^22 polls (each poll may suspend), records the
// failure and lets the kernel run to completion instead of hanging.
__device__ __forceinline__ void mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < (1u << 22); ++i)
    if (mbar_try_wait(bar, parity)) return;
  atomicExch(&g_mp_error, 1u);
}
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(smem_dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Tile order: groups of 8 tile-rows share B panels in L2.
__device__ __forceinline__ void tile_coords(int tiles_m, int tiles_n, int& tm, int& tn) {
  const int id = blockIdx.x;
  const int group = 8;
  const int per_group = group * tiles_n;
  const int g = id / per_group;
  const int first_m = g * group;
  const int gsz = min(tiles_m - first_m, group);
  const int in = id - g * per_group;
  tm = first_m + in % gsz;
  tn = in / gsz;
}

// Compute one k-tile held in shared memory (A swizzled, B plain).  A is read
// as k-pairs (8-byte loads inside the swizzled 16-byte chunk), B as two
// 16-byte vectors per k row.
template <typename T>
__device__ __forceinline__ void load_b8(const T* Bs, int k, int tx, T (&b)[8]) {
  const int4 p0 = *reinterpret_cast<const int4*>(Bs + k * BN + tx * 4);
  const int4 p1 = *reinterpret_cast<const int4*>(Bs + k * BN + 64 + tx * 4);
  const int pp[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
  for (int j = 0; j < 8; ++j) b[j] = *reinterpret_cast<const T*>(&pp[j]);
}

template <typename T, bool FULL>
__device__ __forceinline__ void mma_tile(const T* __restrict__ As, const T* __restrict__ Bs, int kvalid, int tx,
                                         int ty, T (&acc)[8][8]) {
  const int sw = ty & 7;
#pragma unroll
  for (int k = 0; k < BK; k += 2) {
    if (!FULL && k >= kvalid) break;
    T a0[8], a1[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = ty + 16 * i;
      const int2 v = *reinterpret_cast<const int2*>(As + r * BK + (((k >> 2) ^ sw) << 2) + (k & 2));
      a0[i] = *reinterpret_cast<const T*>(&v.x);
      a1[i] = *reinterpret_cast<const T*>(&v.y);
    }
    T b0[8], b1[8];
    load_b8<T>(Bs, k, tx, b0);
    if (FULL || k + 1 < kvalid) {
      load_b8<T>(Bs, k + 1, tx, b1);
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = MP<T>::step2(acc[i][j], a0[i], b0[j], a1[i], b1[j]);
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = MP<T>::step1(acc[i][j], a0[i], b0[j]);
    }
  }
}

template <typename T>
__device__ __forceinline__ void store_tile(T* C, int M, int N, int ldc, int m0, int n0, int tx, int ty,
                                           const T (&acc)[8][8], const T* Aold, int lda, uint32_t* changed) {
  bool diff = false;
  const bool vec = ((ldc & 3) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = m0 + ty + 16 * i;
    if (r >= M) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c0 = n0 + h * 64 + tx * 4;
      if (vec && c0 + 3 < N) {
        int4 v;
        v.x = *reinterpret_cast<const int*>(&acc[i][h * 4 + 0]);
        v.y = *reinterpret_cast<const int*>(&acc[i][h * 4 + 1]);
        v.z = *reinterpret_cast<const int*>(&acc[i][h * 4 + 2]);
        v.w = *reinterpret_cast<const int*>(&acc[i][h * 4 + 3]);
        *reinterpret_cast<int4*>(C + (size_t)r * ldc + c0) = v;
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (c0 + q < N) C[(size_t)r * ldc + c0 + q] = acc[i][h * 4 + q];
      }
      if (Aold) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (c0 + q < N) {
            const T o = Aold[(size_t)r * lda + c0 + q];
            diff |= (*reinterpret_cast<const int*>(&o) != *reinterpret_cast<const int*>(&acc[i][h * 4 + q]));
          }
      }
    }
  }
  if (Aold && __any_sync(0xffffffffu, diff) && (threadIdx.x & 31) == 0) atomicExch(changed, 1u);
}

// TMA pipeline kernel.  `Aold` (nullable): compare results against it and set
// *changed (APSP squaring, where C <= A elementwise because diag(A) = 0).
template <typename T>
__global__ void __launch_bounds__(NT, 2)
    k_minplus_tma(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, T* C, int M,
                  int N, int K, int ldc, const T* Aold, int lda, uint32_t* changed) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  T* As = reinterpret_cast<T*>(base);
  T* Bs = As + STAGES * A_TILE;
  uint64_t* full = reinterpret_cast<uint64_t*>(Bs + STAGES * B_TILE);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  int tm, tn;
  tile_coords((M + BM - 1) / BM, (N + BN - 1) / BN, tm, tn);
  const int m0 = tm * BM, n0 = tn * BN;
  const int KT = (K + BK - 1) / BK;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < STAGES && s < KT; ++s) {
      mbar_expect_tx(&full[s], (A_TILE + B_TILE) * sizeof(T));
      tma_load_2d(As + s * A_TILE, &mapA, s * BK, m0, &full[s]);
      tma_load_2d(Bs + s * B_TILE, &mapB, n0, s * BK, &full[s]);
    }
  }
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = MP<T>::init();
  for (int kt = 0; kt < KT; ++kt) {
    const int s = kt % STAGES;
    mbar_wait(&full[s], (kt / STAGES) & 1);
    const int kvalid = min(BK, K - kt * BK);
    if (kvalid == BK) mma_tile<T, true>(As + s * A_TILE, Bs + s * B_TILE, BK, tx, ty, acc);
    else mma_tile<T, false>(As + s * A_TILE, Bs + s * B_TILE, kvalid, tx, ty, acc);
    __syncthreads();   // every thread is done with stage s
    if (tid == 0 && kt + STAGES < KT) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&full[s], (A_TILE + B_TILE) * sizeof(T));
      tma_load_2d(As + s * A_TILE, &mapA, (kt + STAGES) * BK, m0, &full[s]);
      tma_load_2d(Bs + s * B_TILE, &mapB, n0, (kt + STAGES) * BK, &full[s]);
    }
  }
  store_tile<T>(C, M, N, ldc, m0, n0, tx, ty, acc, Aold, lda, changed);
}

// Plain-load twin for operands TMA cannot address (same tiling, same math).
template <typename T>
__global__ void __launch_bounds__(NT, 2)
    k_minplus_plain(const T* __restrict__ A, const T* __restrict__ B, T* C, int M, int N, int K, int lda, int ldb,
                    int ldc, const T* Aold, uint32_t* changed) {
  __shared__ __align__(16) T As[A_TILE];
  __shared__ __align__(16) T Bs[B_TILE];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  int tm, tn;
  tile_coords((M + BM - 1) / BM, (N + BN - 1) / BN, tm, tn);
  const int m0 = tm * BM, n0 = tn * BN;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = MP<T>::init();
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int idx = tid; idx < A_TILE; idx += NT) {
      const int r = idx / BK, k = idx % BK;
      const int gr = m0 + r, gk = k0 + k;
      const T v = (gr < M && gk < K) ? A[(size_t)gr * lda + gk] : MP<T>::init();
      As[r * BK + (((k >> 2) ^ (r & 7)) << 2) + (k & 3)] = v;   // same swizzle as TMA
    }
    for (int idx = tid; idx < B_TILE; idx += NT) {
      const int k = idx / BN, c = idx % BN;
      const int gk = k0 + k, gc = n0 + c;
      Bs[idx] = (gk < K && gc < N) ? B[(size_t)gk * ldb + gc] : MP<T>::init();
    }
    __syncthreads();
    const int kvalid = min(BK, K - k0);
    if (kvalid == BK) mma_tile<T, true>(As, Bs, BK, tx, ty, acc);
    else mma_tile<T, false>(As, Bs, kvalid, tx, ty, acc);
    __syncthreads();
  }
  store_tile<T>(C, M, N, ldc, m0, n0, tx, ty, acc, Aold, lda, changed);
}

// ---- host ----------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

template <typename T>
bool make_map(CUtensorMap* map, const T* ptr, int rows, int cols, int ld, int box_cols, int box_rows, bool swz) {
  auto fn = encode_fn();
  if (!fn) return false;
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) || ((size_t)ld * sizeof(T)) % 16) return false;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(T)};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt =
      sizeof(T) == 4 && std::is_same<T, float>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_INT32;
  CUresult r = fn(map, dt, 2, const_cast<T*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  swz ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

constexpr size_t kTmaSmem = (size_t)STAGES * (A_TILE + B_TILE) * 4 + STAGES * 8 + 1024;

// Host-side state kept per device: the TMA kernels' dynamic shared-memory
// attribute is a per-device setting, and the error word's device address is
// looked up with that device current.
constexpr int kMaxDevices = 64;
struct DeviceState {
  bool attr_f32 = false;
  bool attr_i32 = false;
  uint32_t* err = nullptr;
};
std::mutex g_dev_mu;
DeviceState g_dev[kMaxDevices];

cudaError_t current_state(DeviceState** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  *out = &g_dev[dev];
  return cudaSuccess;
}

template <typename T>
cudaError_t ensure_smem_attr() {
  DeviceState* d = nullptr;
  cudaError_t e = current_state(&d);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_dev_mu);
  bool& done = std::is_same<T, float>::value ? d->attr_f32 : d->attr_i32;
  if (!done) {
    e = cudaFuncSetAttribute(k_minplus_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaSmem);
    if (e != cudaSuccess) return e;
    done = true;
  }
  return cudaSuccess;
}

// Device address of g_mp_error on the current device.
cudaError_t mp_error_ptr(uint32_t** out) {
  DeviceState* d = nullptr;
  cudaError_t e = current_state(&d);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_dev_mu);
  if (!d->err) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_mp_error);
    if (e != cudaSuccess) return e;
    d->err = (uint32_t*)p;
  }
  *out = d->err;
  return cudaSuccess;
}

// Stream-ordered clear of the error word (allocates nothing).
cudaError_t clear_mp_error(cudaStream_t st) {
  uint32_t* p = nullptr;
  cudaError_t e = mp_error_ptr(&p);
  if (e != cudaSuccess) return e;
  return cudaMemsetAsync(p, 0, sizeof(uint32_t), st);
}

// Wait for the stream, then read the error word: B2_TIMEOUT when a wait of a
// product issued since the last clear gave up.
b2_status read_mp_error(cudaStream_t st) {
  uint32_t* p = nullptr;
  B2_CUDA_TRY(mp_error_ptr(&p));
  uint32_t err = 0;
  B2_CUDA_TRY(cudaMemcpyAsync(&err, p, sizeof(err), cudaMemcpyDeviceToHost, st));
  B2_CUDA_TRY(cudaStreamSynchronize(st));
  return err ? B2_TIMEOUT : B2_SUCCESS;
}

template <typename T>
cudaError_t launch_minplus(const T* A, const T* B, T* C, int M, int N, int K, int lda, int ldb, int ldc,
                           cudaStream_t st, const T* Aold, uint32_t* changed) {
  const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  CUtensorMap ma, mb;
  const bool tma = make_map<T>(&ma, A, M, K, lda, BK, BM, true) && make_map<T>(&mb, B, K, N, ldb, BN, BK, false);
  if (tma) {
    cudaError_t ea = ensure_smem_attr<T>();
    if (ea != cudaSuccess) return ea;
    k_minplus_tma<T><<<tiles, NT, kTmaSmem, st>>>(ma, mb, C, M, N, K, ldc, Aold, lda, changed);
  } else {
    k_minplus_plain<T><<<tiles, NT, 0, st>>>(A, B, C, M, N, K, lda, ldb, ldc, Aold, changed);
  }
  return cudaGetLastError();
}

template <typename T>
b2_status gemm(const T* A, const T* B, T* C, int M, int N, int K, int lda, int ldb, int ldc, b2_stream s) {
  // argument rules of minplus_gemm_f32 (minplus_hip.cpp:132-142)
  if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0 || lda < K || ldb < N || ldc < N) return B2_INVALID_ARGUMENT;
  B2_CUDA_TRY(clear_mp_error((cudaStream_t)s));
  return from_cuda(launch_minplus<T>(A, B, C, M, N, K, lda, ldb, ldc, (cudaStream_t)s, nullptr, nullptr));
}

template <typename T>
b2_status apsp(T* D, int N, b2_stream s, int32_t* squarings) {
  if (!D || N <= 0) return B2_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)s;
  if (squarings) *squarings = 0;
  if (N == 1) return B2_SUCCESS;
  B2_CUDA_TRY(clear_mp_error(st));
  T* tmp = nullptr;
  uint32_t* flag = nullptr;
  uint32_t* hflag = nullptr;
  B2_CUDA_TRY(cudaMalloc((void**)&tmp, (size_t)N * N * sizeof(T)));
  cudaError_t e = cudaMalloc((void**)&flag, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&hflag, sizeof(uint32_t));
  int done = 0;
  int maxsq = 0;
  while ((1ll << maxsq) < (long long)(N - 1)) ++maxsq;   // ceil(log2(N-1)) products reach N-1 hops
  T* cur = D;
  T* nxt = tmp;
  for (int it = 0; it < maxsq && e == cudaSuccess; ++it) {
    e = cudaMemsetAsync(flag, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess) e = launch_minplus<T>(cur, cur, nxt, N, N, N, N, N, N, st, cur, flag);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hflag, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) break;
    ++done;
    std::swap(cur, nxt);
    if (*hflag == 0) break;   // D unchanged: fixpoint reached
  }
  if (e == cudaSuccess && cur != D) {
    e = cudaMemcpyAsync(D, cur, (size_t)N * N * sizeof(T), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  cudaFree(tmp);
  cudaFree(flag);
  if (hflag) cudaFreeHost(hflag);
  if (squarings) *squarings = done;
  if (e != cudaSuccess) return from_cuda(e);
  return read_mp_error(st);
}

// ---- ALU peak calibration (roofline denominator for min-plus) -------------
// The GEMM's own instruction mix on registers only: an 8 x 8 accumulator tile
// per thread updated per k step exactly like mma_tile (int32: one
// __viaddmin_s32 per pair; fp32: two FADD and one 3-input min per two pairs),
// with no shared-memory or global traffic.  The A operand of row i at step k
// is an accumulator of that row (acc[i][(i + k) & 7], a register chosen at
// compile time), so every sum is a new value and no sum can be folded or
// shared between pairs; B is 8 (16 for fp32) runtime constants.  The pair
// count over the device time is the instruction-issue ceiling of the mix.
template <typename T>
__global__ void __launch_bounds__(256) k_calibrate(int iters, T seed, T step, T* sink) {
  T acc[8][8];
  T b0[8], b1[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    b0[j] = step + (T)j;
    b1[j] = step + (T)(j + 8);
  }
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = seed + (T)(threadIdx.x + 8 * i + j);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const T a0 = acc[i][(i + k) & 7];
        const T a1 = acc[i][(i + k + 3) & 7];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (sizeof(T) == 4 && MP<T>::kTwoPerMin) acc[i][j] = MP<T>::step2(acc[i][j], a0, b0[j], a1, b1[j]);
          else acc[i][j] = MP<T>::step1(acc[i][j], a0, b0[j]);
        }
      }
    }
  }
  T r = acc[0][0];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) r = r < acc[i][j] ? r : acc[i][j];
  if (r == (T)-12345) sink[0] = r;
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" b2_status b2_minplus_gemm_f32(const float* dA, const float* dB, float* dC, int32_t M, int32_t N,
                                         int32_t K, int32_t lda, int32_t ldb, int32_t ldc, b2_stream stream) {
  return gemm<float>(dA, dB, dC, M, N, K, lda, ldb, ldc, stream);
}

extern "C" b2_status b2_minplus_gemm_i32(const int32_t* dA, const int32_t* dB, int32_t* dC, int32_t M, int32_t N,
                                         int32_t K, int32_t lda, int32_t ldb, int32_t ldc, b2_stream stream) {
  return gemm<int>(dA, dB, dC, M, N, K, lda, ldb, ldc, stream);
}

extern "C" b2_status b2_apsp_f32(float* d_D, int32_t N, b2_stream stream, int32_t* sq) {
  return apsp<float>(d_D, N, stream, sq);
}

extern "C" b2_status b2_apsp_i32(int32_t* d_D, int32_t N, b2_stream stream, int32_t* sq) {
  return apsp<int>(d_D, N, stream, sq);
}

extern "C" b2_status b2_minplus_status(b2_stream stream) {
  return read_mp_error((cudaStream_t)stream);
}

extern "C" b2_status b2_minplus_calibrate(int32_t is_float, double* pairs_per_second) {
  if (!pairs_per_second) return B2_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256, blocks = sms * 4, iters = 1 << 12;
  void* sink = nullptr;
  B2_CUDA_TRY(cudaMalloc(&sink, 16));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    if (is_float) k_calibrate<float><<<blocks, threads>>>(iters, 0.5f, 0.25f, (float*)sink);
    else k_calibrate<int><<<blocks, threads>>>(iters, 3, 1, (int*)sink);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) return from_cuda(e);
  // per thread and iteration: 8 k steps x 64 updates; an fp32 update is two pairs
  const double pairs = (double)blocks * threads * iters * 8.0 * 64.0 * (is_float ? 2.0 : 1.0);
  *pairs_per_second = pairs / (best * 1e-3);
  return B2_SUCCESS;
}

// ---- allocation-free APSP --------------------------------------------------
// Some callers cannot allocate device memory while they run:
//   * a plugin inside a host whose device memory is owned by another
//     allocator (a framework's caching pool), where a cudaMalloc would
//     fragment or exceed that pool's budget;
//   * a latency-bound serving loop with a fixed memory budget, where
//     cudaMalloc / cudaFree would synchronize the device and add jitter;
//   * code running while a device-wide allocation freeze is in effect.
// b2_apsp_f32_noalloc runs the same repeated squaring as b2_apsp_f32, but its
// ping-pong matrix and change flag live in the fixed array below instead of a
// cudaMalloc'd buffer.  Limits and rules:
//   * N * N * 4 bytes must fit in the array (N <= 2048); larger N is rejected
//     with B2_NOT_SUPPORTED before anything runs;
//   * the array is a module global: every GPU that loads this library holds
//     its 16 MiB until the process exits;
//   * every call on a device shares the one array, and it keeps the previous
//     call's contents (the change flag is cleared before each product): calls
//     that overlap on the GPU (different streams or threads) race and must be
//     serialized by the caller;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
namespace b2 {
namespace {
constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;   // 16 MiB: 2048 x 2048 floats
// scratch matrix, then the change flag in the last 256 bytes
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes + 256];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {};

// Device address of g_noalloc_scratch for the current device (looked up once
// per device; the host-side symbol itself is not a device address).
cudaError_t noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
  }
  *out = (unsigned char*)g_noalloc_ptr[dev];
  return cudaSuccess;
}
}  // namespace
}  // namespace b2

extern "C" b2_status b2_apsp_f32_noalloc(float* d_D, int32_t N, b2_stream stream, int32_t* squarings) {
  using namespace b2;
  if (!d_D || N <= 0) return B2_INVALID_ARGUMENT;
  if ((size_t)N * (size_t)N * sizeof(float) > kNoAllocScratchBytes) return B2_NOT_SUPPORTED;
  cudaStream_t st = (cudaStream_t)stream;
  if (squarings) *squarings = 0;
  if (N == 1) return B2_SUCCESS;
  unsigned char* base = nullptr;
  B2_CUDA_TRY(noalloc_scratch(&base));
  B2_CUDA_TRY(clear_mp_error(st));
  float* tmp = (float*)base;
  uint32_t* flag = (uint32_t*)(base + kNoAllocScratchBytes);
  int maxsq = 0;
  while ((1ll << maxsq) < (long long)(N - 1)) ++maxsq;
  float* cur = d_D;
  float* nxt = tmp;
  int done = 0;
  cudaError_t e = cudaSuccess;
  for (int it = 0; it < maxsq; ++it) {
    uint32_t hflag = 0;
    e = cudaMemsetAsync(flag, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess) e = launch_minplus<float>(cur, cur, nxt, N, N, N, N, N, N, st, cur, flag);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hflag, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) break;
    ++done;
    std::swap(cur, nxt);
    if (hflag == 0) break;
  }
  if (e == cudaSuccess && cur != d_D) {
    e = cudaMemcpyAsync(d_D, cur, (size_t)N * N * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (squarings) *squarings = done;
  if (e != cudaSuccess) return from_cuda(e);
  return read_mp_error(st);
}
