// Device-side building blocks shared by the SSSP, min-plus and serving kernels.
//
// Distance words.  Every SSSP kernel keeps a vertex label in an unsigned word
// that is ordered exactly like the distance it encodes, so a single hardware
// atomicMin performs the relaxation (no CAS loop as in the reference's
// atomic_min_float_nonnegative, HIP_kernel/delta_stepping/src/delta_stepping_hip_CSR.cpp:222-231):
//   * uint32 weights: the word is the distance, INF = 0xFFFFFFFF, and addition
//     saturates to INF on overflow (the reference's DistanceOps<uint32_t>::add,
//     faster_GPU_algo/jasper_oneshot_untested/hip_adds_sssp.cpp:200-213);
//   * float weights: the word is the IEEE bit pattern with the sign bit
//     flipped for positives and all bits flipped for negatives, a bijection
//     that is monotone over all non-NaN floats, so negative Bellman-Ford
//     weights still order correctly.
// With predecessors the label is the 64-bit word (key << 32) | pred, so one
// 64-bit atomicMin updates distance and predecessor together; among equal
// distances the smallest predecessor id wins, which makes pred deterministic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace b2 {

constexpr uint32_t kInfKey = 0xFFFFFFFFu;      // unreachable, both weight types
constexpr uint32_t kNoPred = 0xFFFFFFFFu;
constexpr uint32_t kNoBucket = 0x3fffffffu;    // reference kNoBucket (delta_stepping_hip_CSR.cpp:22)

// ---- error codes written to the control block (host maps them to b2_status)
enum DeviceError : uint32_t {
  kErrNone = 0,
  kErrTimeout = 1,
  kErrQueueOverflow = 2,
  kErrBadIndex = 3,
};

__device__ __forceinline__ uint32_t f32_to_key(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_to_f32(uint32_t k) {
  uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(b);
}

// Weight traits: how a stored edge weight extends a distance key.
struct WU32 {
  static constexpr bool kFloat = false;
  __device__ __forceinline__ static uint32_t zero_key() { return 0u; }
  __device__ __forceinline__ static uint32_t extend(uint32_t key, uint32_t w) {
    uint32_t s = key + w;
    return (s < key) ? kInfKey : s;   // saturating; INF + w stays INF
  }
  __device__ __forceinline__ static bool negative(uint32_t) { return false; }
};

struct WF32 {
  static constexpr bool kFloat = true;
  __device__ __forceinline__ static uint32_t zero_key() { return f32_to_key(0.0f); }
  __device__ __forceinline__ static uint32_t extend(uint32_t key, uint32_t wbits) {
    if (key == kInfKey) return kInfKey;
    float d = key_to_f32(key) + __uint_as_float(wbits);   // IEEE round-to-nearest
    // NaN or an overflow to +inf means "not reached", matching a float
    // Dijkstra whose unreachable label is +inf.
    if (d != d || d == __int_as_float(0x7f800000)) return kInfKey;
    return f32_to_key(d);
  }
};
// +inf encodes to 0xFF800000 under f32_to_key; the solvers use kInfKey for
// "never reached" and translate at the output boundary, so reached-with-+inf
// cannot be confused with unreached (finite weights are validated on input).

// ---- bounded waits -------------------------------------------------------
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// L2-coherent loads for data that other SMs modify between phases (L1 is not
// coherent across SMs, so a plain load could return a line cached in an
// earlier phase).
template <typename T>
__device__ __forceinline__ T ldcg(const T* p) { return __ldcg(p); }

// ---- grid barrier with a serial manager step ------------------------------
// All blocks of a cooperative (co-resident) grid arrive; the LAST block to
// arrive runs `manager()` on one thread while every other block is parked,
// then releases them.  The manager may therefore read and reset any counter
// without racing with producers or consumers.  Every wait is bounded by
// `budget_ns` of globaltimer; on expiry the waiting block records kErrTimeout
// and returns false, and so do all later barriers (the error word is sticky).
struct GridBarrier {
  uint32_t arrive;    // arrivals in the current generation
  uint32_t gen;       // generation counter (release word)
  uint32_t error;     // sticky DeviceError
  uint32_t error_site;
};

template <typename Manager>
__device__ __forceinline__ bool grid_barrier(GridBarrier* bar, uint32_t nblocks, uint64_t budget_ns,
                                             Manager&& manager) {
  __shared__ uint32_t s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    const uint32_t my_gen = ld_relaxed_u32(&bar->gen);
    __threadfence();
    const uint32_t arrived = atomicAdd(&bar->arrive, 1u);
    if (arrived == nblocks - 1) {
      // Last arriver: everybody else has finished the phase.
      __threadfence();
      bar->arrive = 0;
      if (ld_relaxed_u32(&bar->error) == kErrNone) manager();
      __threadfence();
      st_release_u32(&bar->gen, my_gen + 1);
    } else {
      const uint64_t t0 = globaltimer_ns();
      uint32_t spins = 0;
      while (ld_acquire_u32(&bar->gen) == my_gen) {
        if (((++spins) & 63u) == 0) {
          if (ld_relaxed_u32(&bar->error) != kErrNone) { ok = 0; break; }
          if (globaltimer_ns() - t0 > budget_ns) {
            atomicCAS(&bar->error, kErrNone, (uint32_t)kErrTimeout);
            atomicExch(&bar->error_site, 1u);
            ok = 0;
            break;
          }
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    if (ld_relaxed_u32(&bar->error) != kErrNone) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---- warp helpers ---------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  return x;
}

// Warp-aggregated append: every active lane with `want` set gets a distinct
// slot in a queue counted by `*count`; one atomic per warp.
__device__ __forceinline__ uint32_t warp_append(uint32_t* count, bool want) {
  const uint32_t active = __activemask();
  const uint32_t ballot = __ballot_sync(active, want);
  if (ballot == 0) return 0xFFFFFFFFu;
  const uint32_t lane = lane_id();
  const uint32_t leader = __ffs(ballot) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(ballot));
  base = __shfl_sync(active, base, leader);
  return want ? base + __popc(ballot & ((1u << lane) - 1u)) : 0xFFFFFFFFu;
}

}  // namespace b2
