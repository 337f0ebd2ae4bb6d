// Relaxation building blocks shared by the persistent SSSP kernels (the
// bulk-synchronous delta-stepping / Bellman-Ford kernel and the asynchronous
// ADDS worklist kernel): label words, L2-resident label loads and atomics,
// warp bit tricks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "b2_common.cuh"
#include "b2_internal.hpp"

namespace b2 {

// Publish a finished round / bucket to the mapped progress record (one
// thread; `rounds` is stored last with a system-scope release).
__device__ __forceinline__ void publish_progress(ProgressBoard* b, uint32_t rounds, uint32_t changed,
                                                 unsigned long long t_ns) {
  if (!b) return;
  *(volatile uint32_t*)&b->changed = changed;
  *(volatile unsigned long long*)&b->t_ns = t_ns;
  __threadfence_system();
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(&b->rounds), "r"(rounds) : "memory");
}

// ---------------------------------------------------------------------------
// label access
template <bool PRED>
struct Label;
template <>
struct Label<false> {
  using T = uint32_t;
  __device__ __forceinline__ static uint32_t key(T w) { return w; }
  __device__ __forceinline__ static T make(uint32_t key, uint32_t) { return key; }
  static constexpr T kInf = 0xFFFFFFFFu;
};
template <>
struct Label<true> {
  using T = unsigned long long;
  __device__ __forceinline__ static uint32_t key(T w) { return (uint32_t)(w >> 32); }
  __device__ __forceinline__ static T make(uint32_t key, uint32_t pred) {
    return ((unsigned long long)key << 32) | pred;
  }
  static constexpr T kInf = 0xFFFFFFFFFFFFFFFFull;
};

// Label loads and atomics carry an L2 evict_last policy: the label array is
// read once per relaxed edge at random, so it must stay resident while the
// edge stream (evict-first loads) flows through L2.
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint32_t ld_keep(const uint32_t* a, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.cg.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_keep(const unsigned long long* a, uint64_t pol) {
  unsigned long long v;
  asm volatile("ld.global.cg.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(a), "l"(pol) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t atom_min_keep(uint32_t* a, uint32_t x, uint64_t pol) {
  uint32_t old;
  asm volatile("atom.global.L2::cache_hint.min.u32 %0, [%1], %2, %3;" : "=r"(old) : "l"(a), "r"(x), "l"(pol) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long atom_min_keep(unsigned long long* a, unsigned long long x, uint64_t pol) {
  unsigned long long old;
  asm volatile("atom.global.L2::cache_hint.min.u64 %0, [%1], %2, %3;" : "=l"(old) : "l"(a), "l"(x), "l"(pol) : "memory");
  return old;
}

// Predicated forms: the access is made only when `p` holds (the result is then
// `dflt`), with no branch around it, so a loop can issue the accesses of all
// its edge slots before it reads any result and their L2 round trips overlap.
__device__ __forceinline__ uint32_t ld_keep_if(bool p, const uint32_t* a, uint64_t pol, uint32_t dflt) {
  uint32_t v = dflt;
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t"
               "@q ld.global.cg.L2::cache_hint.u32 %0, [%1], %2;\n\t}"
               : "+r"(v) : "l"(a), "l"(pol), "r"((uint32_t)p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_keep_if(bool p, const unsigned long long* a, uint64_t pol,
                                                         unsigned long long dflt) {
  unsigned long long v = dflt;
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t"
               "@q ld.global.cg.L2::cache_hint.u64 %0, [%1], %2;\n\t}"
               : "+l"(v) : "l"(a), "l"(pol), "r"((uint32_t)p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t atom_min_keep_if(bool p, uint32_t* a, uint32_t x, uint64_t pol, uint32_t dflt) {
  uint32_t old = dflt;
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %4, 0;\n\t"
               "@q atom.global.L2::cache_hint.min.u32 %0, [%1], %2, %3;\n\t}"
               : "+r"(old) : "l"(a), "r"(x), "l"(pol), "r"((uint32_t)p) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long atom_min_keep_if(bool p, unsigned long long* a, unsigned long long x,
                                                               uint64_t pol, unsigned long long dflt) {
  unsigned long long old = dflt;
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %4, 0;\n\t"
               "@q atom.global.L2::cache_hint.min.u64 %0, [%1], %2, %3;\n\t}"
               : "+l"(old) : "l"(a), "l"(x), "l"(pol), "r"((uint32_t)p) : "memory");
  return old;
}
__device__ __forceinline__ uint32_t atom_min_if(bool p, uint32_t* a, uint32_t x, uint32_t dflt) {
  uint32_t old = dflt;
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t@q atom.global.min.u32 %0, [%1], %2;\n\t}"
               : "+r"(old) : "l"(a), "r"(x), "r"((uint32_t)p) : "memory");
  return old;
}
__device__ __forceinline__ uint32_t atom_exch_if(bool p, uint32_t* a, uint32_t x, uint32_t dflt) {
  uint32_t old = dflt;
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t@q atom.global.exch.b32 %0, [%1], %2;\n\t}"
               : "+r"(old) : "l"(a), "r"(x), "r"((uint32_t)p) : "memory");
  return old;
}

__device__ __forceinline__ uint32_t lanemask_le() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}

// Position of the (k+1)-th set bit of `mask` (k < popc(mask)); pure register
// arithmetic, 5 halving steps.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t mask, uint32_t k) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t step = 16; step >= 1; step >>= 1) {
    const uint32_t lowcnt = __popc(mask & ((1u << (pos + step)) - 1u));   // bits below pos+step
    if (lowcnt <= k) pos += step;
  }
  return pos;
}

__device__ __forceinline__ unsigned long long shfl64(unsigned long long x, uint32_t src) {
  const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)x, src);
  const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(x >> 32), src);
  return ((unsigned long long)hi << 32) | lo;
}

}  // namespace b2
