// Asynchronous ADDS-style worklist SSSP: one persistent launch, no barrier per
// bucket or per phase.
//
// The reference's hip_adds::sssp (faster_GPU_algo/jasper_oneshot_untested/
// hip_adds_sssp.cpp:460-866) runs a manager thread block that hands ranges of
// paged bucket queues to idle worker blocks, and the ADS float port
// (Charlotte_ADS_Float_Attempt/kernel.hip:66-221, wl.h:1833-1915) pushes into
// 32 priority bags with warp-aggregated appends.  Here there is no manager:
// one warp per block claims a range of up to 1024 entries of a bucket (or 32
// hub chunks) with one compare-and-swap and parks it in a shared-memory pool,
// from which the block's warps take 32 entries (or one chunk) at a time.
//
// Worklist.  A window epoch maps kAddsSlots consecutive buckets of width delta
// to slots 0..kAddsSlots-1 (global bucket W + s); keys past the window go to a
// far pile.  Each slot is a ring of position-tagged words with three counters
// on its own cache line: `reserved` (positions writers reserved), `extra` (hub
// chunks its entries spawned) and `done` (entries and chunks finished), plus a
// `claim` word (epoch << 32 | positions claimed).  A bucket is complete when
// done == reserved + extra: every unit of its work is finished, and since a
// relaxation never lowers a key below its source's bucket, nothing can push
// into it again once every lower bucket is complete.
//
// Window state.  One 64-bit head word (epoch << 32 | position) holds the
// lowest bucket not yet retired, or PREP / SPLIT / DONE.  Warps take entries
// from the `active` buckets starting at the head (the reference's dynamic
// active-bucket count, hip_adds_sssp.cpp:609-647, grows here when warps idle
// while later buckets hold work).  An idle warp retires the complete head
// bucket; when the whole window has retired, the warp that wins the
// compare-and-swap to PREP sets up the next epoch (new bucket width from the
// epoch's utilization, the reference's growth 1.5 / shrink 0.75 feedback,
// hip_adds_sssp.hpp:41-56), and every warp helps route the far pile into it.
// Each change is a compare-and-swap of the head word, so a warp holding a
// stale view changes nothing.
//
// Entries.  Ring words start empty (all ones).  A writer reserves positions
// with one atomic per slot group of a warp (__match_any_sync), waits (bounded)
// for the word of the previous lap to be taken, and stores position << 32 |
// vertex; the taker of position p waits for the word tagged p, takes it and
// writes it back to empty, so a finished solve leaves every ring empty.  A
// per-vertex word qb[v] holds the lowest bucket v is queued in and not yet
// taken: a push happens only when it lowers qb[v], and a warp that takes v
// from bucket b expands it unless qb[v] is below b (v then waits in a lower
// bucket with its newer label).  Fences order the label atomic before the qb
// update on the push side and the qb reset before the label read on the take
// side, so an improvement is never left unexpanded.
//
// High-degree vertices are split into chunks of kChunkEdges edges in a ring
// of position-tagged slots that any warp may take (counted in their bucket's
// `extra` before they are published).  Labels and relaxation are those of the bulk-synchronous kernel
// (b2_relax.cuh): 32-bit keys or packed key|pred words, one hardware atomicMin.
// Every wait is bounded by the solve budget; on expiry the kernel records
// kErrTimeout and every warp leaves.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "b2_common.cuh"
#include "b2_internal.hpp"
#include "b2_relax.cuh"

namespace b2 {
namespace {

constexpr int kAThreads = 512;
constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kEmpty = 0xFFFFFFFFu;       // no vertex: a wait gave up
constexpr unsigned long long kEmpty64 = ~0ull; // empty ring word (bucket rings and the hub ring)
constexpr uint32_t kNotQueued = 0xFFFFFFFFu;   // qb[v]: not waiting in any bucket
constexpr uint32_t kGrab = 32;                 // entries a warp takes from its block's pool (one per lane)
constexpr uint32_t kBlockClaimMin = 64;        // entries a block claims from a bucket at once: its share
constexpr uint32_t kBlockClaimMax = 1024;      //   of the bucket's unclaimed entries, within these bounds
constexpr uint32_t kChunkEdges = 256;          // edges per hub chunk
constexpr uint32_t kHubClaim = 32;             // hub chunks a block claims at once
constexpr int kU = 4;                          // edge slots per lane per step

struct AParams {
  uint32_t n;
  uint32_t source;
  const uint64_t* __restrict__ rowptr;
  const uint2* __restrict__ edges;
  void* dist;              // labels (keys, or key|pred words)
  uint32_t* qb;
  uint32_t* farflag;
  unsigned long long* q;   // kAddsSlots window rings of cap tagged words (position << 32 | vertex)
  uint32_t* far;           // the two far piles, cap entries each
  uint32_t cap;
  ulonglong2* hub;         // ring of {position tag, v | (chunk << 5 | slot) << 32}; tag ~0: empty
  uint32_t hub_cap;
  AddsControl* ctl;
  TraceEntry* trace;
  uint32_t is_float;
  uint32_t width_u;        // initial bucket width (uint32 graphs)
  float inv_width;         // 1 / initial width (float graphs)
  uint32_t active0;        // buckets from the head warps may take at the start of an epoch
  uint32_t active_max;     // the active range never widens past this
  uint32_t hub_degree;
  uint32_t adapt;          // adjust the width at every new epoch
  uint32_t adapt_cap;      // entries per bucket that fill the grid once
  uint32_t warm;           // keep the labels in `warm_in` (initialize_distances = false)
  const void* warm_in;     // caller's distances in input ids (warm start)
  unsigned long long budget_ns;
  void* out_dist;
  int32_t* out_pred;
  uint32_t dist_is_out;
  const uint32_t* perm;    // degree-ordered graph: internal -> input id
  const uint32_t* inv;     // input -> internal id
  ProgressBoard* board;    // mapped progress record (null: no progress callback)
};

// The epoch a warp works in; stable while the warp holds claimed work.
struct View {
  uint32_t epoch, W, kbase, dq, dinv, far_sel;
};

struct ATally {
  unsigned long long edges = 0, impr = 0, pushes = 0, entries = 0, chunks = 0;
  uint64_t keep = 0;
};

__device__ __forceinline__ uint32_t ld_vol(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ unsigned long long ld_vol64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void set_err(const AParams& P, uint32_t code, uint32_t site) {
  if (atomicCAS(&P.ctl->error, kErrNone, code) == kErrNone) atomicExch(&P.ctl->error_site, site);
}

__device__ __forceinline__ View read_view(const AddsControl* c) {
  View E;
  E.epoch = ld_acquire_u32(&c->epoch);
  E.W = ld_vol(&c->W);
  E.kbase = ld_vol(&c->kbase);
  E.dq = ld_vol(&c->dq);
  E.dinv = ld_vol(&c->dinv);
  E.far_sel = ld_vol(&c->far_sel);
  return E;
}
__device__ __forceinline__ View bcast(View E) {
  E.epoch = __shfl_sync(kFull, E.epoch, 0);
  E.W = __shfl_sync(kFull, E.W, 0);
  E.kbase = __shfl_sync(kFull, E.kbase, 0);
  E.dq = __shfl_sync(kFull, E.dq, 0);
  E.dinv = __shfl_sync(kFull, E.dinv, 0);
  E.far_sel = __shfl_sync(kFull, E.far_sel, 0);
  return E;
}

// Window slot of a key in the epoch (kAddsSlots: past the window).
template <class W>
__device__ __forceinline__ uint32_t slot_of(const View& E, uint32_t key) {
  if (key == kInfKey) return kAddsSlots;
  if (!W::kFloat) {
    if (key < E.kbase) return 0;
    const uint32_t s = (key - E.kbase) / E.dq;
    return s < (uint32_t)kAddsSlots ? s : (uint32_t)kAddsSlots;
  }
  const float b = floorf((key_to_f32(key) - key_to_f32(E.kbase)) * __uint_as_float(E.dinv));
  if (!(b < (float)kAddsSlots)) return kAddsSlots;   // also NaN
  return b < 0.0f ? 0u : (uint32_t)b;
}

__device__ __forceinline__ unsigned long long* slot_queue(const AParams& P, uint32_t s) {
  return P.q + (size_t)s * P.cap;
}
__device__ __forceinline__ uint32_t* far_queue(const AParams& P, uint32_t f) { return P.far + (size_t)f * P.cap; }
__device__ __forceinline__ unsigned long long ring_word(uint32_t pos, uint32_t v) {
  return ((unsigned long long)pos << 32) | v;
}

// Bounded wait for the entry of ring position `pos` to be written at p; returns
// its vertex (kEmpty: the wait gave up).  The tag keeps a consumer from taking
// the previous lap's entry that still sits in the word.
__device__ uint32_t wait_word(const AParams& P, const unsigned long long* p, uint32_t pos) {
  unsigned long long w = ld_vol64(p);
  if ((uint32_t)(w >> 32) == pos && w != kEmpty64) return (uint32_t)w;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 0;; ++i) {
    __nanosleep(32);
    w = ld_vol64(p);
    if ((uint32_t)(w >> 32) == pos && w != kEmpty64) return (uint32_t)w;
    if ((i & 63u) == 63u) {
      if (ld_vol(&P.ctl->error)) return kEmpty;
      if (globaltimer_ns() - t0 > P.budget_ns) {
        set_err(P, kErrTimeout, 40);
        return kEmpty;
      }
    }
  }
}
// Bounded wait for the hub chunk of ring position `pos`: its tag is stored
// (release) after its entry, so an acquire of the tag makes the entry
// readable.  Returns the entry (kEmpty64: the wait gave up).
__device__ unsigned long long wait_hub(const AParams& P, ulonglong2* slot, unsigned long long pos) {
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 0;; ++i) {
    if (ld_acquire_u64(&slot->x) == pos) return ld_vol64(&slot->y);
    __nanosleep(32);
    if ((i & 63u) == 63u) {
      if (ld_vol(&P.ctl->error)) return kEmpty64;
      if (globaltimer_ns() - t0 > P.budget_ns) {
        set_err(P, kErrTimeout, 41);
        return kEmpty64;
      }
    }
  }
}

// Append the wanting lanes' vertices to window slots (grouped by slot, one
// atomic per group) -- warp-collective.  A slot queue is a ring of `cap`
// 64-bit words: position p lives at p % cap, tagged with p.  Entries still
// unclaimed never exceed the vertices waiting in the bucket (qb[] allows one
// per vertex), so a ring of n words plus the claims in flight holds them; a
// push that finds the ring full records kErrQueueOverflow (B2_POOL_EXHAUSTED).
// The word at p % cap held position p - cap, claimed already; its taker writes
// it back to empty right after reading it, so the writer waits (bounded) for
// that.  Only the taker of p reads a word tagged p, so a slow taker of p - cap
// never sees p's entry and no entry is taken twice or erased.
__device__ __forceinline__ void push_slots(const AParams& P, bool want, uint32_t s, uint32_t v) {
  if (!__any_sync(kFull, want)) return;
  const uint32_t grp = __match_any_sync(kFull, want ? s : 0xFFFFFFFFu);
  if (!want) return;
  const uint32_t leader = __ffs(grp) - 1;
  uint32_t base = 0, claimed = 0;
  if (lane_id() == leader) {
    base = atomicAdd(&P.ctl->slot[s].reserved, (uint32_t)__popc(grp));
    claimed = (uint32_t)ld_vol64(&P.ctl->slot[s].claim);
  }
  base = __shfl_sync(grp, base, leader);
  claimed = __shfl_sync(grp, claimed, leader);
  const uint32_t pos = base + __popc(grp & ((1u << lane_id()) - 1u));
  // blocks may claim this warp's positions before the claim count is read:
  // a negative distance is no overflow
  if ((int32_t)(pos - claimed) >= (int32_t)P.cap) {
    set_err(P, kErrQueueOverflow, 42);
    return;
  }
  unsigned long long* w = slot_queue(P, s) + (pos % P.cap);
  if (ld_vol64(w) != kEmpty64) {   // the previous lap's taker has not written it back yet
    const uint64_t t0 = globaltimer_ns();
    while (ld_vol64(w) != kEmpty64) {
      __nanosleep(64);
      if (ld_vol(&P.ctl->error)) return;
      if (globaltimer_ns() - t0 > P.budget_ns) {
        set_err(P, kErrTimeout, 46);
        return;
      }
    }
  }
  __stcg(w, ring_word(pos, v));
}

// Append to the epoch's far pile -- warp-collective.
__device__ __forceinline__ void push_far(const AParams& P, const View& E, bool want, uint32_t v, uint32_t key) {
  if (!__any_sync(kFull, want)) return;
  const uint32_t pos = warp_append(&P.ctl->far_count[E.far_sel], want);
  if (want) {
    if (pos < P.cap) __stcg(far_queue(P, E.far_sel) + pos, v);
    else set_err(P, kErrQueueOverflow, 43);
  }
  const uint32_t km = __reduce_min_sync(kFull, want ? key : 0xFFFFFFFFu);
  if (lane_id() == 0 && km != 0xFFFFFFFFu) atomicMin(&P.ctl->far_min_key, km);
}

// Relax kU edge slots per lane: label loads, then the label atomics of every
// slot (issued before any result is read), one fence, then the queue marks
// (again all issued first) and the pushes.  A push happens only when it
// lowers qb[v]; the fence makes the label updates visible before their marks.
template <class W, bool PRED>
__device__ __forceinline__ void relax_route(const AParams& P, const View& E, const bool (&act)[kU],
                                            const uint32_t (&src)[kU], const uint32_t (&dsrc)[kU],
                                            const uint2 (&ed)[kU], ATally& t) {
  using L = Label<PRED>;
  typename L::T* lab = (typename L::T*)P.dist;
  uint32_t cand[kU];
  typename L::T cur[kU], old[kU];
  bool imp[kU];
#pragma unroll
  for (int q = 0; q < kU; ++q) {
    cand[q] = act[q] ? W::extend(dsrc[q], ed[q].y) : kInfKey;
    cur[q] = ld_keep_if(cand[q] != kInfKey, lab + ed[q].x, t.keep, L::kInf);
  }
#pragma unroll
  for (int q = 0; q < kU; ++q) {
    const typename L::T cw = L::make(cand[q], src[q]);
    // not issued: old = 0 reads as "no improvement"
    old[q] = atom_min_keep_if(cand[q] != kInfKey && cw < cur[q], lab + ed[q].x, cw, t.keep, (typename L::T)0);
  }
  bool any_imp = false;
#pragma unroll
  for (int q = 0; q < kU; ++q) {
    imp[q] = cand[q] < L::key(old[q]);
    any_imp = any_imp || imp[q];
    t.edges += act[q] ? 1 : 0;
    t.impr += imp[q] ? 1 : 0;
  }
  if (!__any_sync(kFull, any_imp)) return;
  __threadfence();
  uint32_t s[kU], oq[kU];
#pragma unroll
  for (int q = 0; q < kU; ++q) {
    s[q] = imp[q] ? slot_of<W>(E, cand[q]) : (uint32_t)kAddsSlots;
    // W + kAddsSlots marks "waiting in the far pile"; not issued: 0 reads as "queued lower"
    oq[q] = atom_min_if(imp[q], &P.qb[ed[q].x], E.W + s[q], 0u);
  }
  uint32_t of[kU], kfar = 0xFFFFFFFFu;
#pragma unroll
  for (int q = 0; q < kU; ++q) {
    const bool far = imp[q] && s[q] == kAddsSlots && oq[q] > E.W + s[q];
    of[q] = atom_exch_if(far, &P.farflag[ed[q].x], 1u, 1u);
    // every improvement past the window bounds the next epoch's base, also
    // one whose vertex already waits in the far pile with an older key
    if (imp[q] && s[q] == kAddsSlots) kfar = min(kfar, cand[q]);
  }
  kfar = __reduce_min_sync(kFull, kfar);
  if (lane_id() == 0 && kfar != 0xFFFFFFFFu) atomicMin(&P.ctl->far_min_key, kfar);
#pragma unroll
  for (int q = 0; q < kU; ++q) {
    const bool lowered = imp[q] && oq[q] > E.W + s[q];
    const bool to_slot = lowered && s[q] < kAddsSlots;
    const bool to_far = lowered && s[q] == kAddsSlots && of[q] == 0u;
    push_slots(P, to_slot, s[q], ed[q].x);
    push_far(P, E, to_far, ed[q].x, cand[q]);
    t.pushes += (to_slot || to_far) ? 1 : 0;
  }
}

// Publish `nch` hub chunks of vertex hv taken from slot s (warp-collective):
// the bucket's `extra` grows before any chunk becomes visible.  Ring position
// p lives at p % hub_cap; its writer waits (bounded) until the chunk of the
// previous lap there has been taken, then stores the entry and, last, the tag.
__device__ __forceinline__ void publish_hub(const AParams& P, uint32_t hv, uint32_t nch, uint32_t s) {
  unsigned long long hb = 0;
  if (lane_id() == 0) {
    atomicAdd(&P.ctl->slot[s].extra, nch);
    __threadfence();
    hb = atomicAdd(&P.ctl->hub_reserved, (unsigned long long)nch);
  }
  hb = shfl64(hb, 0);
  for (uint32_t j = lane_id(); j < nch; j += 32) {
    ulonglong2* e = P.hub + (size_t)((hb + j) % P.hub_cap);
    if (ld_vol64(&e->x) != kEmpty64) {
      const uint64_t t0 = globaltimer_ns();
      bool gave_up = false;
      while (ld_vol64(&e->x) != kEmpty64) {
        __nanosleep(64);
        if (ld_vol(&P.ctl->error)) { gave_up = true; break; }
        if (globaltimer_ns() - t0 > P.budget_ns) {
          set_err(P, kErrTimeout, 44);
          gave_up = true;
          break;
        }
      }
      if (gave_up) continue;
    }
    *(volatile unsigned long long*)&e->y = ((unsigned long long)((j << 5) | s) << 32) | hv;
    st_release_u64(&e->x, hb + j);
  }
}

// Expand up to 32 taken vertices, one per lane (`take` lanes hold one).
template <class W, bool PRED>
__device__ void expand(const AParams& P, const View& E, uint32_t v, bool take, uint32_t s, ATally& t) {
  using L = Label<PRED>;
  const uint32_t lane = lane_id();
  uint32_t du = kInfKey;
  uint64_t lo = 0, hi = 0;
  if (take) {
    lo = __ldg(P.rowptr + v);   // row bounds go out with the label load
    hi = __ldg(P.rowptr + v + 1);
    __threadfence();   // the qb reset is visible before the label is read
    du = L::key(ld_keep((const typename L::T*)P.dist + v, t.keep));
    // a label that has dropped into a lower bucket since this entry was
    // queued is expanded from there (it was queued there, or was expanded
    // there already with this label)
    if (du != kInfKey && slot_of<W>(E, du) < s) du = kInfKey;
  }
  uint32_t deg = (du != kInfKey) ? (uint32_t)min(hi - lo, (uint64_t)0xFFFFFFFFull) : 0u;
  uint32_t hubs = __ballot_sync(kFull, deg >= P.hub_degree);
  while (hubs) {
    const uint32_t hl = __ffs(hubs) - 1;
    hubs &= hubs - 1;
    const uint32_t hv = __shfl_sync(kFull, v, hl);
    const uint32_t nch = (__shfl_sync(kFull, deg, hl) + kChunkEdges - 1) / kChunkEdges;
    publish_hub(P, hv, nch, s);
    if (lane == hl) deg = 0;
  }
  const uint32_t nz = __ballot_sync(kFull, deg > 0);
  const uint32_t k = __popc(nz);
  if (k == 0) return;
  const bool has = lane < k;
  const uint32_t sl = nth_set_bit(nz, has ? lane : 0u);
  const uint32_t cv = __shfl_sync(kFull, v, sl);
  const uint32_t cdu = __shfl_sync(kFull, du, sl);
  const uint32_t sdeg = __shfl_sync(kFull, deg, sl);
  const uint32_t cdeg = has ? sdeg : 0u;
  const unsigned long long clo = shfl64(lo, sl);
  const uint32_t incl = warp_incl_scan(cdeg);
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  const uint32_t excl = incl - cdeg;
  const unsigned long long ebase = clo - excl;   // edge index of slot p owned here = ebase + p
  uint32_t started = 0;
  for (uint32_t eb = 0; eb < total; eb += 32 * kU) {
    bool act[kU];
    uint32_t src[kU], dsrc[kU];
    uint2 ed[kU];
#pragma unroll
    for (int q = 0; q < kU; ++q) {
      const uint32_t w0 = eb + 32 * q;
      const uint32_t bit = (has && excl >= w0 && excl < w0 + 32) ? (1u << (excl - w0)) : 0u;
      const uint32_t starts = __reduce_or_sync(kFull, bit);
      uint32_t own = started + __popc(starts & lanemask_le()) - 1;
      started += __popc(starts);
      own = min(own, 31u);
      const uint32_t p = w0 + lane;
      act[q] = p < total;
      src[q] = __shfl_sync(kFull, cv, own);
      dsrc[q] = __shfl_sync(kFull, cdu, own);
      const unsigned long long e = shfl64(ebase, own) + p;
      ed[q] = act[q] ? __ldcs(&P.edges[e]) : make_uint2(0, 0);
    }
    relax_route<W, PRED>(P, E, act, src, dsrc, ed, t);
  }
}

// Finish `units` units of slot s: this warp's pushes are visible first.
__device__ __forceinline__ void finish_units(const AParams& P, uint32_t s, uint32_t units) {
  __threadfence();
  __syncwarp();
  if (lane_id() == 0) atomicAdd(&P.ctl->slot[s].done, units);
}

// Take k claimed entries [c, c + k) of slot s and expand them.
template <class W, bool PRED>
__device__ void take_entries(const AParams& P, const View& E, uint32_t s, uint32_t c, uint32_t k, ATally& t) {
  const uint32_t gb = E.W + s;
  for (uint32_t j0 = 0; j0 < k; j0 += 32) {
    const bool present = j0 + lane_id() < k;
    uint32_t v = 0;
    bool take = false;
    if (present) {
      const uint32_t pos = c + j0 + lane_id();
      unsigned long long* wp = slot_queue(P, s) + (pos % P.cap);
      v = wait_word(P, wp, pos);
      if (v != kEmpty) {
        __stcg(wp, kEmpty64);
        // expand unless v waits in a lower bucket (it is expanded there with
        // its newer label); a duplicate taken after its twin expands again
        const uint32_t old = atomicCAS(&P.qb[v], gb, kNotQueued);
        take = old == gb || old > gb;
      }
    }
    expand<W, PRED>(P, E, v, take, s, t);
  }
  t.entries += k;
  finish_units(P, s, k);
}

// One claimed hub chunk: lane 0 has claimed ring position `pos`.
template <class W, bool PRED>
__device__ void take_chunk(const AParams& P, const View& E, unsigned long long pos, ATally& t) {
  using L = Label<PRED>;
  unsigned long long ent = 0;
  if (lane_id() == 0) {
    ulonglong2* e = P.hub + (size_t)(pos % P.hub_cap);
    ent = wait_hub(P, e, pos);
    if (ent != kEmpty64) st_release_u64(&e->x, kEmpty64);   // after the entry was read
  }
  ent = shfl64(ent, 0);
  if (ent == kEmpty64) return;   // the wait gave up (error recorded)
  const uint32_t v = (uint32_t)ent;
  const uint32_t chunk = (uint32_t)(ent >> 37);
  const uint32_t s = (uint32_t)(ent >> 32) & 31u;
  uint32_t du = L::key(ld_keep((const typename L::T*)P.dist + v, t.keep));
  // a label that has dropped into a lower bucket since the chunk was published
  // is expanded from there, all its chunks included; relaxing from it here
  // could push into a bucket below s that is already complete
  if (du != kInfKey && slot_of<W>(E, du) < s) du = kInfKey;
  const uint64_t rb = __ldg(P.rowptr + v), re = __ldg(P.rowptr + v + 1);
  const uint64_t e0 = rb + (uint64_t)chunk * kChunkEdges;
  const uint64_t e1 = min(re, e0 + kChunkEdges);
  for (uint64_t eb = e0; eb < e1; eb += 32 * kU) {
    bool act[kU];
    uint32_t src[kU], dsrc[kU];
    uint2 ed[kU];
#pragma unroll
    for (int q = 0; q < kU; ++q) {
      const uint64_t e = eb + 32 * q + lane_id();
      act[q] = e < e1 && du != kInfKey;
      src[q] = v;
      dsrc[q] = du;
      ed[q] = act[q] ? __ldcs(&P.edges[e]) : make_uint2(0, 0);
    }
    relax_route<W, PRED>(P, E, act, src, dsrc, ed, t);
  }
  t.chunks += 1;
  finish_units(P, s, 1);
}

__device__ __forceinline__ unsigned long long head_word(uint32_t epoch, uint32_t pos) {
  return ((unsigned long long)epoch << 32) | pos;
}
// ---- per-block work pools --------------------------------------------------
// Claims from the shared queues go through one warp per block: it claims up
// to kBlockClaimMax entries of a bucket (or kHubClaim hub chunks) with one
// compare-and-swap and publishes the range in shared memory, where the
// block's warps take kGrab entries (or one chunk) at a time with a
// shared-memory compare-and-swap on the range's ticket, (generation << 32) |
// next.  The range of a generation sits in the descriptor of its parity,
// tagged with the generation.
struct PoolDesc {
  unsigned long long base;   // first claimed position (entries: slot position; hubs: ring position)
  uint32_t count;
  uint32_t slot;             // entries: bucket slot
  uint32_t gen;
  uint32_t pad;
};
struct BlockPool {
  unsigned long long ticket;   // entries
  unsigned long long hticket;  // hub chunks
  PoolDesc ent[2];
  PoolDesc hub[2];
  uint32_t lock;
  uint32_t pos;                // head position the refilling warp saw last
  View view;                   // the epoch of the ranges published here (set before the first one)
};

__device__ __forceinline__ void publish_range(unsigned long long* ticket, PoolDesc* d, unsigned long long base,
                                              uint32_t count, uint32_t slot) {
  const uint32_t g = (uint32_t)(*(volatile unsigned long long*)ticket >> 32) + 1;
  PoolDesc& x = d[g & 1];
  x.base = base;
  x.count = count;
  x.slot = slot;
  *(volatile uint32_t*)&x.gen = g;
  __threadfence_block();
  atomicExch(ticket, (unsigned long long)g << 32);
}

// Lane 0: take up to `want` items of the block's current range.  Returns the
// count (0: the range is used up) with the first item's position and the slot.
// The descriptor is read between a ticket read and the compare-and-swap that
// advances the ticket; tickets only grow, so a successful swap proves no new
// range was published in between and the descriptor read was the ticket's.
__device__ __forceinline__ uint32_t grab(unsigned long long* ticket, const PoolDesc* d, uint32_t want,
                                         unsigned long long* first, uint32_t* slot) {
  for (int tries = 0; tries < 64; ++tries) {
    const unsigned long long t = *(volatile unsigned long long*)ticket;
    const uint32_t g = (uint32_t)(t >> 32), i = (uint32_t)t;
    const PoolDesc& x = d[g & 1];
    if (*(const volatile uint32_t*)&x.gen != g) return 0;   // being published (by this block's lock holder)
    const uint32_t cnt = *(const volatile uint32_t*)&x.count;
    if (i >= cnt) return 0;
    const unsigned long long base = *(const volatile unsigned long long*)&x.base;
    const uint32_t sl = *(const volatile uint32_t*)&x.slot;
    const uint32_t k = min(want, cnt - i);
    if (atomicCAS(ticket, t, t + k) == t) {
      *first = base + i;
      *slot = sl;
      return k;
    }
  }
  return 0;
}

// Items left in the block's current range (read by the lock holder, the only
// warp that publishes ranges).
__device__ __forceinline__ uint32_t pool_left(const unsigned long long* ticket, const PoolDesc* d) {
  const unsigned long long t = *(const volatile unsigned long long*)ticket;
  const uint32_t g = (uint32_t)(t >> 32), i = (uint32_t)t;
  const PoolDesc& x = d[g & 1];
  if (*(const volatile uint32_t*)&x.gen != g) return 0;
  const uint32_t cnt = *(const volatile uint32_t*)&x.count;
  return i < cnt ? cnt - i : 0u;
}

__device__ __forceinline__ bool slot_complete(const AddsControl* c, uint32_t s);
__device__ void idle_step(const AParams& P);

// Lane 0 of the warp holding the block's lock: claim hub chunks, else
// entries of the active buckets (lowest first), else do the idle step.
// Returns true when a range was published.
__device__ bool refill(const AParams& P, BlockPool& sp) {
  AddsControl* c = P.ctl;
  const unsigned long long hw = ld_acquire_u64(&c->head);
  const uint32_t pos = (uint32_t)hw;
  *(volatile uint32_t*)&sp.pos = pos;
  if (pos > (uint32_t)kAddsSlots) return false;   // a split or the end
  // a range is replaced only once it is used up, so no claimed item is dropped
  if (pool_left(&sp.hticket, sp.hub) || pool_left(&sp.ticket, sp.ent)) return true;
  // the block's copy of the epoch view: a claimed unit pins its epoch, so the
  // view stays right while any warp of the block holds one
  const uint32_t ep = (uint32_t)(hw >> 32);
  if (*(volatile uint32_t*)&sp.view.epoch != ep) {
    const View E = read_view(c);
    if (E.epoch != ep) return false;   // the head moved on meanwhile
    volatile uint32_t* dv = (volatile uint32_t*)&sp.view;
    const uint32_t* sv = (const uint32_t*)&E;
    for (int i = 0; i < (int)(sizeof(View) / 4); ++i) dv[i] = sv[i];
    __threadfence_block();
  }
  // hub chunks
  for (int tries = 0; tries < 4; ++tries) {
    const unsigned long long cl = ld_vol64(&c->hub_claim);
    const unsigned long long R = ld_vol64(&c->hub_reserved);
    if (cl >= R) break;
    const unsigned long long k = min((unsigned long long)kHubClaim, R - cl);
    if (atomicCAS(&c->hub_claim, cl, cl + k) == cl) {
      publish_range(&sp.hticket, sp.hub, cl, (uint32_t)k, 0);
      return true;
    }
  }
  // entries
  const uint32_t epoch = ld_vol(&c->epoch);
  if ((uint32_t)(hw >> 32) == epoch && pos < (uint32_t)kAddsSlots) {
    const uint32_t a = ld_vol(&c->active);
    for (uint32_t j = 0; j < a && pos + j < (uint32_t)kAddsSlots; ++j) {
      const uint32_t ss = pos + j;
      for (int tries = 0; tries < 4; ++tries) {
        const unsigned long long w = ld_vol64(&c->slot[ss].claim);
        if ((uint32_t)(w >> 32) != epoch) return false;
        const uint32_t got = (uint32_t)w;
        const uint32_t R = ld_vol(&c->slot[ss].reserved);
        if (got == R || (int32_t)(R - got) < 0) break;
        const uint32_t avail = R - got;
        const uint32_t share = avail / max(1u, gridDim.x);
        const uint32_t k = min(avail, max(kBlockClaimMin, min(share, kBlockClaimMax)));
        if (atomicCAS(&c->slot[ss].claim, w, w + k) == w) {
          publish_range(&sp.ticket, sp.ent, got, k, ss);
          return true;
        }
      }
    }
  }
  idle_step(P);
  return false;
}

__device__ __forceinline__ bool slot_complete(const AddsControl* c, uint32_t s) {
  const uint32_t d = ld_acquire_u32(&c->slot[s].done);
  const uint32_t r = ld_vol(&c->slot[s].reserved);
  const uint32_t x = ld_vol(&c->slot[s].extra);
  return d == r + x;
}

__device__ __forceinline__ bool claimable(const AddsControl* c, uint32_t s, uint32_t epoch) {
  const unsigned long long w = ld_vol64(&c->slot[s].claim);
  return (uint32_t)(w >> 32) == epoch && (uint32_t)w < ld_vol(&c->slot[s].reserved);
}


// Lane 0 of the warp that moved the head from (epoch, kAddsSlots) to
// (epoch, kAddsPrep): the next epoch, prepared while every warp waits; the
// head then reads (epoch + 1, kAddsSplit) until the far pile is routed.
__device__ void prepare_split(const AParams& P) {
  AddsControl* c = P.ctl;
  __threadfence();
  const uint32_t sel = ld_vol(&c->far_sel);
  const uint32_t fc = min(ld_vol(&c->far_count[sel]), P.cap);
  const uint32_t kmin = ld_vol(&c->far_min_key);
  const uint32_t epoch = ld_vol(&c->epoch);
  uint32_t dq = ld_vol(&c->dq), dinv = ld_vol(&c->dinv);
  if (P.adapt) {
    // ADDS feedback: widen buckets when this epoch's buckets left the grid
    // under-used, narrow them when they overflowed it
    const uint32_t nb = ld_vol(&c->epoch_buckets);
    const double avg = nb ? (double)ld_vol64(&c->epoch_entries) / (double)nb : 0.0;
    double f = 1.0;
    if (avg < 0.35 * (double)P.adapt_cap) f = 1.5;
    else if (avg > 0.85 * (double)P.adapt_cap) f = 0.75;
    if (f != 1.0) {
      c->delta_updates = ld_vol(&c->delta_updates) + 1;
      if (P.is_float) {
        const float wnew = fmaxf(1.0e-6f, (float)((1.0 / (double)__uint_as_float(dinv)) * f));
        dinv = __float_as_uint(1.0f / wnew);
      } else {
        dq = (uint32_t)fmin(4294967295.0, fmax(1.0, floor((double)dq * f + 0.5)));
      }
    }
  }
  for (int s = 0; s < kAddsSlots; ++s) {
    c->slot[s].reserved = 0;
    c->slot[s].extra = 0;
    c->slot[s].done = 0;
    c->slot[s].claim = (unsigned long long)(epoch + 1) << 32;
  }
  c->far_count[sel ^ 1u] = 0;
  c->split_cursor = 0;
  c->split_done = 0;
  c->split_total = fc;
  c->W = ld_vol(&c->W) + kAddsSlots + 1;   // the old far mark W + kAddsSlots is no bucket of the new epoch
  c->kbase = kmin;
  c->dq = dq;
  c->dinv = dinv;
  c->active = P.active0;
  c->far_sel = sel ^ 1u;
  c->far_min_key = 0xFFFFFFFFu;
  c->epoch_entries = 0;
  c->epoch_buckets = 0;
  c->epochs = ld_vol(&c->epochs) + 1;
  __threadfence();
  st_release_u32(&c->epoch, epoch + 1);
  __threadfence();
  st_release_u64(&c->head, head_word(epoch + 1, kAddsSplit));
}

// Every warp: move far-pile entries into the new epoch, 32 at a time.
// Returns false when no chunk was left to take.
template <class W, bool PRED>
__device__ bool split_work(const AParams& P) {
  using L = Label<PRED>;
  AddsControl* c = P.ctl;
  uint32_t i = 0, total = 0;
  View E;
  if (lane_id() == 0) {
    E = read_view(c);
    total = ld_vol(&c->split_total);
    i = atomicAdd(&c->split_cursor, 32u);
  }
  E = bcast(E);
  i = __shfl_sync(kFull, i, 0);
  total = __shfl_sync(kFull, total, 0);
  if (i >= total) return false;
  const uint32_t src = E.far_sel ^ 1u;
  const uint32_t pos = i + lane_id();
  const bool present = pos < total;
  uint32_t v = 0, key = kInfKey, s = kAddsSlots;
  bool to_slot = false, to_far = false;
  if (present) {
    v = __ldcg(far_queue(P, src) + pos);
    if (__ldcg(P.qb + v) == E.W - 1u) {   // waiting in the far pile: route by its label now
      key = L::key(__ldcg((const typename L::T*)P.dist + v));
      s = slot_of<W>(E, key);
      if (s < kAddsSlots) {
        P.qb[v] = E.W + s;
        P.farflag[v] = 0u;
        to_slot = true;
      } else {
        P.qb[v] = E.W + kAddsSlots;
        to_far = true;   // stays in the far pile (its flag stays set)
      }
    } else {
      P.farflag[v] = 0u;   // a newer entry of v lives in a window bucket, or v was expanded
    }
  }
  push_slots(P, to_slot, s, v);
  push_far(P, E, to_far, v, key);
  __threadfence();
  __syncwarp();
  if (lane_id() == 0) {
    const uint32_t cnt = min(32u, total - i);
    const uint32_t prev = atomicAdd(&c->split_done, cnt);
    if (prev + cnt == total) {   // the new window is filled: its buckets open
      c->far_count[src] = 0;
      __threadfence();
      st_release_u64(&c->head, head_word(E.epoch, 0));
    }
  }
  return true;
}

__device__ __forceinline__ void trace_bucket(const AParams& P, uint32_t s, uint32_t gb) {
  if (!P.trace) return;
  AddsControl* c = P.ctl;
  const uint32_t i = atomicAdd(&c->trace_n, 1u);
  if (i >= kTraceCap) return;
  TraceEntry e;
  e.kind = kPhaseProcess;
  e.fcount = ld_vol(&c->slot[s].reserved);
  e.hub_chunks = ld_vol(&c->slot[s].extra);
  e.cur = gb;
  e.t_ns = globaltimer_ns() - c->t_start;
  P.trace[i] = e;
}

// Lane 0 of a warp that found nothing to take: retire complete head buckets,
// widen the active range, or end the epoch.  Every step is a compare-and-swap
// of the (epoch, position) head word, so a warp working from an epoch that
// has ended changes nothing.
__device__ void idle_step(const AParams& P) {
  AddsControl* c = P.ctl;
  unsigned long long hw = ld_acquire_u64(&c->head);
  uint32_t h = (uint32_t)hw;
  while (h < (uint32_t)kAddsSlots && slot_complete(c, h)) {
    if (atomicCAS(&c->head, hw, hw + 1) == hw) {
      const uint32_t r = ld_vol(&c->slot[h].reserved);
      if (r) {
        const uint32_t nb = atomicAdd(&c->buckets, 1u) + 1;
        // buckets before this one had a successor; the last is reported at the end
        if (nb > 1) publish_progress(P.board, nb - 1, 1u, globaltimer_ns() - ld_vol64(&c->t_start));
        atomicAdd(&c->epoch_buckets, 1u);
        atomicAdd(&c->epoch_entries, (unsigned long long)r);
        trace_bucket(P, h, ld_vol(&c->W) + h);
      }
    }
    hw = ld_acquire_u64(&c->head);
    h = (uint32_t)hw;
  }
  if (h == (uint32_t)kAddsSlots) {
    // the window has retired: nothing is in flight, so the far pile is final
    __threadfence();
    const uint32_t sel = ld_vol(&c->far_sel);
    const uint32_t epoch = (uint32_t)(hw >> 32);
    if (ld_vol(&c->far_count[sel]) == 0) {
      if (atomicCAS(&c->head, hw, head_word(epoch, kAddsDone)) == hw) c->converged = 1;
    } else if (atomicCAS(&c->head, hw, head_word(epoch, kAddsPrep)) == hw) {
      prepare_split(P);
    }
    return;
  }
  if (h > (uint32_t)kAddsSlots) return;   // a split or the end
  // later buckets hold work while the active ones have none to give: widen
  const uint32_t a = ld_vol(&c->active);
  const uint32_t epoch = (uint32_t)(hw >> 32);
  for (uint32_t j = a; j < a + 2 && j < P.active_max && h + j < (uint32_t)kAddsSlots; ++j) {
    if (claimable(c, h + j, epoch)) {
      atomicMax(&c->active, j + 1);
      atomicMax(&c->max_active, j + 1);
      break;
    }
  }
}

template <class W, bool PRED>
__device__ void worker(const AParams& P, BlockPool& sp, ATally& t) {
  AddsControl* c = P.ctl;
  uint32_t idle = 0, iter = 0;
  const unsigned long long t_start = ld_vol64(&c->t_start);
  for (;;) {
    uint32_t pos = 0, err = 0;
    if (lane_id() == 0) {
      pos = *(volatile uint32_t*)&sp.pos;
      // the error flag and the budget every 8th pass (every wait checks them too)
      if ((++iter & 7u) == 0u || idle) {
        err = ld_vol(&c->error);
        if (!err && globaltimer_ns() - t_start > P.budget_ns) {
          set_err(P, kErrTimeout, 45);
          err = 1;
        }
      }
    }
    pos = __shfl_sync(kFull, pos, 0);
    err = __shfl_sync(kFull, err, 0);
    if (err || pos == kAddsDone) return;
    if (pos == kAddsSplit) {
      // every warp helps route the far pile; the block's pools are empty
      if (!split_work<W, PRED>(P)) {
        if (lane_id() == 0 && atomicCAS(&sp.lock, 0u, 1u) == 0u) {
          *(volatile uint32_t*)&sp.pos = (uint32_t)ld_acquire_u64(&c->head);
          atomicExch(&sp.lock, 0u);
        }
        __syncwarp();
        __nanosleep(128);
      }
      continue;
    }
    // a hub chunk, else kGrab entries, from the block's pools
    unsigned long long first = 0;
    uint32_t slot = 0, k = 0, kind = 0;
    if (lane_id() == 0) {
      k = grab(&sp.hticket, sp.hub, 1, &first, &slot);
      if (k) kind = 1;
      else if ((k = grab(&sp.ticket, sp.ent, kGrab, &first, &slot)) != 0) kind = 2;
    }
    kind = __shfl_sync(kFull, kind, 0);
    if (kind) {
      first = shfl64(first, 0);
      k = __shfl_sync(kFull, k, 0);
      slot = __shfl_sync(kFull, slot, 0);
      // a claimed unit pins its epoch (its bucket cannot complete), so the
      // block's view, set before the range was published, is its epoch's
      View E;
      {
        const volatile uint32_t* sv = (const volatile uint32_t*)&sp.view;
        uint32_t* dv = (uint32_t*)&E;
        for (int i = 0; i < (int)(sizeof(View) / 4); ++i) dv[i] = sv[i];
      }
      if (kind == 1) take_chunk<W, PRED>(P, E, first, t);
      else take_entries<W, PRED>(P, E, slot, (uint32_t)first, k, t);
      idle = 0;
      continue;
    }
    // both pools are empty: one warp of the block refills them
    uint32_t got = 0;
    if (lane_id() == 0 && atomicCAS(&sp.lock, 0u, 1u) == 0u) {
      got = refill(P, sp) ? 1u : 0u;
      atomicExch(&sp.lock, 0u);
    }
    got = __shfl_sync(kFull, got, 0);
    if (got) { idle = 0; continue; }
    ++idle;
    __nanosleep(idle < 4 ? 64u : (idle < 32 ? 256u : 1024u));
  }
}

template <bool PRED>
__device__ void init_start(const AParams& P) {
  using L = Label<PRED>;
  AddsControl* c = P.ctl;
  const uint32_t zk = P.is_float ? f32_to_key(0.0f) : 0u;
  ((typename L::T*)P.dist)[P.source] = L::make(zk, 0u);
  P.qb[P.source] = 0u;
  slot_queue(P, 0)[0] = ring_word(0u, P.source);
  for (int s = 0; s < kAddsSlots; ++s) {
    c->slot[s].claim = 1ull << 32;
    c->slot[s].reserved = 0;
    c->slot[s].extra = 0;
    c->slot[s].done = 0;
  }
  c->slot[0].reserved = 1;
  c->W = 0;
  c->kbase = zk;
  c->dq = P.width_u;
  c->dinv = __float_as_uint(P.inv_width);
  c->active = P.active0;
  c->max_active = P.active0;
  c->far_sel = 0;
  c->far_count[0] = 0;
  c->far_count[1] = 0;
  c->far_min_key = 0xFFFFFFFFu;
  c->hub_claim = 0;
  c->hub_reserved = 0;
  c->epochs = 1;
  c->t_start = globaltimer_ns();
  __threadfence();
  c->epoch = 1;
  c->head = head_word(1, 0);
}

template <class W, bool PRED>
__global__ void __launch_bounds__(kAThreads, 2) k_adds(AParams P) {
  using L = Label<PRED>;
  AddsControl* c = P.ctl;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  typename L::T* lab = (typename L::T*)P.dist;
  for (size_t v = tid; v < P.n; v += stride) {
    if (!P.warm) {
      lab[v] = L::kInf;
    } else {
      // the caller's distances (input ids) are the starting upper bounds
      const size_t iv = P.perm ? (size_t)__ldg(P.perm + v) : v;
      uint32_t k;
      if (W::kFloat) {
        const float f = ((const float*)P.warm_in)[iv];
        k = (f == f && f != __int_as_float(0x7f800000)) ? f32_to_key(f) : kInfKey;
      } else {
        k = ((const uint32_t*)P.warm_in)[iv];
      }
      if (PRED || !P.dist_is_out || W::kFloat) lab[v] = L::make(k, kNoPred);
    }
    P.qb[v] = kNotQueued;
    P.farflag[v] = 0u;
  }
  ATally t;
  t.keep = l2_keep_policy();
  __shared__ BlockPool sp;
  if (threadIdx.x == 0) {
    memset(&sp, 0, sizeof(sp));   // empty pools (generation 0, no items), position 0
  }
  const bool ok = grid_barrier((GridBarrier*)c, gridDim.x, P.budget_ns, [&] { init_start<PRED>(P); });
  if (ok) worker<W, PRED>(P, sp, t);
  // tallies (one atomic per warp)
  unsigned long long e = t.edges, im = t.impr, pu = t.pushes, en = t.entries, ch = t.chunks;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(kFull, e, o);
    im += __shfl_down_sync(kFull, im, o);
    pu += __shfl_down_sync(kFull, pu, o);
  }
  if (lane_id() == 0) {
    if (e) atomicAdd(&c->edges, e);
    if (im) atomicAdd(&c->improvements, im);
    if (pu) atomicAdd(&c->pushes, pu);
    if (en) atomicAdd(&c->entries, en);
    if (ch) atomicAdd(&c->hub_chunks, ch);
  }
  // outputs: once the head says DONE every label is final
  if ((uint32_t)ld_acquire_u64(&c->head) != kAddsDone || ld_vol(&c->error)) return;
  for (size_t o = tid; o < P.n; o += stride) {
    const size_t v = P.inv ? (size_t)__ldg(P.inv + o) : o;   // internal id of output slot o
    const typename L::T wv = __ldcg(lab + v);
    const uint32_t k = L::key(wv);
    if (W::kFloat) {
      ((float*)P.out_dist)[o] = (k == kInfKey) ? __uint_as_float(0x7f800000u) : key_to_f32(k);
    } else if (!P.dist_is_out) {
      ((uint32_t*)P.out_dist)[o] = k;
    }
    if (PRED && P.out_pred) {
      int32_t pr = -1;
      const uint32_t pv = (uint32_t)(wv & 0xFFFFFFFFull);
      if (k != kInfKey && v != P.source && pv != kNoPred) pr = (int32_t)(P.perm ? __ldg(P.perm + pv) : pv);
      P.out_pred[o] = pr;
    }
  }
}

constexpr int kMaxDevices = 64;
template <class W, bool PRED>
int adds_grid() {
  static std::mutex mu;
  static int cached[kMaxDevices] = {};
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
  std::lock_guard<std::mutex> lock(mu);
  if (cached[dev]) return cached[dev];
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_adds<W, PRED>, kAThreads, 0);
  if (per < 1) per = 1;
  cached[dev] = per * sms;
  return cached[dev];
}

template <class W, bool PRED>
cudaError_t launch_adds(const AParams& P, int grid, cudaStream_t st) {
  AParams copy = P;
  void* args[] = {&copy};
  return cudaLaunchCooperativeKernel((void*)k_adds<W, PRED>, dim3(grid), dim3(kAThreads), args, 0, st);
}

b2_status ensure_adds(b2_graph g, uint32_t cap_opt, cudaStream_t st) {
  Workspace& w = g->ws;
  const size_t n = (size_t)g->n;
  // a bucket ring holds the entries of its waiting vertices (at most n) plus
  // the claims in flight (block pools and warps: under 2^19 on a full grid);
  // small graphs get 2^18 words so a busy bucket seldom laps its ring
  const size_t full = std::max<size_t>(n + std::min<size_t>(n, (size_t)1 << 19), (size_t)1 << 18) + 1024;
  const size_t cap = (cap_opt > 0 && cap_opt < full) ? cap_opt : full;
  if (w.adds_q && w.adds_cap == cap) return B2_SUCCESS;
  free_adds_workspace(w);
  cudaError_t e = cudaMalloc((void**)&w.adds_q, (size_t)kAddsSlots * cap * 8 + (size_t)2 * cap * 4 + 16);
  // chunks waiting at once: at most two expansions' worth of every hub row
  w.adds_hub_cap = std::min<size_t>(4 * ((size_t)g->m / kChunkEdges + 1) + 65536, 0x7FFFFFFFull);
  if (e == cudaSuccess) e = cudaMalloc((void**)&w.adds_hub, w.adds_hub_cap * sizeof(ulonglong2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&w.adds_qb, std::max<size_t>(n * 4, 16));
  if (e == cudaSuccess) e = cudaMalloc((void**)&w.adds_ctl, sizeof(AddsControl));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&w.adds_h_ctl, sizeof(AddsControl));
  if (e != cudaSuccess) {
    free_adds_workspace(w);
    return from_cuda(e);
  }
  w.adds_cap = cap;
  w.adds_dirty = true;
  (void)st;
  return B2_SUCCESS;
}

}  // namespace

void free_adds_workspace(Workspace& w) {
  if (w.adds_q) cudaFree(w.adds_q);
  if (w.adds_hub) cudaFree(w.adds_hub);
  if (w.adds_qb) cudaFree(w.adds_qb);
  if (w.adds_ctl) cudaFree(w.adds_ctl);
  if (w.adds_h_ctl) cudaFreeHost(w.adds_h_ctl);
  w.adds_q = nullptr;
  w.adds_hub = nullptr;
  w.adds_qb = nullptr;
  w.adds_ctl = nullptr;
  w.adds_h_ctl = nullptr;
  w.adds_cap = 0;
  w.adds_hub_cap = 0;
  w.adds_dirty = true;
}

b2_status run_adds(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred, const b2_sssp_opts* o_in,
                   cudaStream_t st, b2_stats* stats) {
  if (!g || !d_dist) return B2_INVALID_ARGUMENT;
  if ((int64_t)source >= g->n) return B2_INVALID_ARGUMENT;
  b2_sssp_opts o;
  if (o_in) o = *o_in; else b2_sssp_opts_default(&o);
  if (g->has_negative) return B2_INVALID_WEIGHT;
  const bool isf = g->weight_type == B2_W_F32;
  const bool pred = d_pred != nullptr;
  const bool warm = o.keep_distances != 0;
  uint32_t policy_used = 0;
  double delta = o.delta;
  if (o.policy == 1) {
    double mult = 1.0;
    uint32_t fuse = 0;
    float pull = 8.0f;
    const b2_status ps = policy_decide(g, &mult, &fuse, &pull);   // ADDS takes the width only
    if (ps == B2_SUCCESS) {
      double nf = 1.0;
      b2_delta_heuristic(g, o.delta_scale > 0 ? o.delta_scale : 16.0, &nf);
      delta = nf * mult;
      policy_used = 1;
    } else if (ps != B2_NOT_SUPPORTED) {
      return ps;
    }
  }
  if (!(delta > 0.0)) b2_delta_heuristic(g, o.delta_scale > 0 ? o.delta_scale : 16.0, &delta);
  std::lock_guard<std::mutex> lock(g->mu);
  b2_status s = ensure_workspace(g, pred);
  if (s != B2_SUCCESS) return s;
  s = ensure_adds(g, o.worklist_capacity, st);
  if (s != B2_SUCCESS) return s;
  Workspace& w = g->ws;

  AParams P;
  memset(&P, 0, sizeof(P));
  P.n = (uint32_t)g->n;
  P.source = internal_id(g, source);
  P.rowptr = g->rowptr;
  P.edges = g->edges;
  P.qb = w.adds_qb;
  P.farflag = w.farflag;
  P.q = (unsigned long long*)w.adds_q;
  P.far = (uint32_t*)((char*)w.adds_q + (size_t)kAddsSlots * w.adds_cap * 8);
  P.cap = (uint32_t)w.adds_cap;
  P.hub = (ulonglong2*)w.adds_hub;
  P.hub_cap = (uint32_t)w.adds_hub_cap;
  P.ctl = w.adds_ctl;
  P.trace = o.trace ? w.trace : nullptr;
  P.is_float = isf ? 1u : 0u;
  P.hub_degree = std::max<uint32_t>(64u, o.hub_degree ? o.hub_degree : 512u);
  P.active0 = o.active_buckets > 0 ? std::min<uint32_t>(o.active_buckets, kAddsSlots) : 2u;
  P.active_max = o.max_active_buckets > 0 ? std::min<uint32_t>(o.max_active_buckets, kAddsSlots) : (uint32_t)kAddsSlots;
  P.active_max = std::max(P.active_max, P.active0);
  P.adapt = o.adds_fixed_delta ? 0u : 1u;
  P.budget_ns = (unsigned long long)(std::max(0.001, o.timeout_ms > 0 ? o.timeout_ms : 20000.0) * 1.0e6);
  P.out_dist = d_dist;
  P.out_pred = d_pred;
  P.perm = g->perm;
  P.inv = g->perm ? g->inv : nullptr;
  P.warm = warm ? 1u : 0u;
  P.warm_in = d_dist;
  if (pred || g->perm) {
    P.dist = w.dist_a;
    P.dist_is_out = 0;
  } else {
    P.dist = d_dist;   // keys are built in the caller's buffer, converted in place
    P.dist_is_out = 1;
  }
  if (isf) {
    const float df = (float)delta;
    if (!(df > 0.0f) || !std::isfinite(df)) return B2_INVALID_ARGUMENT;
    P.inv_width = 1.0f / df;
    P.width_u = 1u;
  } else {
    const double dd = std::max(1.0, std::floor(delta));
    P.width_u = (uint32_t)std::min(dd, 4294967295.0);
    P.inv_width = 0.0f;
    delta = (double)P.width_u;
  }
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int grid = 0;
  if (isf) grid = pred ? adds_grid<WF32, true>() : adds_grid<WF32, false>();
  else grid = pred ? adds_grid<WU32, true>() : adds_grid<WU32, false>();
  if (o.grid_blocks && (int)o.grid_blocks < grid) grid = (int)o.grid_blocks;
  if (grid <= 0) return B2_CUDA_ERROR;
  P.adapt_cap = (uint32_t)grid * (kAThreads / 32) * kGrab;   // one grab per warp fills the grid
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->delta_used = delta;
    stats->policy_used = policy_used;
  }
  if (w.adds_dirty) {
    B2_CUDA_TRY(cudaMemsetAsync(w.adds_q, 0xFF, (size_t)kAddsSlots * w.adds_cap * 8, st));
    B2_CUDA_TRY(cudaMemsetAsync(w.adds_hub, 0xFF, w.adds_hub_cap * sizeof(ulonglong2), st));
  }
  B2_CUDA_TRY(cudaMemsetAsync(w.adds_ctl, 0, sizeof(AddsControl), st));
  s = progress_begin(g, o, &P.board);
  if (s != B2_SUCCESS) return s;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  cudaError_t e;
  if (isf) e = pred ? launch_adds<WF32, true>(P, grid, st) : launch_adds<WF32, false>(P, grid, st);
  else e = pred ? launch_adds<WU32, true>(P, grid, st) : launch_adds<WU32, false>(P, grid, st);
  cudaEventRecord(e1, st);
  if (e != cudaSuccess) { cudaEventDestroy(e0); cudaEventDestroy(e1); return from_cuda(e); }
  uint32_t reported = 0;
  if (P.board) progress_poll(g, o, e1, -1, &reported);
  e = cudaMemcpyAsync(w.adds_h_ctl, w.adds_ctl, sizeof(AddsControl), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return from_cuda(e);
  const AddsControl& hc = *w.adds_h_ctl;
  if (P.board) progress_finish(g, o, -1, hc.buckets, hc.converged ? 0 : 1, &reported);
  w.adds_dirty = hc.error != kErrNone;
  w.trace_n = o.trace ? std::min<uint32_t>(hc.trace_n, kTraceCap) : 0;
  if (stats) {
    stats->iterations_used = (int32_t)hc.buckets;
    stats->converged = (int32_t)hc.converged;
    stats->phases = (int32_t)hc.epochs;
    stats->edges_scanned = hc.edges;
    stats->improvements = hc.improvements;
    stats->pushes = hc.pushes;
    stats->kernel_ms = ms;
    stats->device_error = hc.error;
    stats->device_error_site = hc.error_site;
    stats->grid_blocks = (uint32_t)grid;
    stats->delta_updates = hc.delta_updates;
    float inv;
    memcpy(&inv, &hc.dinv, 4);
    stats->delta_final = isf ? 1.0 / (double)inv : (double)hc.dq;
    stats->work_items = hc.entries + hc.hub_chunks;
    stats->active_buckets_max = hc.max_active;
  }
  switch (hc.error) {
    case kErrNone: break;
    case kErrTimeout: return B2_TIMEOUT;
    case kErrQueueOverflow: return B2_POOL_EXHAUSTED;
    default: return B2_DEVICE_ERROR;
  }
  if (stats && o.collect_reach) return collect_reach(g, (pred || g->perm) ? w.dist_a : d_dist, pred, isf, st, stats);
  return B2_SUCCESS;
}

}  // namespace b2
