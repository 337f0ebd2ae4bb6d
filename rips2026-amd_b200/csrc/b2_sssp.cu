// Persistent single-launch SSSP: frontier Bellman-Ford (Jacobi rounds) and
// delta-stepping with device-resident ring buckets.
//
// One cooperative launch runs the whole solve.  Phases are separated by a
// grid barrier whose last arriver runs a one-thread manager step (see
// b2_common.cuh): it reads the phase's counters, picks the next phase and
// resets consumed counters while every other block is parked.  There is no
// host round-trip per bucket or iteration, unlike the reference
// (delta_stepping_hip_CSR.cpp:701-780: several D2H syncs per bucket;
// bf_hip_CSR.cpp:58-95: one sync per iteration).
//
// Relaxation (per phase): warps take work items from a phase counter: first
// the 256-edge chunks of high-degree vertices found in the previous phase,
// then 32-vertex frontier chunks.  For a frontier chunk the warp drops the
// vertices with nothing to relax, scans the rest's edge counts and walks the
// concatenated edge ranges 128 slots per step (4 per lane), so lanes read
// consecutive (dst, w) pairs with evict-first loads (the edge stream must not
// push the label array out of L2).  The owner of an edge slot comes from one
// warp-OR of "range starts here" bits per 32-slot window plus a popcount, and
// all four edges' loads are issued before their atomics.  A relaxation is an
// L2 load (filter) plus one hardware atomicMin on the 32-bit key or the
// packed 64-bit key|pred word; pushes are warp-aggregated.
//
// Delta-stepping (replaces the reference's host-driven current / pending /
// heavy queues, delta_stepping_hip_CSR.cpp:367-529):
//   * adjacency lists are sorted by weight when the graph is built, so the
//     light edges (w <= delta) of a vertex are a prefix of its row; the
//     prefix length per vertex is computed once per delta (k_light_count);
//   * light sub-phases relax only the prefix; every vertex settled in them is
//     appended once (stamp) to a member list, and a heavy phase relaxes the
//     suffix of each member once with its final label, like the reference's
//     heavy queue (relax_heavy_edges_kernel, :425-459);
//   * near queues (2, ping-pong) hold same-bucket improvements, deduplicated
//     per phase by a stamp word;
//   * a window of kRing buckets [win, win + kRing), one queue each,
//     deduplicated by a per-vertex "smallest bucket pushed" word;
//   * a far pile for buckets past the window, one entry per vertex (flag),
//     split into the next aligned window when the window is exhausted.
// The bucket rule is the reference's: uint32 weights use bucket = d / delta;
// float weights use floorf(d * (1.0f / delta)) clamped like bucket_index
// (delta_stepping_hip_CSR.cpp:233-239).  iterations_used counts buckets in
// which at least one vertex was settled, exactly the reference's count of
// outer iterations.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "b2_common.cuh"
#include "b2_internal.hpp"
#include "b2_relax.cuh"

namespace b2 {

enum Mode : int { kModeBF = 0, kModeDelta = 1 };
constexpr int kThreads = 512;
#ifndef B2_UNROLL
#define B2_UNROLL 4
#endif
#ifndef B2_SSSP_MINB      // resident blocks per SM the register budget of k_sssp is sized for
#define B2_SSSP_MINB 2
#endif
#ifndef B2_HUB_UNROLL
#define B2_HUB_UNROLL 4
#endif
#ifndef B2_HUB_GRAB
#define B2_HUB_GRAB 2
#endif
#ifndef B2_STATIC_NUM   // share of a phase's items dealt round-robin: NUM / 4 (the rest from a counter)
#define B2_STATIC_NUM 4
#endif
constexpr int kUnroll = B2_UNROLL;   // edge slots per lane per step

struct Params {
  uint32_t n;
  uint32_t source;
  const uint64_t* __restrict__ rowptr;
  const uint2* __restrict__ edges;
  const uint32_t* __restrict__ lightcnt;   // null: relax whole rows in every sub-phase
  void* dist;        // labels receiving atomicMin (BF: round k+1 values)
  void* dist_cur;    // BF: labels of round k (read side)
  uint32_t* pstamp;
  uint32_t* bstamp;
  uint32_t* farflag;
  uint32_t* hstamp;
  uint32_t* queues;
  HubEntry* hubs;
  uint32_t hub_cap;
  Control* ctl;
  TraceEntry* trace;
  uint32_t delta_u;
  float inv_delta;
  uint32_t hub_degree;
  uint32_t max_iters;
  uint32_t phase_base;
  uint32_t detect_negcycle;
  unsigned long long budget_ns;
  void* out_dist;
  int32_t* out_pred;
  uint32_t dist_is_out;   // `dist` aliases out_dist (no separate label buffer)
  const uint32_t* perm;   // degree-ordered graph: internal -> input id of every output slot (else null)
  const uint32_t* inv;    // degree-ordered graph: input -> internal id (else null)
  const uint64_t* __restrict__ in_rowptr;   // incoming CSR for the pull heavy pass (null: push only)
  const uint2* __restrict__ in_edges;       // (source, weight bits), rows sorted by weight
  const uint32_t* __restrict__ in_lightcnt; // light prefix of each incoming row
  float pull_factor;      // pull when the members' heavy out-edges exceed pull_factor x n
  uint32_t is_float;
  uint32_t fusion;        // light frontiers up to this size run as a LOCAL phase (0: off)
  uint32_t dense_min;     // delta: near / slot frontiers of at least this many entries are swept
  uint32_t qcap;          // entries each worklist queue may hold (<= n; a push past it is kErrQueueOverflow)
  ProgressBoard* board;   // mapped progress record (null: no progress callback)
};

// Bucket of a distance key under the phase's mapping
//   bucket = dbase_b + floor((d - dbase) / width).
// With dbase = 0 and dbase_b = 0 (delta-stepping; ADDS before its first
// re-basing) this is the reference rule: d / delta for uint32 and
// floorf(d * (1.0f / delta)) clamped to [0, kNoBucket) for float.  Keys below
// dbase belong to settled buckets and map to dbase_b - 1.
template <class W>
__device__ __forceinline__ uint32_t bucket_of(const PhaseRec& R, uint32_t key) {
  if (!W::kFloat) {
    if (key < R.dbase) return R.dbase_b ? R.dbase_b - 1 : 0;
    const uint32_t b = (key - R.dbase) / R.dq;
    return R.dbase_b + b;
  }
  const float d = key_to_f32(key);
  if (!isfinite(d)) return kNoBucket;
  const float bf = floorf((d - __uint_as_float(R.dbase)) * __uint_as_float(R.dinv));
  if (bf < 0.0f) return (R.dbase_b && R.dbase) ? R.dbase_b - 1 : R.dbase_b;
  if (bf + (float)R.dbase_b >= (float)kNoBucket) return kNoBucket - 1;
  return R.dbase_b + (uint32_t)bf;
}

__device__ __forceinline__ uint32_t* queue_ptr(const Params& P, uint32_t id) {
  return P.queues + (size_t)id * P.n;
}

__device__ __forceinline__ void set_error(const Params& P, uint32_t code, uint32_t site) {
  atomicCAS(&P.ctl->error, kErrNone, code);
  atomicExch(&P.ctl->error_site, site);
}

__device__ __forceinline__ PhaseRec load_rec(const Control* c) {
  PhaseRec r;
  const volatile uint32_t* src = (const volatile uint32_t*)&c->rec;
  uint32_t* dst = (uint32_t*)&r;
#pragma unroll
  for (int i = 0; i < (int)(sizeof(PhaseRec) / 4); ++i) dst[i] = src[i];
  return r;
}
__device__ __forceinline__ void store_rec(Control* c, const PhaseRec& r) {
  volatile uint32_t* dst = (volatile uint32_t*)&c->rec;
  const uint32_t* src = (const uint32_t*)&r;
#pragma unroll
  for (int i = 0; i < (int)(sizeof(PhaseRec) / 4); ++i) dst[i] = src[i];
}

// Per-warp push staging (shared memory).  Worklist insertions are collected
// per warp and published with one global atomicAdd per flush, so the queue
// counters (one address each) see ~1/100 of the per-push atomics; flushes
// happen when a buffer passes half full and at the end of every phase.
constexpr int kWarpsPerBlock = kThreads / 32;
constexpr uint32_t kNearBuf = 256, kFarBuf = 256, kSlotBuf = 256, kMemBuf = 128;
constexpr uint32_t kDenseSpan = 256;   // vertices per sweep work item (8 per lane)
constexpr uint32_t kListBuf = kDenseSpan + 32;   // one span's vertices + fewer than 32 carried
constexpr uint32_t kStageWords = kNearBuf + kFarBuf + 2 * kSlotBuf + kMemBuf + kListBuf;
constexpr size_t kStageBytes = (size_t)kWarpsPerBlock * kStageWords * 4;
struct WarpQ {
  uint32_t* nearb;   // kNearBuf vertex ids
  uint32_t* farb;    // kFarBuf
  uint32_t* slotb;   // kSlotBuf (vertex, slot) pairs as 2 words
  uint32_t* memb;    // kMemBuf
  uint32_t* listb;   // kListBuf frontier vertices found by a sweep
  uint32_t nn = 0, nf = 0, ns = 0, nm = 0;
};

struct Tally {
  unsigned long long edges = 0, impr = 0, pushes = 0;
  uint64_t keep = 0;   // L2 evict_last cache policy for label traffic
  WarpQ q;
};

// ---------------------------------------------------------------------------
// Append the wanting lanes' vertices to a warp buffer (warp-collective).
__device__ __forceinline__ void stage(uint32_t* buf, uint32_t& cnt, bool want, uint32_t v) {
  const uint32_t b = __ballot_sync(0xffffffffu, want);
  if (want) buf[cnt + __popc(b & ((1u << lane_id()) - 1u))] = v;
  cnt += __popc(b);
}

// Publish a staged buffer to queue `qid` with one atomic (warp-collective).
__device__ __forceinline__ void publish(const Params& P, uint32_t* counter, uint32_t qid, const uint32_t* buf,
                                        uint32_t cnt, uint32_t site) {
  if (cnt == 0) return;
  __syncwarp();
  uint32_t base = 0;
  if (lane_id() == 0) base = atomicAdd(counter, cnt);
  base = __shfl_sync(0xffffffffu, base, 0);
  if ((uint64_t)base + cnt > P.qcap) {
    if (lane_id() == 0) set_error(P, kErrQueueOverflow, site);
    return;
  }
  uint32_t* dst = queue_ptr(P, qid) + base;
  for (uint32_t i = lane_id(); i < cnt; i += 32) dst[i] = buf[i];
  __syncwarp();
}

// Window-slot entries carry their slot: publish one slot group at a time.
__device__ __forceinline__ void publish_slots(const Params& P, WarpQ& q) {
  Control* c = P.ctl;
  __syncwarp();
  uint32_t remaining = q.ns;
  // entries are (v, slot) pairs; process in rounds, one distinct slot per round
  while (remaining) {
    uint32_t s0 = q.slotb[2 * 0 + 1];
    // lane-strided scan: count entries with slot s0
    uint32_t mine = 0;
    for (uint32_t i = lane_id(); i < q.ns; i += 32)
      if (q.slotb[2 * i + 1] == s0) ++mine;
    const uint32_t incl = warp_incl_scan(mine);
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(&c->slot_count[s0], total);
    base = __shfl_sync(0xffffffffu, base, 0);
    if ((uint64_t)base + total > P.qcap) {
      if (lane_id() == 0) set_error(P, kErrQueueOverflow, 12);
      q.ns = 0;
      return;
    }
    uint32_t pos = base + incl - mine;
    uint32_t* dst = queue_ptr(P, kQSlot0 + s0);
    for (uint32_t i = lane_id(); i < q.ns; i += 32)
      if (q.slotb[2 * i + 1] == s0) dst[pos++] = q.slotb[2 * i];
    __syncwarp();
    if (total == q.ns) {   // one slot only (the usual case)
      q.ns = 0;
      return;
    }
    // compact the entries of other slots to the front, 32 at a time: every
    // lane reads its entry before any lane writes, and a write position never
    // passes the chunk being read
    uint32_t kept = 0;
    for (uint32_t i0 = 0; i0 < q.ns; i0 += 32) {
      const uint32_t i = i0 + lane_id();
      uint32_t ev = 0, es = s0;
      if (i < q.ns) { ev = q.slotb[2 * i]; es = q.slotb[2 * i + 1]; }
      const bool keep = es != s0;
      const uint32_t bal = __ballot_sync(0xffffffffu, keep);
      __syncwarp();
      if (keep) {
        const uint32_t d = kept + __popc(bal & ((1u << lane_id()) - 1u));
        q.slotb[2 * d] = ev;
        q.slotb[2 * d + 1] = es;
      }
      kept += __popc(bal);
      __syncwarp();
    }
    q.ns = kept;
    remaining = kept;
  }
}

template <int MODE>
__device__ __forceinline__ void flush_all(const Params& P, const PhaseRec& R, WarpQ& q, bool force) {
  Control* c = P.ctl;
  if (q.nn && (force || q.nn > kNearBuf / 2)) {
    publish(P, &c->near_count[R.push_q & 1], R.push_q, q.nearb, q.nn, 11);
    q.nn = 0;
  }
  if (MODE == kModeBF) return;
  if (q.nf && (force || q.nf > kFarBuf / 2)) {
    publish(P, &c->far_count[R.far_sel], kQFar0 + R.far_sel, q.farb, q.nf, 13);
    q.nf = 0;
  }
  if (q.nm && (force || q.nm > kMemBuf / 2)) {
    publish(P, &c->members_count, kQMembers, q.memb, q.nm, 14);
    q.nm = 0;
  }
  if (q.ns && (force || q.ns > kSlotBuf / 2)) publish_slots(P, q);
  // (a relax batch adds at most 4 x 32 entries per buffer, so flushing past
  //  half of a 256-entry buffer never overflows it)
}

// Route one improvement per lane into the right worklist (warp-collective:
// all 32 lanes call it with `improved` possibly false).  Dedup atomics stay
// per vertex; the insertion itself is staged in the warp's buffers.
template <class W, int MODE>
__device__ __forceinline__ void route(const Params& P, const PhaseRec& R, bool improved, uint32_t v,
                                      uint32_t cand, Tally& t) {
  if (!__any_sync(0xffffffffu, improved)) return;
  Control* c = P.ctl;
  if (MODE == kModeBF) {
    const bool want = improved && atomicExch(&P.pstamp[v], R.stamp) != R.stamp;
    stage(t.q.nearb, t.q.nn, want, v);
    t.pushes += want ? 1 : 0;
    return;
  }
  uint32_t b = 0;
  int cls = 0;  // 1 near, 2 window slot, 3 far
  if (improved) {
    b = bucket_of<W>(R, cand);
    if (b <= R.cur) cls = 1;
    else if (b < R.win + (uint32_t)kRing) cls = 2;
    else cls = 3;
  }
  if (__any_sync(0xffffffffu, cls == 1)) {
    const bool want = (cls == 1) && atomicExch(&P.pstamp[v], R.stamp) != R.stamp;
    stage(t.q.nearb, t.q.nn, want, v);
    t.pushes += want ? 1 : 0;
  }
  if (__any_sync(0xffffffffu, cls == 2)) {
    const bool want = (cls == 2) && atomicMin(&P.bstamp[v], b) > b;
    const uint32_t bal = __ballot_sync(0xffffffffu, want);
    if (want) {
      const uint32_t pos = t.q.ns + __popc(bal & ((1u << lane_id()) - 1u));
      t.q.slotb[2 * pos] = v;
      t.q.slotb[2 * pos + 1] = b - R.win;
    }
    t.q.ns += __popc(bal);
    t.pushes += want ? 1 : 0;
  }
  if (__any_sync(0xffffffffu, cls == 3)) {
    bool want = false;
    uint32_t bmin = 0xFFFFFFFFu;
    if (cls == 3 && atomicMin(&P.bstamp[v], b) > b) {
      bmin = b;
      want = atomicExch(&P.farflag[v], 1u) == 0u;
    }
    bmin = __reduce_min_sync(0xffffffffu, bmin);
    if (lane_id() == 0 && bmin != 0xFFFFFFFFu) atomicMin(&c->far_min, bmin);
    stage(t.q.farb, t.q.nf, want, v);
    t.pushes += want ? 1 : 0;
  }
}

// Route the improvements of U edge slots per lane (warp-collective).  The
// dedup atomics of every slot go out before any result is read, so their
// round trips overlap; then each slot is staged in order.  Staged pushes are
// flushed after every kUnroll slots, so a warp buffer never takes more than
// kUnroll x 32 entries past its flush mark.
template <class W, int MODE, int U>
__device__ __forceinline__ void route_batch(const Params& P, const PhaseRec& R, const bool (&imp)[U],
                                            const uint2 (&ed)[U], const uint32_t (&cand)[U], Tally& t) {
  bool any_imp = false;
#pragma unroll
  for (int q = 0; q < U; ++q) any_imp = any_imp || imp[q];
  if (!__any_sync(0xffffffffu, any_imp)) return;
  Control* c = P.ctl;
  uint32_t b[U], onear[U], obuck[U];
  int cls[U];   // 0 none, 1 near, 2 window slot, 3 far
#pragma unroll
  for (int q = 0; q < U; ++q) {
    b[q] = 0;
    cls[q] = 0;
    if (imp[q]) {
      if (MODE == kModeBF) {
        cls[q] = 1;
      } else {
        b[q] = bucket_of<W>(R, cand[q]);
        cls[q] = b[q] <= R.cur ? 1 : (b[q] < R.win + (uint32_t)kRing ? 2 : 3);
      }
    }
    // defaults read as "already queued"
    onear[q] = atom_exch_if(cls[q] == 1, &P.pstamp[ed[q].x], R.stamp, R.stamp);
    obuck[q] = MODE == kModeBF ? 0u : atom_min_if(cls[q] >= 2, &P.bstamp[ed[q].x], b[q], 0u);
  }
  uint32_t ofar[U];
  bool any_far = false;
#pragma unroll
  for (int q = 0; q < U; ++q) {
    const bool f = MODE != kModeBF && cls[q] == 3 && obuck[q] > b[q];
    any_far = any_far || f;
    ofar[q] = f ? 0u : 1u;
  }
  if (MODE != kModeBF && any_far) {
#pragma unroll
    for (int q = 0; q < U; ++q) ofar[q] = atom_exch_if(ofar[q] == 0u, &P.farflag[ed[q].x], 1u, 1u);
  }
#pragma unroll
  for (int q = 0; q < U; ++q) {
    const uint32_t v = ed[q].x;
    if (__any_sync(0xffffffffu, cls[q] == 1)) {
      const bool want = cls[q] == 1 && onear[q] != R.stamp;
      stage(t.q.nearb, t.q.nn, want, v);
      t.pushes += want ? 1 : 0;
    }
    if (MODE != kModeBF) {
      if (__any_sync(0xffffffffu, cls[q] == 2)) {
        const bool want = cls[q] == 2 && obuck[q] > b[q];
        const uint32_t bal = __ballot_sync(0xffffffffu, want);
        if (want) {
          const uint32_t pos = t.q.ns + __popc(bal & ((1u << lane_id()) - 1u));
          t.q.slotb[2 * pos] = v;
          t.q.slotb[2 * pos + 1] = b[q] - R.win;
        }
        t.q.ns += __popc(bal);
        t.pushes += want ? 1 : 0;
      }
      if (__any_sync(0xffffffffu, cls[q] == 3)) {
        const bool lowered = cls[q] == 3 && obuck[q] > b[q];
        const bool want = lowered && ofar[q] == 0u;
        const uint32_t bmin = __reduce_min_sync(0xffffffffu, lowered ? b[q] : 0xFFFFFFFFu);
        if (lane_id() == 0 && bmin != 0xFFFFFFFFu) atomicMin(&c->far_min, bmin);
        stage(t.q.farb, t.q.nf, want, v);
        t.pushes += want ? 1 : 0;
      }
    }
    if ((q % kUnroll) == kUnroll - 1) flush_all<MODE>(P, R, t.q, false);
  }
}

// Relax U edge slots per lane: label loads first, then the atomics of every
// slot (issued before any result is read), then routing.
template <class W, bool PRED, int MODE, int U>
__device__ __forceinline__ void relax_batch(const Params& P, const PhaseRec& R, const bool (&act)[U],
                                            const uint32_t (&src)[U], const uint32_t (&dsrc)[U],
                                            const uint2 (&ed)[U], Tally& t) {
  using L = Label<PRED>;
  typename L::T* lab = (typename L::T*)P.dist;
  uint32_t cand[U];
  typename L::T cur[U], old[U];
  bool imp[U];
#pragma unroll
  for (int q = 0; q < U; ++q) {
    cand[q] = act[q] ? W::extend(dsrc[q], ed[q].y) : kInfKey;
    cur[q] = ld_keep_if(cand[q] != kInfKey, lab + ed[q].x, t.keep, L::kInf);
  }
#pragma unroll
  for (int q = 0; q < U; ++q) {
    const typename L::T cw = L::make(cand[q], src[q]);
    // not issued: old = 0 reads as "no improvement"
    old[q] = atom_min_keep_if(cand[q] != kInfKey && cw < cur[q], lab + ed[q].x, cw, t.keep, (typename L::T)0);
  }
#pragma unroll
  for (int q = 0; q < U; ++q) {
    // (PRED: a smaller predecessor at an equal distance updates the word
    //  but does not re-expand the vertex.)
    imp[q] = cand[q] < L::key(old[q]);
    t.edges += act[q] ? 1 : 0;
    t.impr += imp[q] ? 1 : 0;
  }
  route_batch<W, MODE, U>(P, R, imp, ed, cand, t);
}

template <class W, bool PRED, int MODE>
__device__ __forceinline__ uint32_t src_key(const Params& P, uint32_t v) {
  using L = Label<PRED>;
  const typename L::T* lab = (const typename L::T*)(MODE == kModeBF ? P.dist_cur : P.dist);
  return L::key(ldcg(lab + v));
}

// Edge range of v relaxed by this phase: the light prefix, the heavy suffix,
// or the whole row.
__device__ __forceinline__ void phase_range(const Params& P, const PhaseRec& R, uint32_t v, uint64_t& lo,
                                            uint64_t& hi, bool& has_heavy, uint64_t* row_end = nullptr) {
  const uint64_t b = __ldg(&P.rowptr[v]);
  const uint64_t e = __ldg(&P.rowptr[v + 1]);
  if (row_end) *row_end = e;
  has_heavy = false;
  if (P.lightcnt) {
    const uint64_t l = b + __ldg(&P.lightcnt[v]);
    if (R.heavy) { lo = l; hi = e; }
    else { lo = b; hi = l; has_heavy = e > l; }
  } else {
    lo = b;
    hi = e;
  }
}

// ---------------------------------------------------------------------------
// One hub chunk: 256 consecutive edges of a high-degree vertex's phase range.
template <class W, bool PRED, int MODE>
__device__ __forceinline__ void hub_chunk(const Params& P, const PhaseRec& R, uint32_t item, Tally& t) {
  const uint32_t lane = lane_id();
  const HubEntry* H = P.hubs + (size_t)(R.hub_in & 1) * P.hub_cap;
  const uint2 h = ldcg(reinterpret_cast<const uint2*>(H + item));
  const uint32_t v = h.x;
  uint64_t rlo, rhi;
  bool hh;
  phase_range(P, R, v, rlo, rhi, hh);   // issued with the label load
  const uint32_t du = src_key<W, PRED, MODE>(P, v);
  bool valid = du != kInfKey;
  if (MODE == kModeDelta) valid = valid && bucket_of<W>(R, du) == R.cur;
  if (!valid) return;
  const uint64_t e0 = rlo + (uint64_t)h.y * kHubChunk;
  const uint64_t e1 = min(rhi, e0 + kHubChunk);
  // B2_HUB_UNROLL edge loads per lane in flight per step
  constexpr int U = B2_HUB_UNROLL;
  for (uint64_t eb = e0; eb < e1; eb += 32 * U) {
    bool act[U];
    uint32_t src[U], dsrc[U];
    uint2 ed[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
      const uint64_t e = eb + 32 * q + lane;
      act[q] = e < e1;
      src[q] = v;
      dsrc[q] = du;
      ed[q] = act[q] ? __ldcs(&P.edges[e]) : make_uint2(0, 0);
    }
    relax_batch<W, PRED, MODE, U>(P, R, act, src, dsrc, ed, t);
  }
}

// Expand up to 32 frontier vertices, one per lane (`present` lanes hold one).
template <class W, bool PRED, int MODE>
__device__ __forceinline__ void expand_vertices(const Params& P, const PhaseRec& R, uint32_t v, bool present,
                                                Tally& t) {
  const uint32_t lane = lane_id();
  Control* c = P.ctl;
  const bool members = MODE == kModeDelta && P.lightcnt && !R.heavy;
  uint32_t du = kInfKey;
  uint64_t lo = 0, hi = 0, row_end = 0;
  bool valid = false, has_heavy = false;
  if (present) {
    // the row bounds do not depend on the label: both loads go out together
    // (one dependent memory round trip less per item)
    phase_range(P, R, v, lo, hi, has_heavy, &row_end);
    du = src_key<W, PRED, MODE>(P, v);
    valid = du != kInfKey;
    if (MODE == kModeDelta) valid = valid && bucket_of<W>(R, du) == R.cur;
    if (!valid) {
      lo = hi = row_end = 0;
      has_heavy = false;
    }
  }
  if (MODE == kModeDelta) {
    if (__any_sync(0xffffffffu, valid) && lane == 0 && ldcg(&c->bucket_valid) == 0) c->bucket_valid = 1;
    if (members) {
      // settled in this light round: its heavy suffix is relaxed once by the heavy phase
      const bool want = valid && has_heavy && atomicExch(&P.hstamp[v], R.hround) != R.hround;
      if (P.in_rowptr) {
        // push cost of the heavy pass and the bucket's smallest label (the pull's early-exit bound)
        unsigned long long hv = want ? (unsigned long long)(row_end - hi) : 0ull;
        uint32_t mk = valid ? du : 0xFFFFFFFFu;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          hv += __shfl_xor_sync(0xffffffffu, hv, o);
          mk = min(mk, __shfl_xor_sync(0xffffffffu, mk, o));
        }
        if (lane == 0) {
          if (hv) atomicAdd(&c->member_heavy, hv);
          if (mk != 0xFFFFFFFFu) atomicMin(&c->cur_min_key, mk);
        }
      }
      stage(t.q.memb, t.q.nm, want, v);
      if (t.q.nm > kMemBuf / 2) {
        publish(P, &c->members_count, kQMembers, t.q.memb, t.q.nm, 14);
        t.q.nm = 0;
      }
    }
  }
  uint32_t deg = valid ? (uint32_t)min(hi - lo, (uint64_t)0xFFFFFFFFull) : 0u;
  // high-degree ranges -> one hub-list entry per 256-edge chunk, written by
  // the whole warp, taken by any warp in the next phase
  const uint32_t hub_deg = R.kind == kPhaseLocal ? 0xFFFFFFFFu : P.hub_degree;
  uint32_t hubs = __ballot_sync(0xffffffffu, deg >= hub_deg);
  while (hubs) {
    const uint32_t hl = __ffs(hubs) - 1;
    hubs &= hubs - 1;
    const uint32_t hv = __shfl_sync(0xffffffffu, v, hl);
    const uint32_t nch = (__shfl_sync(0xffffffffu, deg, hl) + kHubChunk - 1) / kHubChunk;
    uint32_t hb = 0;
    if (lane == 0) hb = atomicAdd(&c->hub_count[R.hub_out & 1], nch);
    hb = __shfl_sync(0xffffffffu, hb, 0);
    if ((uint64_t)hb + nch <= P.hub_cap) {
      HubEntry* H = P.hubs + (size_t)(R.hub_out & 1) * P.hub_cap;
      for (uint32_t j = lane; j < nch; j += 32)
        *reinterpret_cast<uint2*>(H + hb + j) = make_uint2(hv, j);
    } else if (lane == 0) {
      set_error(P, kErrQueueOverflow, 20);
    }
    if (lane == hl) deg = 0;
  }
  // compact the lanes that have edges to relax
  const uint32_t nz = __ballot_sync(0xffffffffu, deg > 0);
  const uint32_t k = __popc(nz);
  if (k == 0) return;
  const bool has = lane < k;
  const uint32_t sl = nth_set_bit(nz, has ? lane : 0u);
  const uint32_t cv = __shfl_sync(0xffffffffu, v, sl);
  const uint32_t cdu = __shfl_sync(0xffffffffu, du, sl);
  const uint32_t sdeg = __shfl_sync(0xffffffffu, deg, sl);
  const uint32_t cdeg = has ? sdeg : 0u;
  const unsigned long long clo = shfl64(lo, sl);
  const uint32_t incl = warp_incl_scan(cdeg);
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  const uint32_t excl = incl - cdeg;
  const unsigned long long ebase = clo - excl;   // edge index of slot p owned here = ebase + p
  uint32_t started = 0;                           // ranges that start before the window
  for (uint32_t eb = 0; eb < total; eb += 32 * kUnroll) {
    bool act[kUnroll];
    uint32_t src[kUnroll], dsrc[kUnroll];
    uint2 ed[kUnroll];
#pragma unroll
    for (int q = 0; q < kUnroll; ++q) {
      const uint32_t w0 = eb + 32 * q;
      const uint32_t bit = (has && excl >= w0 && excl < w0 + 32) ? (1u << (excl - w0)) : 0u;
      const uint32_t starts = __reduce_or_sync(0xffffffffu, bit);
      uint32_t own = started + __popc(starts & lanemask_le()) - 1;
      started += __popc(starts);
      own = min(own, 31u);
      const uint32_t p = w0 + lane;
      act[q] = p < total;
      src[q] = __shfl_sync(0xffffffffu, cv, own);
      dsrc[q] = __shfl_sync(0xffffffffu, cdu, own);
      const unsigned long long e = shfl64(ebase, own) + p;
      ed[q] = act[q] ? __ldcs(&P.edges[e]) : make_uint2(0, 0);
    }
    relax_batch<W, PRED, MODE, kUnroll>(P, R, act, src, dsrc, ed, t);
  }
}

// Append the frontier's vertices among [span * 256, span * 256 + 256) (stamp
// == R.fstamp; 8 consecutive vertices per lane) to the warp's list after its
// `carry` entries, in vertex order; returns the new length.  A stamp that
// changes under the sweep belongs to a vertex improved again in this phase: it
// sits in this phase's near queue and is expanded next phase with its newer
// label.
__device__ __forceinline__ uint32_t sweep_span(const Params& P, const PhaseRec& R, uint32_t span, uint32_t* list,
                                               uint32_t carry) {
  const uint32_t lane = lane_id();
  const uint32_t* S = R.dense == kDenseSlot ? P.bstamp : P.pstamp;
  const uint32_t v0 = span * kDenseSpan + 8u * lane;
  uint32_t m = 0;
  if ((uint64_t)v0 + 8 <= P.n) {
    const uint4 a = __ldcg(reinterpret_cast<const uint4*>(S + v0));
    const uint4 b = __ldcg(reinterpret_cast<const uint4*>(S + v0 + 4));
    m = (a.x == R.fstamp ? 1u : 0u) | (a.y == R.fstamp ? 2u : 0u) | (a.z == R.fstamp ? 4u : 0u) |
        (a.w == R.fstamp ? 8u : 0u) | (b.x == R.fstamp ? 16u : 0u) | (b.y == R.fstamp ? 32u : 0u) |
        (b.z == R.fstamp ? 64u : 0u) | (b.w == R.fstamp ? 128u : 0u);
  } else {
    for (uint32_t k = 0; k < 8 && v0 + k < P.n; ++k) m |= (ldcg(S + v0 + k) == R.fstamp ? 1u : 0u) << k;
  }
  const uint32_t cnt = __popc(m);
  const uint32_t incl = warp_incl_scan(cnt);
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0) return carry;
  __syncwarp();   // the previous item's reads of the list are done
  uint32_t pos = carry + incl - cnt;
  while (m) {
    const uint32_t k = __ffs(m) - 1;
    m &= m - 1;
    list[pos++] = v0 + k;
  }
  __syncwarp();
  return carry + total;
}

// One frontier work item: entries [g item, g item + g) of the frontier queue
// (g <= 32 vertices, one per lane), or the frontier vertices of sweep span
// `item`.  A sweep expands only whole groups of 32 and carries the rest
// (`carry`) into the warp's next item, so sparse spans do not run lanes idle;
// `flush` expands the carried rest at the end of the phase.
template <class W, bool PRED, int MODE>
__device__ __forceinline__ void frontier_item(const Params& P, const PhaseRec& R, uint32_t item, bool dense,
                                              bool flush, uint32_t& carry, Tally& t, uint32_t g = 32) {
  const uint32_t lane = lane_id();
  const uint32_t base = item * g;
  uint32_t total, limit;
  if (dense) {
    total = flush ? carry : sweep_span(P, R, item, t.q.listb, carry);
    limit = flush ? total : (total & ~31u);
  } else {
    total = min(g, R.fcount - base);
    limit = total;
  }
  for (uint32_t j0 = 0; j0 < limit; j0 += 32) {
    const bool present = j0 + lane < total;
    uint32_t v = 0;
    if (present) v = dense ? t.q.listb[j0 + lane] : ldcg(queue_ptr(P, R.fq) + base + lane);
    expand_vertices<W, PRED, MODE>(P, R, v, present, t);
  }
  if (dense) {
    const uint32_t rest = total - limit;   // < 32
    if (limit && rest) {
      __syncwarp();
      const uint32_t v = lane < rest ? t.q.listb[limit + lane] : 0u;
      __syncwarp();
      if (lane < rest) t.q.listb[lane] = v;
      __syncwarp();
    }
    carry = rest;
  }
}

// One frontier chunk of the queue (block-local sub-phases).
template <class W, bool PRED, int MODE>
__device__ __forceinline__ void frontier_chunk(const Params& P, const PhaseRec& R, uint32_t base, Tally& t) {
  uint32_t carry = 0;
  frontier_item<W, PRED, MODE>(P, R, base / 32, false, false, carry, t);
}

constexpr uint32_t kHubGrab = B2_HUB_GRAB;   // hub chunks per work item

// A relaxation phase: hub chunks of the previous phase (two per item), then
// 32-vertex frontier chunks (or 256-vertex sweep items).  Whole rounds of
// items are dealt round-robin to the warps (no atomics); only the last partial
// round (fewer items than warps) is handed out from a phase counter.  Handing
// out a quarter of the items from the counter, so that no warp idles behind a
// long item, measured 8 % slower on a grid and 2 % on RMAT-24: thousands of
// warps contend for one counter.
//
// Queue items hold g vertices: 32 when the frontier gives every warp at least
// one full item, else the largest power of two that still does, down to one
// vertex per warp.  A small frontier of long rows (a few hundred vertices of
// ~200 edges) then spreads over the grid instead of leaving a few warps to
// walk 32 long rows each while the rest wait at the barrier.
template <class W, bool PRED, int MODE>
__device__ void process_phase(const Params& P, const PhaseRec& R, Tally& t) {
  const uint32_t nhub = min(R.hub_in_chunks, P.hub_cap);
  const uint32_t nhg = (nhub + kHubGrab - 1) / kHubGrab;
  const bool dense = MODE == kModeDelta && R.dense != kDenseOff;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t g = 32;
  if (!dense)
    while (g > 1 && (R.fcount + g - 1) / g < nwarps) g >>= 1;
  const uint32_t nfc = dense ? (P.n + kDenseSpan - 1) / kDenseSpan : (R.fcount + g - 1) / g;
  const uint32_t items = nhg + nfc;
  const uint32_t rounds = (items * B2_STATIC_NUM / 4) / nwarps;
  const uint32_t nstatic = rounds * nwarps;
  Control* c = P.ctl;
  uint32_t carry = 0;   // swept vertices waiting in the warp's list
  for (uint32_t r = 0;; ++r) {
    uint32_t item = 0;
    if (r < rounds) {
      item = r * nwarps + gwarp;
    } else {
      if (lane_id() == 0) item = atomicAdd(&c->work_next, 1u);
      item = __shfl_sync(0xffffffffu, item, 0) + nstatic;
    }
    const bool done = item >= items;
    if (done && carry == 0) break;
    if (!done && item < nhg) {
      const uint32_t h1 = min(nhub, (item + 1) * kHubGrab);
      for (uint32_t h = item * kHubGrab; h < h1; ++h) hub_chunk<W, PRED, MODE>(P, R, h, t);
    } else {
      frontier_item<W, PRED, MODE>(P, R, done ? 0u : item - nhg, dense, done, carry, t, g);
    }
    if (done) break;
  }
  flush_all<MODE>(P, R, t.q, true);
}

// Heavy pass in the pull direction (delta mode).  The push pass relaxes the
// heavy out-edges (w > delta) of every member, i.e. of every vertex whose label
// lies in the current bucket.  Here each unsettled vertex v scans its heavy
// in-edges in weight order and keeps the smallest (distance, source) word over
// in-neighbours in the current bucket -- the same minimum the push pass's
// atomics reach.  A member's label is at least lb (the smallest label of the
// bucket), so once lb + w cannot beat v's best the rest of the row cannot
// either and the scan stops.  One lane per vertex; improvements are routed
// like pushed ones.
template <class W, bool PRED>
__device__ void pull_phase(const Params& P, const PhaseRec& R, Tally& t) {
  using L = Label<PRED>;
  typename L::T* lab = (typename L::T*)P.dist;
  const uint32_t lb = ldcg(&P.ctl->cur_min_key);
  const uint32_t lane = lane_id();
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base = gwarp * 32; base < P.n; base += nwarps * 32) {
    const uint32_t v = base + lane;
    bool improved = false;
    uint32_t best_key = kInfKey;
    if (v < P.n && lb != 0xFFFFFFFFu) {
      const typename L::T cw = ld_keep(lab + v, t.keep);
      const uint32_t ck = L::key(cw);
      if (ck == kInfKey || bucket_of<W>(R, ck) > R.cur) {
        uint64_t e = __ldg(&P.in_rowptr[v]) + __ldg(&P.in_lightcnt[v]);
        const uint64_t e1 = __ldg(&P.in_rowptr[v + 1]);
        typename L::T best = cw;
        unsigned long long scanned = 0;
        for (; e < e1; ++e) {
          const uint2 ed = __ldg(&P.in_edges[e]);
          const uint32_t bound = W::extend(lb, ed.y);   // no member reaches v for less via this or later edges
          if (PRED ? bound > L::key(best) : bound >= L::key(best)) break;
          ++scanned;
          const uint32_t ku = L::key(ld_keep(lab + ed.x, t.keep));
          if (ku == kInfKey || bucket_of<W>(R, ku) != R.cur) continue;
          const typename L::T cand = L::make(W::extend(ku, ed.y), ed.x);
          if (cand < best) best = cand;
        }
        t.edges += scanned;
        if (best < cw) {
          const typename L::T old = atom_min_keep(lab + v, best, t.keep);
          best_key = L::key(best);
          improved = best_key < L::key(old);
          t.impr += improved ? 1 : 0;
        }
      }
    }
    route<W, kModeDelta>(P, R, improved, v, best_key, t);
    flush_all<kModeDelta>(P, R, t.q, false);
  }
  flush_all<kModeDelta>(P, R, t.q, true);
}

// ---------------------------------------------------------------------------
// Manager steps (one thread, every other block parked at the barrier).
__device__ __forceinline__ uint32_t vld(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ unsigned long long vld64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}

__device__ __forceinline__ void trace_phase(const Params& P, const PhaseRec& r, uint32_t tag) {
  if (!P.trace) return;
  Control* c = P.ctl;
  const uint32_t i = vld(&c->trace_n);
  if (i >= kTraceCap) return;
  TraceEntry e;
  e.kind = r.kind | (r.heavy ? 0x100u : 0u) | (r.dense ? 0x200u : 0u);
  e.fcount = r.fcount;
  e.hub_chunks = r.hub_in_chunks;
  e.cur = tag;
  e.t_ns = globaltimer_ns() - c->t_start;
  P.trace[i] = e;
  c->trace_n = i + 1;
}

template <bool PRED, int MODE>
__device__ void manager_init(const Params& P) {
  using L = Label<PRED>;
  Control* c = P.ctl;
  typename L::T* lab = (typename L::T*)P.dist;
  // Source label: key 0 with predecessor field 0, so no equal-distance
  // candidate can ever replace it; the output maps pred[source] to -1.
  const uint32_t zk = P.is_float ? f32_to_key(0.0f) : 0u;
  lab[P.source] = L::make(zk, 0u);
  if (MODE == kModeBF) ((typename L::T*)P.dist_cur)[P.source] = L::make(zk, 0u);
  queue_ptr(P, kQNear0)[0] = P.source;
  c->near_count[0] = 1;
  c->near_count[1] = 0;
  c->far_min = 0xFFFFFFFFu;
  c->far_min_next = 0xFFFFFFFFu;
  c->t_start = globaltimer_ns();
  PhaseRec r;
  memset(&r, 0, sizeof(r));
  r.kind = kPhaseProcess;
  r.phase = 1;
  r.fq = kQNear0;
  r.fcount = 1;
  r.push_q = kQNear1;
  r.stamp = P.phase_base + 1;
  c->stamp_ctr = 2;
  r.hround = P.phase_base + 1;
  r.hub_in = 1;
  r.hub_out = 0;
  r.iter = 1;
  r.dq = P.delta_u;
  r.dinv = __float_as_uint(P.inv_delta);
  r.dbase = 0;
  r.dbase_b = 0;
  c->cur_min_key = 0xFFFFFFFFu;
  c->member_heavy = 0;
  store_rec(c, r);
}

// Whole-solve budget: a phase sequence that outlives it ends the kernel with
// kErrTimeout instead of looping.
__device__ __forceinline__ bool over_budget(const Params& P, PhaseRec& nx) {
  Control* c = P.ctl;
  if (globaltimer_ns() - c->t_start > P.budget_ns || nx.phase > 0x7fffffffu) {
    atomicCAS(&c->error, kErrNone, (uint32_t)kErrTimeout);
    c->error_site = 2;
    nx.kind = kPhaseDone;
    store_rec(c, nx);
    return true;
  }
  return false;
}

__device__ __forceinline__ void consume_queue(Control* c, uint32_t fq) {
  if (fq == kQNear0 || fq == kQNear1) c->near_count[fq] = 0;
  else if (fq == kQMembers) c->members_count = 0;
  else if (fq >= kQSlot0 && fq < kQSlot0 + kRing) c->slot_count[fq - kQSlot0] = 0;
}

__device__ __forceinline__ void consume_process_counters(Control* c, const PhaseRec& r) {
  if (r.fq == kQNear0 || r.fq == kQNear1) c->near_count[r.fq] = 0;
  else if (r.fq == kQMembers) c->members_count = 0;
  else if (r.fq >= kQSlot0 && r.fq < kQSlot0 + kRing) c->slot_count[r.fq - kQSlot0] = 0;
  if (r.hub_in_chunks) c->hub_count[r.hub_in & 1] = 0u;
}

// BF round bookkeeping.  PhaseRec.aux is the round's role: 0 ordinary round,
// 2 ordinary round whose commit precedes the negative-cycle probe, 1 the probe
// round (python reference: one extra relaxation after max_iters,
// minplus_bellman_ford.py:92-99).  At FINAL, aux = 1 means "output the
// committed round".
__device__ void manager_bf(const Params& P) {
  Control* c = P.ctl;
  const PhaseRec r = load_rec(c);
  trace_phase(P, r, r.iter);
  PhaseRec nx = r;
  nx.phase = r.phase + 1;
  c->phases = vld(&c->phases) + 1;
  if (r.kind == kPhaseFinal) { nx.kind = kPhaseDone; store_rec(c, nx); return; }
  if (over_budget(P, nx)) return;
  if (r.kind == kPhaseCommit) {
    nx.kind = kPhaseProcess;
    nx.fq = r.fq;
    nx.fcount = r.fcount;
    nx.push_q = r.fq ^ 1u;
    nx.stamp = P.phase_base + (c->stamp_ctr++);
    nx.hub_in = r.hub_out ^ 1u;
    nx.hub_in_count = 0;
    nx.hub_in_chunks = 0;
    nx.iter = r.iter + 1;
    nx.aux = (r.aux == 2u) ? 1u : 0u;
    store_rec(c, nx);
    return;
  }
  consume_process_counters(c, r);
  const uint32_t hch = vld(&c->hub_count[r.hub_out & 1]);
  const uint32_t hcnt = hch;
  if (hch > 0) {   // hub chunks of this round: same round, same push queue and stamp
    nx.kind = kPhaseProcess;
    nx.fq = kQNone;
    nx.fcount = 0;
    nx.hub_in = r.hub_out;
    nx.hub_in_count = hcnt;
    nx.hub_in_chunks = hch;
    nx.hub_out = r.hub_out ^ 1u;
    store_rec(c, nx);
    return;
  }
  const uint32_t nn = vld(&c->near_count[r.push_q & 1]);
  const bool changed = nn > 0;
  nx.hub_in_chunks = 0;
  nx.hub_in_count = 0;
  if (r.aux == 1u) {
    c->negative_cycle = changed ? 1u : 0u;
    nx.kind = kPhaseFinal;   // aux stays 1: output the committed round
    store_rec(c, nx);
    return;
  }
  c->iterations = r.iter;
  publish_progress(P.board, r.iter, changed ? 1u : 0u, globaltimer_ns() - c->t_start);
  if (!changed) {
    c->converged = 1;
    c->first_unchanged = r.iter;
    nx.kind = kPhaseFinal;
    nx.aux = 0u;
    store_rec(c, nx);
    return;
  }
  if (r.iter >= P.max_iters && !P.detect_negcycle) {
    nx.kind = kPhaseFinal;
    nx.aux = 0u;
    store_rec(c, nx);
    return;
  }
  nx.kind = kPhaseCommit;
  nx.fq = r.push_q;
  nx.fcount = nn;
  nx.aux = (r.iter >= P.max_iters) ? 2u : 0u;
  store_rec(c, nx);
}

// A large near or slot frontier is found by a stamp sweep (see sweep_span).
__device__ __forceinline__ void set_dense(const Params& P, PhaseRec& nx, uint32_t kind, uint32_t stamp) {
  if (nx.kind == kPhaseProcess && nx.fcount >= P.dense_min) {
    nx.dense = kind;
    nx.fstamp = stamp;
  }
}

// Every counter a delta manager step may read, loaded at once: independent
// volatile loads issue back to back, so the step costs about one L2 round
// trip instead of one per decision.
struct MgrSnap {
  uint32_t phases, probe_valid, local_q, local_total, local_iters, fusion_off, members, bucket_valid;
  uint32_t iterations, heavy_pulls, far_min, far_min_next;
  uint32_t hub[2], near[2], far[2], slot[kRing];
  unsigned long long member_heavy;
};
__device__ __forceinline__ MgrSnap snapshot(const Control* c) {
  MgrSnap m;
  m.phases = vld(&c->phases);
  m.probe_valid = vld(&c->probe_valid);
  m.local_q = vld(&c->local_q);
  m.local_total = vld(&c->local_total);
  m.local_iters = vld(&c->local_iters);
  m.fusion_off = vld(&c->fusion_off);
  m.members = vld(&c->members_count);
  m.bucket_valid = vld(&c->bucket_valid);
  m.iterations = vld(&c->iterations);
  m.heavy_pulls = vld(&c->heavy_pulls);
  m.far_min = vld(&c->far_min);
  m.far_min_next = vld(&c->far_min_next);
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    m.hub[i] = vld(&c->hub_count[i]);
    m.near[i] = vld(&c->near_count[i]);
    m.far[i] = vld(&c->far_count[i]);
  }
#pragma unroll
  for (int s = 0; s < kRing; ++s) m.slot[s] = vld(&c->slot_count[s]);
  m.member_heavy = vld64(&c->member_heavy);
  return m;
}

__device__ void manager_delta(const Params& P) {
  Control* c = P.ctl;
  const PhaseRec r = load_rec(c);
  MgrSnap m = snapshot(c);
  trace_phase(P, r, r.cur);
  PhaseRec nx = r;
  nx.dense = kDenseOff;
  nx.fstamp = 0u;
  nx.phase = r.phase + 1;
  nx.stamp = P.phase_base + (c->stamp_ctr++);
  c->phases = m.phases + 1;
  if (r.kind == kPhaseFinal) { nx.kind = kPhaseDone; store_rec(c, nx); return; }
  if (over_budget(P, nx)) return;
  if (r.kind == kPhaseProbe) {
    c->converged = m.probe_valid ? 0u : 1u;
    nx.kind = kPhaseFinal;
    store_rec(c, nx);
    return;
  }
  uint32_t win = r.win;
  uint32_t far_sel = r.far_sel;
  uint32_t from_slot = 0;   // first window slot to look at
  if (r.kind == kPhaseSplit) {
    c->far_count[r.far_sel] = 0;
    m.far[r.far_sel] = 0;
    far_sel = r.far_sel ^ 1u;
    c->far_min = m.far_min_next;
    m.far_min = m.far_min_next;
    c->far_min_next = 0xFFFFFFFFu;
    from_slot = 0;
  } else {  // PROCESS (light or heavy) or LOCAL
    PhaseRec rr = r;
    if (r.kind == kPhaseLocal) {
      // the local loop consumed every frontier it ran; its last pushes sit in local_q
      rr.fq = kQNone;
      rr.hub_in_chunks = 0;
      rr.push_q = m.local_q;
      rr.heavy = 0;
      c->local_total = m.local_total + m.local_iters;
    }
    const PhaseRec& r = rr;
    consume_process_counters(c, r);
    // the same consumption in the snapshot
    if (r.fq == kQNear0 || r.fq == kQNear1) m.near[r.fq] = 0;
    else if (r.fq == kQMembers) m.members = 0;
    else if (r.fq >= kQSlot0 && r.fq < kQSlot0 + kRing) m.slot[r.fq - kQSlot0] = 0;
    if (r.hub_in_chunks) m.hub[r.hub_in & 1] = 0u;
    const uint32_t hch = m.hub[r.hub_out & 1];
    const uint32_t nn = m.near[r.push_q & 1];
    nx.hub_in = r.hub_out;
    nx.hub_in_count = hch;
    nx.hub_in_chunks = hch;
    nx.hub_out = r.hub_out ^ 1u;
    if (r.heavy) {
      if (hch > 0) {             // heavy hub chunks first; near pushes keep accumulating
        nx.fq = kQNone;
        nx.fcount = 0;
        nx.stamp = r.stamp;
        store_rec(c, nx);
        return;
      }
      if (nn > 0) {              // a heavy relaxation landed in this bucket: new light round
        nx.kind = kPhaseProcess;
        nx.heavy = 0;
        nx.fq = r.push_q;
        nx.fcount = nn;
        nx.push_q = r.push_q ^ 1u;
        nx.hround = P.phase_base + nx.phase;
        set_dense(P, nx, kDenseNear, r.stamp);
        store_rec(c, nx);
        return;
      }
    } else {
      if (nn > 0 || hch > 0) {
        nx.kind = kPhaseProcess;
        nx.fq = nn ? r.push_q : kQNone;
        nx.fcount = nn;
        nx.push_q = r.push_q ^ 1u;
        if (hch == 0 && nn <= P.fusion && !m.fusion_off) nx.kind = kPhaseLocal;
        // (a LOCAL phase's last pushes carry a stamp drawn inside it: no sweep after one)
        if (nn > 0 && r.kind != kPhaseLocal) set_dense(P, nx, kDenseNear, r.stamp);
        store_rec(c, nx);
        return;
      }
      const uint32_t mc = m.members;
      if (mc > 0) {              // light rounds of this bucket are done: heavy pass
        nx.heavy = 1;
        c->member_heavy = 0;     // a later heavy pass of this bucket counts only its own members
        if (P.in_rowptr && (double)m.member_heavy > (double)P.pull_factor * (double)P.n) {
          // push would relax more heavy edges than a pull over every vertex costs
          c->members_count = 0;
          c->heavy_pulls = m.heavy_pulls + 1;
          nx.kind = kPhasePull;
          nx.fq = kQNone;
          nx.fcount = P.n;
          nx.hub_in_chunks = 0;
          nx.hub_in_count = 0;
        } else {
          nx.kind = kPhaseProcess;
          nx.fq = kQMembers;
          nx.fcount = mc;
        }
        store_rec(c, nx);
        return;
      }
    }
    // bucket r.cur is settled
    c->cur_min_key = 0xFFFFFFFFu;
    c->member_heavy = 0;
    if (m.bucket_valid) {
      m.iterations += 1;
      c->iterations = m.iterations;
      c->bucket_valid = 0;
      // the previous bucket had a successor (the reference's `changed`,
      // delta_stepping_hip_CSR.cpp:744-756); the last one is reported at the end
      if (m.iterations > 1) publish_progress(P.board, m.iterations - 1, 1u, globaltimer_ns() - c->t_start);
    }
    if (m.iterations >= P.max_iters) {
      nx.kind = kPhaseProbe;
      nx.heavy = 0;
      nx.hub_in_chunks = 0;
      store_rec(c, nx);
      return;
    }
    from_slot = r.cur - r.win + 1;
  }
  // next non-empty window slot
  int found = -1;
  for (int s = (int)from_slot; s < kRing; ++s) {
    if (m.slot[s]) { found = s; break; }
  }
  nx.heavy = 0;
  nx.hround = P.phase_base + nx.phase;
  nx.far_sel = far_sel;
  nx.hub_in = r.hub_out;
  nx.hub_in_count = 0;
  nx.hub_in_chunks = 0;
  nx.hub_out = r.hub_out ^ 1u;
  if (found >= 0) {
    nx.kind = kPhaseProcess;
    nx.win = win;
    nx.cur = win + (uint32_t)found;
    nx.fq = kQSlot0 + (uint32_t)found;
    nx.fcount = m.slot[found];
    nx.push_q = kQNear0;   // both near queues are empty at a bucket boundary
    if (nx.fcount <= P.fusion && !m.fusion_off) nx.kind = kPhaseLocal;
    set_dense(P, nx, kDenseSlot, nx.cur);
    store_rec(c, nx);
    return;
  }
  const uint32_t fc = m.far[far_sel];
  if (fc > 0) {
    // the next aligned window holding the smallest far bucket
    const uint32_t fmin_b = m.far_min;
    uint32_t nwin = win + kRing;
    const uint32_t aligned = (fmin_b / kRing) * kRing;
    if (fmin_b != 0xFFFFFFFFu && aligned > nwin) nwin = aligned;
    nx.kind = kPhaseSplit;
    nx.fq = kQFar0 + far_sel;
    nx.fcount = fc;
    nx.win = nwin;
    nx.cur = nwin;
    c->far_min_next = 0xFFFFFFFFu;
    store_rec(c, nx);
    return;
  }
  c->converged = 1;
  nx.kind = kPhaseFinal;
  store_rec(c, nx);
}

// Bucket fusion: block 0 alone runs consecutive light sub-phases of one
// bucket while the frontier stays at or under P.fusion, separated by block
// barriers instead of grid barriers; every other block waits at the next grid
// barrier.  Same relaxation code, same dedup stamps (drawn from the shared
// stamp counter), no hub splitting.  Exits when the frontier empties or grows
// past the threshold; the manager continues from local_q.  A sub-phase that
// scans more than kLocalEdgesPerVertex * P.fusion edges ends the loop and
// turns fusion off for the rest of the solve: on graphs whose small frontiers
// carry many edges one block is slower than the whole grid.
constexpr uint32_t kMaxLocalIters = 1u << 16;
constexpr uint32_t kLocalEdgesPerVertex = 8;

template <class W, bool PRED, int MODE>
__device__ void local_phase(const Params& P, const PhaseRec& R0, Tally& t) {
  __shared__ uint32_t s_l[5];
  __shared__ unsigned long long s_edges;
  Control* c = P.ctl;
  PhaseRec L = R0;
  const uint32_t w = threadIdx.x >> 5;
  const uint32_t nw = blockDim.x >> 5;
  const unsigned long long edge_cap = (unsigned long long)P.fusion * kLocalEdgesPerVertex;
  if (threadIdx.x == 0) s_edges = 0;
  __syncthreads();
  for (uint32_t iter = 0;; ++iter) {
    const unsigned long long e0 = t.edges;
    const uint32_t nfc = (L.fcount + 31) / 32;
    for (uint32_t ch = w; ch < nfc; ch += nw) frontier_chunk<W, PRED, MODE>(P, L, ch * 32, t);
    flush_all<MODE>(P, L, t.q, true);
    {
      unsigned long long de = t.edges - e0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) de += __shfl_down_sync(0xffffffffu, de, o);
      if ((threadIdx.x & 31u) == 0 && de) atomicAdd(&s_edges, de);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      consume_queue(c, L.fq);
      const uint32_t nn = ldcg(&c->near_count[L.push_q & 1]);
      const bool budget = globaltimer_ns() - c->t_start > P.budget_ns;
      if (budget) atomicCAS(&c->error, kErrNone, (uint32_t)kErrTimeout);
      const bool heavy_edges = s_edges > edge_cap;
      s_edges = 0;
      if (heavy_edges) c->fusion_off = 1u;
      uint32_t done =
          (nn == 0 || nn > P.fusion || iter + 1 >= kMaxLocalIters || budget || heavy_edges) ? 1u : 0u;
      if (!done) {
        s_l[0] = L.push_q;
        s_l[1] = nn;
        s_l[2] = L.push_q ^ 1u;
        s_l[3] = P.phase_base + (c->stamp_ctr++);
      }
      s_l[4] = done;
      c->local_q = L.push_q;
      c->local_iters = iter + 1;
    }
    __syncthreads();
    if (s_l[4]) break;
    L.fq = s_l[0];
    L.fcount = s_l[1];
    L.push_q = s_l[2];
    L.stamp = s_l[3];
  }
}

// ---------------------------------------------------------------------------
template <class W, bool PRED, int MODE>
__global__ void __launch_bounds__(kThreads, B2_SSSP_MINB) k_sssp(Params P) {
  using L = Label<PRED>;
  __shared__ PhaseRec s_rec;
  extern __shared__ uint32_t s_stage[];   // kStageWords per warp
  Tally t;
  t.keep = l2_keep_policy();
  {
    uint32_t* wb = s_stage + (threadIdx.x >> 5) * kStageWords;
    t.q.nearb = wb;
    t.q.farb = wb + kNearBuf;
    t.q.slotb = wb + kNearBuf + kFarBuf;
    t.q.memb = wb + kNearBuf + kFarBuf + 2 * kSlotBuf;
    t.q.listb = t.q.memb + kMemBuf;
  }
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  Control* c = P.ctl;

  // INIT: all labels unreached; delta bucket stamps / far flags cleared.
  for (size_t v = tid; v < P.n; v += stride) {
    ((typename L::T*)P.dist)[v] = L::kInf;
    if (MODE == kModeBF) ((typename L::T*)P.dist_cur)[v] = L::kInf;
    if (MODE == kModeDelta) {
      P.bstamp[v] = 0xFFFFFFFFu;
      P.farflag[v] = 0u;
    }
  }
  bool ok = grid_barrier((GridBarrier*)c, gridDim.x, P.budget_ns, [&] { manager_init<PRED, MODE>(P); });
  while (ok) {
    if (threadIdx.x == 0) s_rec = load_rec(c);
    __syncthreads();
    PhaseRec R = s_rec;
    if (R.kind == kPhaseDone) break;
    R.fcount = min(R.fcount, P.qcap);
    if (R.kind == kPhaseProcess) {
      process_phase<W, PRED, MODE>(P, R, t);
    } else if (R.kind == kPhaseLocal) {
      if (MODE == kModeDelta && blockIdx.x == 0) local_phase<W, PRED, MODE>(P, R, t);
    } else if (R.kind == kPhasePull) {
      if (MODE == kModeDelta) pull_phase<W, PRED>(P, R, t);
    } else if (R.kind == kPhaseCommit) {
      const uint32_t* F = queue_ptr(P, R.fq);
      for (size_t i = tid; i < R.fcount; i += stride) {
        const uint32_t v = ldcg(F + i);
        ((typename L::T*)P.dist_cur)[v] = ldcg((const typename L::T*)P.dist + v);
      }
    } else if (R.kind == kPhaseSplit) {
      const uint32_t* F = queue_ptr(P, R.fq);
      uint32_t kmin = 0xFFFFFFFFu;
      for (size_t base = tid - lane_id(); base < R.fcount; base += stride) {
        const size_t i = base + lane_id();
        int cls = 0;
        uint32_t v = 0, b = 0;
        uint32_t k = 0xFFFFFFFFu;
        if (i < R.fcount) {
          v = ldcg(F + i);
          k = L::key(ldcg((const typename L::T*)P.dist + v));
          b = bucket_of<W>(R, k);
          if (b < R.win) { cls = 0; P.farflag[v] = 0u; }
          else if (b < R.win + (uint32_t)kRing) { cls = 2; P.farflag[v] = 0u; P.bstamp[v] = b; }
          else { cls = 3; kmin = min(kmin, b); P.bstamp[v] = b; }
        }
        if (cls == 2) {
          const uint32_t s = b - R.win;
          const uint32_t grp = __match_any_sync(__activemask(), s);
          const uint32_t leader = __ffs(grp) - 1;
          uint32_t bs = 0;
          if (lane_id() == leader) bs = atomicAdd(&c->slot_count[s], (uint32_t)__popc(grp));
          bs = __shfl_sync(grp, bs, leader);
          const uint32_t pos = bs + __popc(grp & ((1u << lane_id()) - 1u));
          if (pos < P.qcap) queue_ptr(P, kQSlot0 + s)[pos] = v;
          else set_error(P, kErrQueueOverflow, 30);
        }
        const uint32_t pos = warp_append(&c->far_count[R.far_sel ^ 1u], cls == 3);
        if (cls == 3) {
          if (pos < P.qcap) queue_ptr(P, kQFar0 + (R.far_sel ^ 1u))[pos] = v;
          else set_error(P, kErrQueueOverflow, 31);
        }
      }
      kmin = __reduce_min_sync(0xffffffffu, kmin);
      if (lane_id() == 0 && kmin != 0xFFFFFFFFu) atomicMin(&c->far_min_next, kmin);
    } else if (R.kind == kPhaseProbe) {
      bool any = false;
      const uint32_t first = R.cur - R.win + 1;
      for (uint32_t s = first; s < (uint32_t)kRing && !any; ++s) {
        const uint32_t cnt = min(ldcg(&c->slot_count[s]), P.qcap);
        const uint32_t* F = queue_ptr(P, kQSlot0 + s);
        for (size_t i = tid; i < cnt; i += stride) {
          const uint32_t v = ldcg(F + i);
          const uint32_t k = L::key(ldcg((const typename L::T*)P.dist + v));
          if (k != kInfKey && bucket_of<W>(R, k) == R.win + s) { any = true; break; }
        }
      }
      {
        const uint32_t cnt = min(ldcg(&c->far_count[R.far_sel]), P.qcap);
        const uint32_t* F = queue_ptr(P, kQFar0 + R.far_sel);
        for (size_t i = tid; i < cnt && !any; i += stride) {
          const uint32_t v = ldcg(F + i);
          const uint32_t k = L::key(ldcg((const typename L::T*)P.dist + v));
          if (k != kInfKey && bucket_of<W>(R, k) >= R.win + (uint32_t)kRing) any = true;
        }
      }
      if (any) c->probe_valid = 1u;
    } else if (R.kind == kPhaseFinal) {
      const typename L::T* srcl =
          (const typename L::T*)((MODE == kModeBF && R.aux == 1u) ? P.dist_cur : P.dist);
      // in output order: a degree-ordered graph gathers each slot's label
      // (mostly L2-resident) instead of scattering 4-byte writes
      for (size_t o = tid; o < P.n; o += stride) {
        const size_t v = P.inv ? (size_t)__ldg(P.inv + o) : o;   // internal id of output slot o
        const typename L::T wv = ldcg(srcl + v);
        const uint32_t k = L::key(wv);
        if (W::kFloat) {
          ((float*)P.out_dist)[o] = (k == kInfKey) ? __uint_as_float(0x7f800000u) : key_to_f32(k);
        } else if (!P.dist_is_out || (const void*)srcl != P.out_dist) {
          ((uint32_t*)P.out_dist)[o] = k;
        }
        if (PRED && P.out_pred) {
          int32_t pr = -1;
          if (k != kInfKey && v != P.source) {
            const uint32_t pv = (uint32_t)(wv & 0xFFFFFFFFull);
            pr = (int32_t)(P.perm ? __ldg(P.perm + pv) : pv);
          }
          P.out_pred[o] = pr;
        }
      }
    }
    if (MODE == kModeBF) {
      ok = grid_barrier((GridBarrier*)c, gridDim.x, P.budget_ns, [&] { c->work_next = 0; manager_bf(P); });
    } else {
      ok = grid_barrier((GridBarrier*)c, gridDim.x, P.budget_ns, [&] { c->work_next = 0; manager_delta(P); });
    }
  }
  // flush tallies (one atomic per warp)
  unsigned long long e = t.edges, im = t.impr, pu = t.pushes;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
    pu += __shfl_down_sync(0xffffffffu, pu, o);
  }
  if (lane_id() == 0) {
    if (e) atomicAdd(&c->edges, e);
    if (im) atomicAdd(&c->improvements, im);
    if (pu) atomicAdd(&c->pushes, pu);
  }
}

// Light prefix length of every row for one delta (rows sorted by weight):
// the number of edges with weight <= delta, by binary search.
__global__ void k_light_count(uint32_t n, const uint64_t* __restrict__ rowptr, const uint2* __restrict__ edges,
                              int is_float, uint32_t delta_u, float delta_f, uint32_t* out) {
  for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x) {
    uint64_t lo = rowptr[v], hi = rowptr[v + 1];
    const uint64_t b = lo;
    while (lo < hi) {   // first edge with weight > delta
      const uint64_t mid = (lo + hi) >> 1;
      const uint32_t w = edges[mid].y;
      const bool light = is_float ? (__uint_as_float(w) <= delta_f) : (w <= delta_u);
      if (light) lo = mid + 1; else hi = mid;
    }
    out[v] = (uint32_t)min(lo - b, (uint64_t)0xFFFFFFFFull);
  }
}

// Reached vertices and their out-edges (the TEPS numerator).
template <bool PRED>
__global__ void k_reach(uint32_t n, const uint64_t* rowptr, const void* labels, int is_float,
                        unsigned long long* out) {
  unsigned long long r = 0, re = 0;
  for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x) {
    bool reached;
    if (PRED) reached = (((const unsigned long long*)labels)[v] >> 32) != 0xFFFFFFFFull;
    else if (is_float) reached = isfinite(((const float*)labels)[v]);
    else reached = ((const uint32_t*)labels)[v] != 0xFFFFFFFFu;
    if (reached) { ++r; re += rowptr[v + 1] - rowptr[v]; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    r += __shfl_down_sync(0xffffffffu, r, o);
    re += __shfl_down_sync(0xffffffffu, re, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(&out[0], r); atomicAdd(&out[1], re); }
}

// ---------------------------------------------------------------------------
// host side
// Co-resident grid of one kernel instance on the current device.  The
// shared-memory attribute and the occupancy are per-device facts, so both are
// settled once per (instance, device).
constexpr int kMaxDevices = 64;
template <class W, bool PRED, int MODE>
int max_grid() {
  static std::mutex mu;
  static int cached[kMaxDevices] = {};
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
  std::lock_guard<std::mutex> lock(mu);
  if (cached[dev]) return cached[dev];
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaFuncSetAttribute(k_sssp<W, PRED, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageBytes) !=
      cudaSuccess)
    return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sssp<W, PRED, MODE>, kThreads, kStageBytes);
  if (per < 1) per = 1;
  cached[dev] = per * sms;
  return cached[dev];
}

template <class W, bool PRED, int MODE>
cudaError_t launch(const Params& P, int grid, cudaStream_t st) {
  Params copy = P;
  void* args[] = {&copy};
  return cudaLaunchCooperativeKernel((void*)k_sssp<W, PRED, MODE>, dim3(grid), dim3(kThreads), args, kStageBytes,
                                     st);
}

b2_status map_device_error(uint32_t e) {
  switch (e) {
    case kErrNone: return B2_SUCCESS;
    case kErrTimeout: return B2_TIMEOUT;
    case kErrQueueOverflow: return B2_POOL_EXHAUSTED;
    default: return B2_DEVICE_ERROR;
  }
}

b2_status ensure_light_counts(b2_graph g, bool isf, uint32_t delta_u, float delta_f, cudaStream_t st) {
  Workspace& w = g->ws;
  uint32_t key;
  memcpy(&key, &delta_f, 4);
  if (!isf) key = delta_u;
  if (w.light_key_valid && w.light_key == key) return B2_SUCCESS;
  k_light_count<<<1184, 256, 0, st>>>((uint32_t)g->n, g->rowptr, g->edges, isf ? 1 : 0, delta_u, delta_f,
                                      w.lightcnt);
  B2_CUDA_TRY(cudaGetLastError());
  w.light_key = key;
  w.light_key_valid = 1;
  return B2_SUCCESS;
}

// The same light prefix for the incoming rows (pull heavy pass).
b2_status ensure_in_light_counts(b2_graph g, bool isf, uint32_t delta_u, float delta_f, cudaStream_t st) {
  Workspace& w = g->ws;
  uint32_t key;
  memcpy(&key, &delta_f, 4);
  if (!isf) key = delta_u;
  if (w.in_light_key_valid && w.in_light_key == key) return B2_SUCCESS;
  k_light_count<<<1184, 256, 0, st>>>((uint32_t)g->n, g->in_rowptr, g->in_edges, isf ? 1 : 0, delta_u, delta_f,
                                      w.in_lightcnt);
  B2_CUDA_TRY(cudaGetLastError());
  w.in_light_key = key;
  w.in_light_key_valid = 1;
  return B2_SUCCESS;
}

b2_status progress_begin(b2_graph g, const b2_sssp_opts& o, ProgressBoard** board_d) {
  *board_d = nullptr;
  if (!o.progress) return B2_SUCCESS;
  Workspace& w = g->ws;
  if (!w.board_h) {
    B2_CUDA_TRY(cudaHostAlloc((void**)&w.board_h, sizeof(ProgressBoard), cudaHostAllocMapped));
    cudaError_t e = cudaHostGetDevicePointer((void**)&w.board_d, w.board_h, 0);
    if (e != cudaSuccess) {
      cudaFreeHost(w.board_h);
      w.board_h = nullptr;
      return from_cuda(e);
    }
  }
  *(volatile uint32_t*)&w.board_h->rounds = 0;
  *(volatile uint32_t*)&w.board_h->changed = 0;
  *(volatile unsigned long long*)&w.board_h->t_ns = 0;
  *board_d = w.board_d;
  return B2_SUCCESS;
}

namespace {
void report_upto(const b2_sssp_opts& o, int32_t max_iters, uint32_t upto, uint32_t last_changed, double ms,
                 uint32_t* reported) {
  while (*reported < upto) {
    ++*reported;
    b2_progress p;
    p.iteration = (int32_t)*reported;
    p.max_iters = max_iters;
    p.changed = (*reported < upto) ? 1 : (int32_t)last_changed;   // every round before the last one changed
    p.reserved = 0;
    p.elapsed_ms = ms;
    o.progress(&p, o.progress_user);
  }
}
}  // namespace

void progress_poll(b2_graph g, const b2_sssp_opts& o, cudaEvent_t done, int32_t max_iters, uint32_t* reported) {
  const volatile ProgressBoard* b = g->ws.board_h;
  for (;;) {
    const cudaError_t q = cudaEventQuery(done);
    const uint32_t r = b->rounds;
    std::atomic_thread_fence(std::memory_order_acquire);
    if (r > *reported) report_upto(o, max_iters, r, b->changed, (double)b->t_ns * 1e-6, reported);
    if (q != cudaErrorNotReady) return;
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

void progress_finish(b2_graph g, const b2_sssp_opts& o, int32_t max_iters, uint32_t final_rounds, int32_t last_changed,
                     uint32_t* reported) {
  const volatile ProgressBoard* b = g->ws.board_h;
  report_upto(o, max_iters, final_rounds, (uint32_t)last_changed, (double)b->t_ns * 1e-6, reported);
}

b2_status run_sssp(b2_graph g, int mode, uint32_t source, void* d_dist, int32_t* d_pred,
                   const b2_sssp_opts* o_in, cudaStream_t st, b2_stats* stats) {
  if (!g || !d_dist) return B2_INVALID_ARGUMENT;
  if ((int64_t)source >= g->n) return B2_INVALID_ARGUMENT;
  b2_sssp_opts o;
  if (o_in) o = *o_in; else b2_sssp_opts_default(&o);
  if (o.keep_distances) return B2_NOT_SUPPORTED;   // warm start: ADDS only
  if (mode == kModeDelta && g->has_negative) return B2_INVALID_WEIGHT;
  const bool isf = g->weight_type == B2_W_F32;
  const bool pred = d_pred != nullptr;
  uint32_t policy_used = 0;
  if (mode == kModeDelta && o.policy == 1) {
    // learned schedule (computes and caches the graph's features on first use,
    // which runs solves of its own: before this solve takes the handle lock)
    double mult = 1.0;
    uint32_t fuse = 0;
    float pull = 8.0f;
    const b2_status ps = policy_decide(g, &mult, &fuse, &pull);
    if (ps == B2_SUCCESS) {
      double nf = 1.0;
      b2_delta_heuristic(g, o.delta_scale > 0 ? o.delta_scale : 16.0, &nf);
      o.delta = nf * mult;
      if (o.fusion_threshold == 0) o.fusion_threshold = fuse;
      o.light_heavy = 1;
      o.pull_fraction = pull;   // the predicted push/pull switch point (0: push only)
      policy_used = 1;
    } else if (ps != B2_NOT_SUPPORTED) {
      return ps;
    }
  }
  std::lock_guard<std::mutex> lock(g->mu);
  b2_status s = ensure_workspace(g, pred);
  if (s != B2_SUCCESS) return s;
  Workspace& w = g->ws;

  Params P;
  memset(&P, 0, sizeof(P));
  P.n = (uint32_t)g->n;
  P.qcap = (o.worklist_capacity > 0 && (int64_t)o.worklist_capacity < g->n) ? o.worklist_capacity : P.n;
  P.source = internal_id(g, source);
  P.perm = g->perm;
  P.inv = g->perm ? g->inv : nullptr;
  P.rowptr = g->rowptr;
  P.edges = g->edges;
  P.pstamp = w.pstamp;
  P.bstamp = w.bstamp;
  P.farflag = w.farflag;
  P.hstamp = w.hstamp;
  P.queues = w.queues;
  P.hubs = w.hubs;
  P.hub_cap = (uint32_t)w.hub_cap;
  P.ctl = w.ctl;
  P.trace = o.trace ? w.trace : nullptr;
  P.hub_degree = std::max<uint32_t>(32u, o.hub_degree ? o.hub_degree : 256u);
  P.out_dist = d_dist;
  P.out_pred = d_pred;
  P.is_float = isf ? 1u : 0u;
  P.budget_ns = (unsigned long long)(std::max(0.001, o.timeout_ms > 0 ? o.timeout_ms : 20000.0) * 1.0e6);
  if (pred || g->perm) {   // labels in the workspace (degree order: outputs are scattered back)
    P.dist = w.dist_a;
    P.dist_cur = w.dist_b;
    P.dist_is_out = 0;
  } else {
    P.dist = d_dist;        // keys are built in the caller's buffer, converted in place
    P.dist_cur = w.dist_b;
    P.dist_is_out = 1;
  }
  double delta = 1.0;
  if (mode == kModeBF) {
    int64_t mi = o.max_iters < 0 ? g->n - 1 : o.max_iters;
    if (mi > 0x7fffffff) mi = 0x7fffffff;
    P.max_iters = (uint32_t)mi;
    P.detect_negcycle = o.detect_negative_cycle ? 1u : 0u;
    P.inv_delta = 1.0f;
    P.delta_u = 1u;
  } else {
    delta = o.delta;
    if (!(delta > 0.0)) b2_delta_heuristic(g, o.delta_scale > 0 ? o.delta_scale : 16.0, &delta);
    float df = 0.0f;
    if (isf) {
      df = (float)delta;
      if (!(df > 0.0f) || !std::isfinite(df)) return B2_INVALID_ARGUMENT;
      P.inv_delta = 1.0f / df;
      P.delta_u = 1u;
    } else {
      const double dd = std::max(1.0, std::floor(delta));
      P.delta_u = (uint32_t)std::min(dd, 4294967295.0);
      P.inv_delta = 0.0f;
      delta = (double)P.delta_u;
    }
    P.max_iters = o.max_iters < 0 ? 0xFFFFFFFFu : (uint32_t)o.max_iters;
    P.fusion = o.fusion_threshold;
    // stamp sweeps pay on low-degree graphs; on skewed ones the vertex order
    // bunches heavy rows into the same sweep items (a long tail per phase)
    const float dfrac = o.dense_fraction != 0.0f ? o.dense_fraction : (g->max_degree <= 64 ? 1.0f / 16.0f : -1.0f);
    P.dense_min = dfrac > 0.0f ? (uint32_t)std::min(4294967295.0, std::max(1.0, std::ceil((double)dfrac * g->n)))
                               : 0xFFFFFFFFu;
    if (o.light_heavy && g->rows_sorted) {
      s = ensure_light_counts(g, isf, P.delta_u, df, st);
      if (s != B2_SUCCESS) return s;
      P.lightcnt = w.lightcnt;
      // push/pull switch of the heavy pass: only graphs dense enough for a pull to pay off
      if (o.pull_fraction > 0.0f && (double)g->m >= (double)o.pull_fraction * (double)g->n) {
        s = ensure_incoming(g, st);
        if (s == B2_SUCCESS) s = ensure_in_light_counts(g, isf, P.delta_u, df, st);
        if (s != B2_SUCCESS) return s;
        P.in_rowptr = g->in_rowptr;
        P.in_edges = g->in_edges;
        P.in_lightcnt = w.in_lightcnt;
        P.pull_factor = o.pull_fraction;
      }
    }
  }
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->delta_used = delta;
    stats->policy_used = policy_used;
  }
  // zero iterations: only the source is reached (the reference loop never runs)
  if (P.max_iters == 0) {
    if (isf) {
      std::vector<float> h((size_t)g->n, INFINITY);
      h[source] = 0.0f;
      B2_CUDA_TRY(cudaMemcpyAsync(d_dist, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st));
      B2_CUDA_TRY(cudaStreamSynchronize(st));
    } else {
      std::vector<uint32_t> h((size_t)g->n, 0xFFFFFFFFu);
      h[source] = 0u;
      B2_CUDA_TRY(cudaMemcpyAsync(d_dist, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st));
      B2_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (pred) B2_CUDA_TRY(cudaMemsetAsync(d_pred, 0xFF, (size_t)g->n * 4, st));
    B2_CUDA_TRY(cudaStreamSynchronize(st));
    return B2_SUCCESS;
  }
  // phase stamps never repeat across solves on this workspace
  if (w.phase_epoch > 0xF0000000u) {
    B2_CUDA_TRY(cudaMemsetAsync(w.pstamp, 0, (size_t)g->n * 4, st));
    B2_CUDA_TRY(cudaMemsetAsync(w.hstamp, 0, (size_t)g->n * 4, st));
    w.phase_epoch = 1;
  }
  P.phase_base = w.phase_epoch;

  s = progress_begin(g, o, &P.board);
  if (s != B2_SUCCESS) return s;
  int grid = 0;
  cudaError_t e = cudaSuccess;
  B2_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(Control), st));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  // small graphs: about one thread per vertex (every grid barrier costs an
  // arrival per block, and a graph of a few thousand vertices cannot use more)
  const int small_grid = (int)std::max<int64_t>(1, (g->n + kThreads - 1) / kThreads);
#define B2_LAUNCH(WT, PR, MD)                                              \
  do {                                                                     \
    grid = max_grid<WT, PR, MD>();                                         \
    if (o.grid_blocks && (int)o.grid_blocks < grid) grid = o.grid_blocks;  \
    else if (!o.grid_blocks && small_grid < grid) grid = small_grid;       \
    e = grid > 0 ? launch<WT, PR, MD>(P, grid, st) : cudaErrorInvalidConfiguration; \
  } while (0)
  if (mode == kModeBF) {
    if (isf) { if (pred) B2_LAUNCH(WF32, true, kModeBF); else B2_LAUNCH(WF32, false, kModeBF); }
    else { if (pred) B2_LAUNCH(WU32, true, kModeBF); else B2_LAUNCH(WU32, false, kModeBF); }
  } else {
    if (isf) { if (pred) B2_LAUNCH(WF32, true, kModeDelta); else B2_LAUNCH(WF32, false, kModeDelta); }
    else { if (pred) B2_LAUNCH(WU32, true, kModeDelta); else B2_LAUNCH(WU32, false, kModeDelta); }
  }
#undef B2_LAUNCH
  cudaEventRecord(e1, st);
  if (e != cudaSuccess) { cudaEventDestroy(e0); cudaEventDestroy(e1); return from_cuda(e); }
  const int32_t prog_max = mode == kModeBF ? (int32_t)P.max_iters : (o.max_iters < 0 ? -1 : o.max_iters);
  uint32_t reported = 0;
  if (P.board) progress_poll(g, o, e1, prog_max, &reported);
  e = cudaMemcpyAsync(w.h_ctl, w.ctl, sizeof(Control), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return from_cuda(e);
  const Control& hc = *w.h_ctl;
  if (P.board) progress_finish(g, o, prog_max, hc.iterations, hc.converged ? 0 : 1, &reported);
  w.phase_epoch += std::max(hc.rec.phase, hc.stamp_ctr) + 2;
  w.trace_n = o.trace ? hc.trace_n : 0;
  b2_status ds = map_device_error(hc.error);
  if (stats) {
    stats->iterations_used = (int32_t)hc.iterations;
    stats->converged = (int32_t)hc.converged;
    stats->has_negative_cycle = (int32_t)hc.negative_cycle;
    stats->phases = (int32_t)hc.phases;
    stats->edges_scanned = hc.edges;
    stats->improvements = hc.improvements;
    stats->pushes = hc.pushes;
    stats->kernel_ms = ms;
    stats->device_error = hc.error;
    stats->device_error_site = hc.error_site;
    stats->grid_blocks = (uint32_t)grid;
    stats->first_unchanged = hc.first_unchanged;
    stats->local_subphases = hc.local_total;
    stats->delta_updates = hc.delta_updates;
    stats->heavy_pulls = hc.heavy_pulls;
    if (mode == kModeDelta) {
      float inv;
      memcpy(&inv, &hc.rec.dinv, 4);
      stats->delta_final = isf ? 1.0 / (double)inv : (double)hc.rec.dq;
    } else
      stats->delta_final = delta;
  }
  if (ds != B2_SUCCESS) return ds;
  if (stats && o.collect_reach) return collect_reach(g, (pred || g->perm) ? w.dist_a : d_dist, pred, isf, st, stats);
  return B2_SUCCESS;
}

b2_status collect_reach(b2_graph g, const void* lab, bool pred, bool isf, cudaStream_t st, b2_stats* stats) {
  unsigned long long* d_r = g->ws.reach;   // workspace counters: no allocation (a cudaFree would sync the device)
  B2_CUDA_TRY(cudaMemsetAsync(d_r, 0, 16, st));
  if (pred) k_reach<true><<<1024, 256, 0, st>>>((uint32_t)g->n, g->rowptr, lab, isf, d_r);
  else k_reach<false><<<1024, 256, 0, st>>>((uint32_t)g->n, g->rowptr, lab, isf, d_r);
  B2_CUDA_TRY(cudaGetLastError());
  unsigned long long hr[2] = {0, 0};
  B2_CUDA_TRY(cudaMemcpyAsync(hr, d_r, 16, cudaMemcpyDeviceToHost, st));
  B2_CUDA_TRY(cudaStreamSynchronize(st));
  stats->reached = hr[0];
  stats->reached_edges = hr[1];
  return B2_SUCCESS;
}

}  // namespace b2

using namespace b2;

extern "C" b2_status b2_sssp_bf(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred,
                                const b2_sssp_opts* opts, b2_stream stream, b2_stats* stats) {
  return run_sssp(g, kModeBF, source, d_dist, d_pred, opts, (cudaStream_t)stream, stats);
}

extern "C" b2_status b2_sssp_delta(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred,
                                   const b2_sssp_opts* opts, b2_stream stream, b2_stats* stats) {
  return run_sssp(g, kModeDelta, source, d_dist, d_pred, opts, (cudaStream_t)stream, stats);
}

// ADDS (adds_sssp_hip, Charlotte_oneshot/sssp_hip.cpp:428-595; hip_adds::sssp,
// jasper_oneshot_untested/hip_adds_sssp.cpp:1138-1301): the asynchronous
// worklist kernel of b2_adds.cu.
extern "C" b2_status b2_sssp_adds(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred,
                                  const b2_sssp_opts* opts, b2_stream stream, b2_stats* stats) {
  return run_adds(g, source, d_dist, d_pred, opts, (cudaStream_t)stream, stats);
}

extern "C" b2_status b2_graph_trace(b2_graph g, b2_trace_entry* entries, int32_t capacity, int32_t* count) {
  if (!g || !count || (capacity > 0 && !entries)) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g->mu);
  const int32_t n = (int32_t)std::min<uint32_t>(g->ws.trace_n, (uint32_t)std::max(capacity, 0));
  *count = n;
  if (n == 0 || !g->ws.trace) return B2_SUCCESS;
  static_assert(sizeof(TraceEntry) == sizeof(b2_trace_entry), "trace layout");
  B2_CUDA_TRY(cudaMemcpy(entries, g->ws.trace, (size_t)n * sizeof(TraceEntry), cudaMemcpyDeviceToHost));
  return B2_SUCCESS;
}
