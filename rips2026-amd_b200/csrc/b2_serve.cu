// Batched multi-query serving: one thread block solves one single-source
// query alone (delta-stepping with a near queue and a far pile, block
// barriers only), and a batch launch runs as many queries at once as the
// GPU holds blocks.  No reference counterpart (the reference answers one
// query per launch sequence).
//
// A query owns a slot of the server's device arena (no word is shared
// between queries):
//   labels  n x 4 B (8 B with predecessors: key << 32 | pred)
//   stamp   n x 4 B   near-queue dedup (phase stamp)
//   farflag n x 4 B   1 while the vertex sits in the far pile
//   qa, qb  n x 4 B   near queue ping-pong
//   fa, fb  n x 4 B   far pile ping-pong
// The block writes the distances (and predecessors) straight into the
// caller's buffer -- page-locked host memory, so the result is in host memory
// when the query's completion record flips, independently of the other
// queries of the batch -- or device memory.
// Distances equal the full-GPU solvers' (the label fixpoint does not depend
// on the relaxation order); with predecessors ties go to the smallest id.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <random>
#include <vector>

#include <cooperative_groups.h>

#include "b2_common.cuh"
#include "b2_internal.hpp"

namespace cg = cooperative_groups;

namespace b2 {

// Completion record of one query, in mapped page-locked host memory: the
// solving block fills the counters, fences, then publishes `flag`.
struct ServeRecord {
  uint32_t flag;        // 0 running, 1 done
  uint32_t status;      // 0 ok, kErrTimeout, kErrQueueOverflow
  uint32_t phases;
  uint32_t pad;
  unsigned long long edges_scanned;
  unsigned long long reached;
  unsigned long long reached_edges;
};

struct ServeQuery {
  const uint64_t* rowptr;
  const uint2* edges;
  uint32_t n;
  uint32_t source;
  uint32_t is_float;
  uint32_t pred;
  uint32_t delta_u;     // uint32 bucket width
  float inv_delta;      // float: bucket = floor(d * inv_delta)
  void* labels;
  uint32_t* stamp;
  uint32_t* farflag;
  uint32_t* qa;
  uint32_t* qb;
  uint32_t* fa;
  uint32_t* fb;
  uint32_t* out_dist;   // caller's buffer: device memory or mapped page-locked host memory
  int32_t* out_pred;    // nullable
  ServeRecord* rec;     // mapped page-locked host memory
  const uint32_t* perm; // degree-ordered graph: internal -> input id (else null); source is internal
};

namespace {

constexpr int kServeThreads = 512;
constexpr uint32_t kBlockHubDeg = 512;     // rows at least this long are relaxed by the whole block
constexpr uint32_t kHubListCap = 128;

template <bool PRED>
struct SLabel;
template <>
struct SLabel<false> {
  using T = uint32_t;
  __device__ static T inf() { return kInfKey; }
  __device__ static T make(uint32_t key, uint32_t) { return key; }
  __device__ static uint32_t key(T x) { return x; }
  __device__ static T atomic_min(T* a, T v) { return atomicMin(a, v); }
};
template <>
struct SLabel<true> {
  using T = unsigned long long;
  __device__ static T inf() { return ~0ull; }
  __device__ static T make(uint32_t key, uint32_t p) { return ((T)key << 32) | p; }
  __device__ static uint32_t key(T x) { return (uint32_t)(x >> 32); }
  __device__ static T atomic_min(T* a, T v) { return atomicMin(a, v); }
};

// Bucket of a label key; kSNone for unreached.  Buckets only order the work
// (any monotone map gives the same distances), so huge float distances are
// clamped into the last bucket.
constexpr uint32_t kSNone = 0xFFFFFFFFu;
template <class W>
__device__ __forceinline__ uint32_t sbucket(const ServeQuery& q, uint32_t key) {
  if (key == kInfKey) return kSNone;
  if (!W::kFloat) return key / q.delta_u;    // <= 0xFFFFFFFE
  const float b = floorf(key_to_f32(key) * q.inv_delta);
  return b >= 4294967040.0f ? 0xFFFFFFFEu : (uint32_t)b;
}

struct SShared {
  uint32_t ncount;     // current near frontier
  uint32_t next_count; // pushes into the next near queue
  uint32_t fcount;     // far pile entries
  uint32_t fnext;      // kept far entries during a split
  uint32_t cur;        // current bucket
  uint32_t minb;       // split: smallest live bucket
  uint32_t stop;
  uint32_t nhub;
  uint32_t hubs[kHubListCap];
  unsigned long long red[3];
};

// The team that solves one query: one thread block, or a cluster of
// kClusterCTAs blocks (co-scheduled by the hardware) that share the lead
// block's SShared through distributed shared memory and meet at cluster
// barriers.  Large graphs get a cluster, so a long query runs on several SMs.
constexpr uint32_t kClusterCTAs = 8;
struct TeamCTA {
  __device__ static uint32_t tid() { return threadIdx.x; }
  __device__ static uint32_t threads() { return kServeThreads; }
  __device__ static void sync() { __syncthreads(); }
  template <class T>
  __device__ static T* lead(T* p) { return p; }
};
struct TeamCluster {
  __device__ static uint32_t tid() { return cg::this_cluster().block_rank() * kServeThreads + threadIdx.x; }
  __device__ static uint32_t threads() { return kClusterCTAs * kServeThreads; }
  __device__ static void sync() { cg::this_cluster().sync(); }
  template <class T>
  __device__ static T* lead(T* p) { return cg::this_cluster().map_shared_rank(p, 0); }
};

// Relax kSU edges per lane (u's label key -> v): all edge loads are issued
// first, then all label loads, then the atomics, so one lane keeps kSU
// independent memory requests in flight; improved vertices go to the next
// near queue or the far pile (warp-aggregated appends).
constexpr int kSU = 4;

template <class W, bool PRED>
__device__ __forceinline__ void relax_edges(const ServeQuery& q, SShared& sh, const uint32_t (&ukey)[kSU],
                                            const uint32_t (&u)[kSU], const uint2 (&e)[kSU], const bool (&valid)[kSU],
                                            uint32_t next_stamp, uint32_t* qnext) {
  using L = SLabel<PRED>;
  typename L::T* lab = (typename L::T*)q.labels;
  uint32_t nd[kSU], cur[kSU];
#pragma unroll
  for (int k = 0; k < kSU; ++k) {
    nd[k] = valid[k] ? W::extend(ukey[k], e[k].y) : kInfKey;
    cur[k] = nd[k] != kInfKey ? L::key(__ldcg(lab + e[k].x)) : kInfKey;
  }
  bool imp[kSU];
#pragma unroll
  for (int k = 0; k < kSU; ++k) {
    imp[k] = false;
    // with predecessors an equal distance may still lower the predecessor id
    if (nd[k] != kInfKey && (PRED ? nd[k] <= cur[k] : nd[k] < cur[k])) {
      const typename L::T old = L::atomic_min(lab + e[k].x, L::make(nd[k], u[k]));
      imp[k] = nd[k] < L::key(old);
    }
  }
#pragma unroll
  for (int k = 0; k < kSU; ++k) {
    bool to_near = false, to_far = false;
    const uint32_t v = e[k].x;
    if (imp[k]) {
      if (sbucket<W>(q, nd[k]) <= sh.cur) to_near = atomicExch(q.stamp + v, next_stamp) != next_stamp;
      else to_far = atomicExch(q.farflag + v, 1u) == 0u;
    }
    const uint32_t pn = warp_append(&sh.next_count, to_near);
    if (to_near) qnext[pn] = v;
    const uint32_t pf = warp_append(&sh.fcount, to_far);
    if (to_far) q.fa[pf] = v;
  }
}

// One near phase: warps take 32-vertex chunks of the frontier and walk the
// chunk's edges lane-parallel; rows of kBlockHubDeg or more edges are
// collected and relaxed afterwards by the whole block.
template <class W, bool PRED, class Team>
__device__ void near_phase(const ServeQuery& q, SShared& sh, const uint32_t* qcur, uint32_t* qnext,
                           uint32_t next_stamp, unsigned long long& edges) {
  using L = SLabel<PRED>;
  const uint32_t lane = threadIdx.x & 31u, warp = Team::tid() >> 5;
  const uint32_t cnt = sh.ncount;
  typename L::T* lab = (typename L::T*)q.labels;
  for (uint32_t base = warp * 32; base < cnt; base += Team::threads()) {
    const uint32_t i = base + lane;
    uint32_t u = 0, ukey = kInfKey, deg = 0;
    uint64_t start = 0;
    if (i < cnt) {
      u = qcur[i];
      ukey = L::key(__ldcg(lab + u));
      start = __ldg(q.rowptr + u);
      const uint64_t d = __ldg(q.rowptr + u + 1) - start;
      if (d >= kBlockHubDeg) {
        const uint32_t slot = atomicAdd(&sh.nhub, 1u);
        if (slot < kHubListCap) sh.hubs[slot] = u;
        else deg = (uint32_t)d;            // hub list full: this warp walks the row
      } else {
        deg = (uint32_t)d;
      }
    }
    const uint32_t incl = warp_incl_scan(deg);
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t excl = incl - deg;
    for (uint32_t e0 = 0; e0 < total; e0 += 32 * kSU) {
      uint32_t okey[kSU], ou[kSU];
      uint2 ed[kSU];
      bool valid[kSU];
#pragma unroll
      for (int k = 0; k < kSU; ++k) {
        const uint32_t e = e0 + 32u * k + lane;
        // owner: first lane whose inclusive prefix exceeds e
        uint32_t lo = 0;
#pragma unroll
        for (uint32_t s = 16; s > 0; s >>= 1) {
          const uint32_t pv = __shfl_sync(0xffffffffu, incl, lo + s - 1);
          if (pv <= e) lo += s;
        }
        const uint32_t owner = lo > 31 ? 31 : lo;
        const uint32_t oex = __shfl_sync(0xffffffffu, excl, owner);
        const uint64_t ost = __shfl_sync(0xffffffffu, start, owner);
        okey[k] = __shfl_sync(0xffffffffu, ukey, owner);
        ou[k] = __shfl_sync(0xffffffffu, u, owner);
        valid[k] = e < total;
        ed[k] = valid[k] ? __ldcs(q.edges + ost + (e - oex)) : make_uint2(0, 0);
      }
      relax_edges<W, PRED>(q, sh, okey, ou, ed, valid, next_stamp, qnext);
    }
    edges += deg;
  }
  Team::sync();
  const uint32_t nh = min(sh.nhub, kHubListCap);
  for (uint32_t h = 0; h < nh; ++h) {
    const uint32_t u = sh.hubs[h];
    const uint32_t ukey = L::key(__ldcg(lab + u));
    const uint64_t start = __ldg(q.rowptr + u), end = __ldg(q.rowptr + u + 1);
    const uint64_t len = end - start;
    // every thread of the team runs the same number of iterations (warp_append needs whole warps)
    for (uint64_t k0 = 0; k0 < len; k0 += (uint64_t)Team::threads() * kSU) {
      uint32_t okey[kSU], ou[kSU];
      uint2 ed[kSU];
      bool valid[kSU];
#pragma unroll
      for (int j = 0; j < kSU; ++j) {
        const uint64_t k = k0 + (uint64_t)j * Team::threads() + Team::tid();
        valid[j] = k < len;
        okey[j] = ukey;
        ou[j] = u;
        ed[j] = valid[j] ? __ldcs(q.edges + start + k) : make_uint2(0, 0);
      }
      relax_edges<W, PRED>(q, sh, okey, ou, ed, valid, next_stamp, qnext);
    }
    if (Team::tid() == 0) edges += len;
  }
}

template <class W, bool PRED, class Team>
__device__ void team_solve(ServeQuery& q, SShared& sh, uint64_t t0, uint64_t budget_ns) {
  using L = SLabel<PRED>;
  typename L::T* lab = (typename L::T*)q.labels;
  const uint32_t n = q.n;
  for (uint32_t v = Team::tid(); v < n; v += Team::threads()) {
    lab[v] = L::inf();
    q.stamp[v] = 0u;
    q.farflag[v] = 0u;
  }
  Team::sync();
  if (Team::tid() == 0) {
    lab[q.source] = L::make(W::zero_key(), kNoPred);
    q.qa[0] = q.source;
    q.stamp[q.source] = 1u;
    sh.ncount = 1;
    sh.next_count = 0;
    sh.fcount = 0;
    sh.cur = sbucket<W>(q, W::zero_key());
    sh.stop = 0;
    sh.nhub = 0;
  }
  Team::sync();
  unsigned long long edges = 0;
  uint32_t phase = 1;
  uint32_t* qcur = q.qa;
  uint32_t* qnext = q.qb;
  uint32_t status = 0;
  for (;;) {
    // light phases of the current bucket
    while (sh.ncount > 0) {
      near_phase<W, PRED, Team>(q, sh, qcur, qnext, phase + 1, edges);
      Team::sync();
      ++phase;
      uint32_t* t = qcur;
      qcur = qnext;
      qnext = t;
      if (Team::tid() == 0) {
        sh.ncount = sh.next_count;
        sh.next_count = 0;
        sh.nhub = 0;
        if (globaltimer_ns() - t0 > budget_ns) sh.stop = kErrTimeout;
        if (phase >= 0xFFFFFFF0u) sh.stop = kErrQueueOverflow;   // stamp space exhausted
      }
      Team::sync();
      if (sh.stop) break;
    }
    if (sh.stop) { status = sh.stop; break; }
    if (sh.fcount == 0) break;
    // far split, pass 1: smallest live bucket above the current one
    if (Team::tid() == 0) sh.minb = kSNone;
    Team::sync();
    const uint32_t fc = sh.fcount, cur = sh.cur;
    uint32_t mb = kSNone;
    for (uint32_t i = Team::tid(); i < fc; i += Team::threads()) {
      const uint32_t b = sbucket<W>(q, L::key(__ldcg(lab + q.fa[i])));
      if (b > cur && b < mb) mb = b;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mb = min(mb, __shfl_xor_sync(0xffffffffu, mb, o));
    if ((threadIdx.x & 31u) == 0 && mb != kSNone) atomicMin(&sh.minb, mb);
    Team::sync();
    const uint32_t nb = sh.minb;
    if (nb == kSNone) break;                          // every far entry is settled
    if (Team::tid() == 0) { sh.cur = nb; sh.fnext = 0; sh.next_count = 0; }
    Team::sync();
    // pass 2: entries of bucket nb go to the near queue, later ones are kept
    const uint32_t st = phase + 1;
    for (uint32_t i0 = 0; i0 < fc; i0 += Team::threads()) {
      const uint32_t i = i0 + Team::tid();
      bool to_near = false, keep = false;
      uint32_t v = 0;
      if (i < fc) {
        v = q.fa[i];
        const uint32_t b = sbucket<W>(q, L::key(__ldcg(lab + v)));
        if (b <= cur) {
          q.farflag[v] = 0u;                          // reached the near queue earlier
        } else if (b <= nb) {
          q.farflag[v] = 0u;
          to_near = atomicExch(q.stamp + v, st) != st;
        } else {
          keep = true;
        }
      }
      const uint32_t pn = warp_append(&sh.next_count, to_near);
      if (to_near) qcur[pn] = v;
      const uint32_t pk = warp_append(&sh.fnext, keep);
      if (keep) q.fb[pk] = v;
    }
    Team::sync();
    ++phase;
    uint32_t* t = q.fa;
    q.fa = q.fb;
    q.fb = t;
    if (Team::tid() == 0) {
      sh.ncount = sh.next_count;
      sh.next_count = 0;
      sh.fcount = sh.fnext;
    }
    Team::sync();
  }
  // output into the caller's buffers, then the completion record
  unsigned long long reached = 0, redges = 0;
  for (uint32_t v = Team::tid(); v < n; v += Team::threads()) {
    const typename L::T x = __ldcg(lab + v);
    const uint32_t k = L::key(x);
    uint32_t out = k;
    if (W::kFloat) out = (k == kInfKey) ? 0x7f800000u : __float_as_uint(key_to_f32(k));
    const uint32_t o = q.perm ? __ldg(q.perm + v) : v;   // input id of internal vertex v
    q.out_dist[o] = out;
    if (PRED && q.out_pred) {
      const uint32_t pv = (uint32_t)(x & 0xFFFFFFFFull);
      q.out_pred[o] = (k == kInfKey || v == q.source) ? -1 : (int32_t)(q.perm ? __ldg(q.perm + pv) : pv);
    }
    if (k != kInfKey) {
      ++reached;
      redges += __ldg(q.rowptr + v + 1) - __ldg(q.rowptr + v);
    }
  }
  __threadfence_system();
  if (Team::tid() < 3) sh.red[Team::tid()] = 0;
  Team::sync();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    edges += __shfl_xor_sync(0xffffffffu, edges, o);
    reached += __shfl_xor_sync(0xffffffffu, reached, o);
    redges += __shfl_xor_sync(0xffffffffu, redges, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    atomicAdd(&sh.red[0], edges);
    atomicAdd(&sh.red[1], reached);
    atomicAdd(&sh.red[2], redges);
  }
  Team::sync();
  if (Team::tid() == 0) {
    ServeRecord* r = q.rec;
    r->status = status;
    r->phases = phase;
    r->edges_scanned = sh.red[0];
    r->reached = sh.red[1];
    r->reached_edges = sh.red[2];
    __threadfence_system();
    asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(&r->flag), "r"(1u) : "memory");
  }
}

// Teams take queries from the batch in order (one atomic per query) until
// the batch is exhausted.  Descriptors live in mapped page-locked host memory.
template <class Team>
__device__ __forceinline__ void serve_loop(const ServeQuery* qs, uint32_t nq, uint32_t* next,
                                           unsigned long long budget_ns, SShared* sh_mine, uint32_t* q_mine) {
  SShared& sh = *Team::lead(sh_mine);
  uint32_t* s_q = Team::lead(q_mine);
  for (;;) {
    if (Team::tid() == 0) *s_q = atomicAdd(next, 1u);
    Team::sync();
    const uint32_t qi = *s_q;
    Team::sync();
    if (qi >= nq) break;
    ServeQuery q = qs[qi];
    const uint64_t t0 = globaltimer_ns();
    if (q.is_float) {
      if (q.pred) team_solve<WF32, true, Team>(q, sh, t0, budget_ns);
      else team_solve<WF32, false, Team>(q, sh, t0, budget_ns);
    } else {
      if (q.pred) team_solve<WU32, true, Team>(q, sh, t0, budget_ns);
      else team_solve<WU32, false, Team>(q, sh, t0, budget_ns);
    }
    Team::sync();
  }
}

__global__ void __launch_bounds__(kServeThreads, 2)
    k_serve(const ServeQuery* qs, uint32_t nq, uint32_t* next, unsigned long long budget_ns) {
  __shared__ SShared sh;
  __shared__ uint32_t s_q;
  serve_loop<TeamCTA>(qs, nq, next, budget_ns, &sh, &s_q);
}

// One query per cluster of kClusterCTAs blocks (grid: a multiple of it).
__global__ void __cluster_dims__(kClusterCTAs, 1, 1) __launch_bounds__(kServeThreads, 2)
    k_serve_cluster(const ServeQuery* qs, uint32_t nq, uint32_t* next, unsigned long long budget_ns) {
  __shared__ SShared sh;
  __shared__ uint32_t s_q;
  serve_loop<TeamCluster>(qs, nq, next, budget_ns, &sh, &s_q);
}

}  // namespace
}  // namespace b2

// ===========================================================================
// Host engine: arena, admission, batch launches on a few streams, per-query
// completion, and the built-in Poisson load generator.
// ===========================================================================
namespace b2 {
namespace {

using Clock = std::chrono::steady_clock;
inline uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now().time_since_epoch()).count();
}

// First-fit range allocator with coalescing (offsets in bytes, 256-B units).
class RangeAlloc {
 public:
  void reset(size_t cap) {
    free_.clear();
    if (cap) free_[0] = cap;
    cap_ = cap;
    used_ = 0;
  }
  bool alloc(size_t sz, size_t* off) {
    sz = (sz + 255) & ~(size_t)255;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= sz) {
        *off = it->first;
        const size_t rest = it->second - sz, at = it->first + sz;
        free_.erase(it);
        if (rest) free_[at] = rest;
        used_ += sz;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t sz) {
    sz = (sz + 255) & ~(size_t)255;
    used_ -= sz;
    auto it = free_.emplace(off, sz).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t cap() const { return cap_; }
  size_t used() const { return used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t cap_ = 0, used_ = 0;
};

size_t slot_bytes(uint32_t n, bool pred) {
  const size_t r = ((size_t)n * 4 + 255) & ~(size_t)255;
  return (pred ? 2 : 1) * r + 6 * r;   // labels + stamp, farflag, qa, qb, fa, fb
}

struct SrvGraph {
  b2_graph g;
  uint32_t n;
  bool isf;
  bool big;             // solved by a block cluster instead of one block
  double delta_scale;   // Near-Far constant of the bucket width
  uint32_t delta_u;
  float inv_delta;
  bool tuned;           // big / delta_scale were picked by measurement
};

struct SrvQuery {
  uint64_t ticket;
  int32_t gid;
  uint32_t source;
  void* out_dist;
  int32_t* out_pred;
  uint64_t t_submit;
  size_t off = 0, bytes = 0;
  int32_t rec = -1;
};

struct Lane {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  uint32_t* d_next = nullptr;
  ServeQuery* h_desc = nullptr;   // mapped page-locked, max_batch entries
  bool busy = false;
  bool big = false;               // launches cluster batches (queries on big graphs)
  // The launch sequence of a batch (reset the query counter, run the teams)
  // as an instantiated CUDA graph per team kind; each batch updates the
  // kernel node's grid and arguments and replays it.
  // (the source graph stays alive with its instantiation: kernel-node
  // updates name a node of the graph the executable was made from)
  cudaGraph_t gsrc[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  cudaGraphNode_t knode[2] = {nullptr, nullptr};
  bool graph_failed = false;      // graph API refused: launch directly
};

// Build (once per lane and kind) or update the batch graph and launch it.
cudaError_t launch_batch_graph(Lane& ln, bool big, uint32_t grid, uint32_t nq, unsigned long long budget) {
  const int k = big ? 1 : 0;
  const ServeQuery* desc = ln.h_desc;
  uint32_t* next = ln.d_next;
  void* args[] = {(void*)&desc, (void*)&nq, (void*)&next, (void*)&budget};
  cudaKernelNodeParams kp;
  memset(&kp, 0, sizeof(kp));
  kp.func = big ? (void*)k_serve_cluster : (void*)k_serve;
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(kServeThreads);
  kp.sharedMemBytes = 0;
  kp.kernelParams = args;
  cudaError_t e = cudaSuccess;
  if (!ln.gexec[k]) {
    cudaGraph_t graph = nullptr;
    e = cudaGraphCreate(&graph, 0);
    cudaGraphNode_t mnode = nullptr;
    if (e == cudaSuccess) {
      cudaMemsetParams mp;
      memset(&mp, 0, sizeof(mp));
      mp.dst = ln.d_next;
      mp.value = 0;
      mp.elementSize = 4;
      mp.width = 1;
      mp.height = 1;
      e = cudaGraphAddMemsetNode(&mnode, graph, nullptr, 0, &mp);
    }
    if (e == cudaSuccess) e = cudaGraphAddKernelNode(&ln.knode[k], graph, &mnode, 1, &kp);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ln.gexec[k], graph, 0);
    if (e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      ln.gexec[k] = nullptr;
      ln.knode[k] = nullptr;
      return e;
    }
    ln.gsrc[k] = graph;
  } else {
    e = cudaGraphExecKernelNodeSetParams(ln.gexec[k], ln.knode[k], &kp);
    if (e != cudaSuccess) return e;
  }
  return cudaGraphLaunch(ln.gexec[k], ln.st);
}

bool mapped_or_device(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged ||
         (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr);
}

}  // namespace
}  // namespace b2

struct b2_server_s {
  b2_server_opts o;
  int device = 0;
  char* arena = nullptr;
  b2::RangeAlloc alloc;
  std::vector<b2::SrvGraph> graphs;
  std::deque<b2::SrvQuery> pending;
  std::vector<b2::SrvQuery> running;
  std::vector<b2_completion> done;
  std::vector<b2::Lane> lanes;
  b2::ServeRecord* recs = nullptr;   // mapped page-locked
  std::vector<int32_t> free_recs;
  uint64_t next_ticket = 1;
  uint32_t grid_cap = 0;
  uint32_t cluster_cap = 0;   // clusters resident at once
  uint32_t big_n = 0;         // graphs with at least this many vertices are big
  std::mutex mu;
};

namespace b2 {
namespace {

// One batch of queries of the lane's kind (big-graph queries on cluster lanes,
// the others on block lanes), FIFO within the kind.  With a single lane the
// lane takes the kind of the oldest pending query.
b2_status srv_launch(b2_server s, Lane& ln) {
  std::vector<SrvQuery> batch;
  bool big = ln.big;
  if (s->lanes.size() < 2 && !s->pending.empty()) big = s->graphs[s->pending.front().gid].big;
  for (auto it = s->pending.begin();
       it != s->pending.end() && (int32_t)batch.size() < s->o.max_batch && !s->free_recs.empty();) {
    SrvQuery& q = *it;
    const SrvGraph& G = s->graphs[q.gid];
    if (G.big != big) { ++it; continue; }
    q.bytes = slot_bytes(G.n, q.out_pred != nullptr);
    if (!s->alloc.alloc(q.bytes, &q.off)) break;   // HBM budget: wait for running queries to finish
    q.rec = s->free_recs.back();
    s->free_recs.pop_back();
    batch.push_back(q);
    it = s->pending.erase(it);
  }
  if (batch.empty()) return B2_SUCCESS;
  for (size_t i = 0; i < batch.size(); ++i) {
    const SrvQuery& q = batch[i];
    const SrvGraph& G = s->graphs[q.gid];
    const size_t r = ((size_t)G.n * 4 + 255) & ~(size_t)255;
    char* base = s->arena + q.off;
    const bool pred = q.out_pred != nullptr;
    ServeQuery& d = ln.h_desc[i];
    d.rowptr = G.g->rowptr;
    d.edges = G.g->edges;
    d.n = G.n;
    d.source = internal_id(G.g, q.source);
    d.perm = G.g->perm;
    d.is_float = G.isf ? 1u : 0u;
    d.pred = pred ? 1u : 0u;
    d.delta_u = G.delta_u;
    d.inv_delta = G.inv_delta;
    d.labels = base;
    char* p = base + (pred ? 2 : 1) * r;
    d.stamp = (uint32_t*)p;
    d.farflag = (uint32_t*)(p + r);
    d.qa = (uint32_t*)(p + 2 * r);
    d.qb = (uint32_t*)(p + 3 * r);
    d.fa = (uint32_t*)(p + 4 * r);
    d.fb = (uint32_t*)(p + 5 * r);
    d.out_dist = (uint32_t*)q.out_dist;
    d.out_pred = q.out_pred;
    s->recs[q.rec].flag = 0;
    d.rec = s->recs + q.rec;
  }
  std::atomic_thread_fence(std::memory_order_seq_cst);
  const uint32_t nq = (uint32_t)batch.size();
  const uint32_t grid = big ? std::min(nq, s->cluster_cap) * kClusterCTAs : std::min(nq, s->grid_cap);
  // per-query device budget in ns (at least 1 ns: a tiny budget must still time out)
  const unsigned long long budget = (unsigned long long)std::max(1.0, s->o.timeout_ms * 1.0e6);
  cudaError_t ge = cudaErrorNotSupported;
  if (!ln.graph_failed) {
    ge = launch_batch_graph(ln, big, grid, nq, budget);
    if (ge != cudaSuccess) {
      cudaGetLastError();
      ln.graph_failed = true;   // the same two launches, issued directly from now on
    }
  }
  if (ge != cudaSuccess) {
    B2_CUDA_TRY(cudaMemsetAsync(ln.d_next, 0, 4, ln.st));
    if (big) k_serve_cluster<<<grid, kServeThreads, 0, ln.st>>>(ln.h_desc, nq, ln.d_next, budget);
    else k_serve<<<grid, kServeThreads, 0, ln.st>>>(ln.h_desc, nq, ln.d_next, budget);
    B2_CUDA_TRY(cudaGetLastError());
  }
  B2_CUDA_TRY(cudaEventRecord(ln.done, ln.st));
  ln.busy = true;
  for (auto& q : batch) s->running.push_back(q);
  return B2_SUCCESS;
}

int srv_reap(b2_server s) {
  int got = 0;
  const uint64_t t = now_ns();
  for (size_t i = 0; i < s->running.size();) {
    SrvQuery& q = s->running[i];
    volatile ServeRecord* r = s->recs + q.rec;
    if (r->flag == 1u) {
      std::atomic_thread_fence(std::memory_order_acquire);
      b2_completion c;
      memset(&c, 0, sizeof(c));
      c.ticket = q.ticket;
      c.graph_id = q.gid;
      c.source = q.source;
      c.status = r->status == 0 ? B2_SUCCESS : (r->status == kErrTimeout ? B2_TIMEOUT : B2_POOL_EXHAUSTED);
      c.phases = r->phases;
      c.edges_scanned = r->edges_scanned;
      c.reached = r->reached;
      c.reached_edges = r->reached_edges;
      c.latency_us = (double)(t - q.t_submit) * 1e-3;
      s->done.push_back(c);
      s->alloc.release(q.off, q.bytes);
      s->free_recs.push_back(q.rec);
      s->running[i] = s->running.back();
      s->running.pop_back();
      ++got;
    } else {
      ++i;
    }
  }
  for (auto& ln : s->lanes)
    if (ln.busy && cudaEventQuery(ln.done) == cudaSuccess) ln.busy = false;
  return got;
}

b2_status srv_progress(b2_server s) {
  srv_reap(s);
  for (auto& ln : s->lanes) {
    if (s->pending.empty()) break;
    if (ln.busy) continue;
    b2_status st = srv_launch(s, ln);
    if (st != B2_SUCCESS) return st;
  }
  return B2_SUCCESS;
}

// Autotuner: for one graph, time batches of queries that fill the GPU under
// each candidate (team: one block or an 8-block cluster; Near-Far constant 2,
// 4 or 8) and keep the configuration with the highest throughput.  Every
// tuning query writes the same device buffer (results are discarded; the
// stores do not interact).  Runs only on an idle server.
b2_status set_bucket_width(SrvGraph& G, double scale);
b2_status srv_submit(b2_server s, int32_t graph_id, uint32_t source, void* out_dist, int32_t* out_pred,
                     uint64_t t_submit, bool check_ptrs, uint64_t* ticket);
b2_status srv_tune_graph(b2_server s, int32_t gid) {
  SrvGraph& G0 = s->graphs[gid];
  const size_t slot = slot_bytes(G0.n, false);
  uint32_t* d_out = nullptr;
  B2_CUDA_TRY(cudaMalloc((void**)&d_out, (size_t)G0.n * 4));
  const double scales[3] = {2.0, 4.0, 8.0};
  double best_qps = -1.0;
  bool best_big = s->graphs[gid].big;
  double best_scale = s->graphs[gid].delta_scale;
  b2_status status = B2_SUCCESS;
  for (int team = 0; team < 2 && status == B2_SUCCESS; ++team) {
    const uint32_t fill = team ? s->cluster_cap : s->grid_cap;
    const size_t free_b = s->alloc.cap() - s->alloc.used();
    const uint32_t q = (uint32_t)std::min<size_t>(std::min<size_t>(fill, (size_t)s->o.max_batch), free_b / slot);
    if (q == 0) continue;
    for (double sc : scales) {
      SrvGraph& G = s->graphs[gid];
      G.big = team == 1;
      if (set_bucket_width(G, sc) != B2_SUCCESS) continue;
      double elapsed = 0.0;
      uint64_t done_q = 0;
      for (int rep = 0; rep < 8 && status == B2_SUCCESS; ++rep) {
        const uint64_t t0 = now_ns();
        for (uint32_t i = 0; i < q; ++i) {
          uint64_t tk = 0;
          status = srv_submit(s, gid, (uint32_t)(((uint64_t)i * 2654435761ull) % G.n), d_out, nullptr, t0, false,
                              &tk);
          if (status != B2_SUCCESS) break;
        }
        const uint64_t tlim = t0 + (uint64_t)(4.0 * s->o.timeout_ms * 1e6) + 60000000000ull;
        while (status == B2_SUCCESS && (!s->pending.empty() || !s->running.empty())) {
          status = srv_progress(s);
          if (now_ns() > tlim) status = B2_TIMEOUT;
        }
        s->done.clear();
        if (rep == 0) continue;                    // warm-up batch
        elapsed += (double)(now_ns() - t0) * 1e-9;
        done_q += q;
        if (elapsed > 0.05 && rep >= 2) break;
      }
      const double qps = elapsed > 0 ? (double)done_q / elapsed : 0.0;
      if (qps > best_qps) {
        best_qps = qps;
        best_big = team == 1;
        best_scale = sc;
      }
    }
  }
  cudaFree(d_out);
  SrvGraph& G = s->graphs[gid];
  G.big = best_big;
  b2_status st2 = set_bucket_width(G, best_scale);
  G.tuned = status == B2_SUCCESS && st2 == B2_SUCCESS;
  return status != B2_SUCCESS ? status : st2;
}

// Whole device: cancel nothing, wait for every running query (bounded by the
// per-query budget, which the kernels enforce themselves).
b2_status srv_drain_running(b2_server s) {
  for (auto& ln : s->lanes)
    if (ln.busy) {
      B2_CUDA_TRY(cudaEventSynchronize(ln.done));
      ln.busy = false;
    }
  srv_reap(s);
  return B2_SUCCESS;
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" void b2_server_opts_default(b2_server_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->hbm_budget_bytes = (size_t)1 << 30;
  o->max_batch = 512;
  o->lanes = 16;   // concurrent batch launches: a long query holds only its own lane
  o->max_inflight = 8192;
  o->timeout_ms = 20000.0;
  o->delta_scale = 4.0;   // narrower than the full-GPU default: a CTA's phases end with block barriers
  o->blocks_per_sm = 0;
}

extern "C" b2_status b2_server_create(const b2_server_opts* opts, b2_server* out) {
  if (!out) return B2_INVALID_ARGUMENT;
  b2_server_opts o;
  if (opts) o = *opts; else b2_server_opts_default(&o);
  if (o.max_batch <= 0 || o.lanes <= 0 || o.lanes > 64 || o.max_inflight <= 0 || o.hbm_budget_bytes < 256)
    return B2_INVALID_ARGUMENT;
  b2_server s = new b2_server_s();
  s->o = o;
  cudaGetDevice(&s->device);
  auto fail = [&](cudaError_t e) {
    b2_server_destroy(s);
    return from_cuda(e);
  };
  cudaError_t e = cudaMalloc((void**)&s->arena, o.hbm_budget_bytes);
  if (e != cudaSuccess) return fail(e);
  s->alloc.reset(o.hbm_budget_bytes & ~(size_t)255);
  e = cudaHostAlloc((void**)&s->recs, sizeof(ServeRecord) * (size_t)o.max_inflight, cudaHostAllocMapped);
  if (e != cudaSuccess) return fail(e);
  memset(s->recs, 0, sizeof(ServeRecord) * (size_t)o.max_inflight);
  for (int32_t i = o.max_inflight - 1; i >= 0; --i) s->free_recs.push_back(i);
  s->lanes.resize(o.lanes);
  for (auto& ln : s->lanes) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ln.st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc((void**)&ln.d_next, 4);
    if (e == cudaSuccess)
      e = cudaHostAlloc((void**)&ln.h_desc, sizeof(ServeQuery) * (size_t)o.max_batch, cudaHostAllocMapped);
  }
  if (e != cudaSuccess) return fail(e);
  int per = 0, sms = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_serve, kServeThreads, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  if (o.blocks_per_sm > 0) per = std::min(per, o.blocks_per_sm);
  s->grid_cap = (uint32_t)std::max(1, per * sms);
  {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCTAs);
    cfg.blockDim = dim3(kServeThreads);
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kClusterCTAs;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, (void*)k_serve_cluster, &cfg) != cudaSuccess || clusters < 1) {
      cudaGetLastError();
      clusters = std::max(1, (int)(s->grid_cap / (2 * kClusterCTAs)));
    }
    s->cluster_cap = (uint32_t)clusters;
  }
  s->big_n = o.big_vertices > 0 ? (uint32_t)o.big_vertices : (o.big_vertices < 0 ? 0xFFFFFFFFu : (1u << 19));
  // a quarter of the lanes (at least one) launch cluster batches
  const int nbig = std::max(1, o.lanes / 4);
  for (int i = 0; i < o.lanes; ++i) s->lanes[i].big = o.lanes >= 2 && i >= o.lanes - nbig;
  *out = s;
  return B2_SUCCESS;
}

extern "C" b2_status b2_server_destroy(b2_server s) {
  if (!s) return B2_INVALID_ARGUMENT;
  for (auto& ln : s->lanes)
    if (ln.st) cudaStreamSynchronize(ln.st);
  for (auto& ln : s->lanes) {
    for (int k = 0; k < 2; ++k) {
      if (ln.gexec[k]) cudaGraphExecDestroy(ln.gexec[k]);
      if (ln.gsrc[k]) cudaGraphDestroy(ln.gsrc[k]);
    }
    if (ln.st) cudaStreamDestroy(ln.st);
    if (ln.done) cudaEventDestroy(ln.done);
    cudaFree(ln.d_next);
    if (ln.h_desc) cudaFreeHost(ln.h_desc);
  }
  if (s->recs) cudaFreeHost(s->recs);
  cudaFree(s->arena);
  delete s;
  return B2_SUCCESS;
}

namespace b2 {
namespace {
b2_status set_bucket_width(SrvGraph& G, double scale) {
  double delta = 1.0;
  b2_delta_heuristic(G.g, scale, &delta);
  if (G.isf) {
    const float df = (float)delta;
    if (!(df > 0.0f) || !std::isfinite(df)) return B2_INVALID_ARGUMENT;
    G.inv_delta = 1.0f / df;
    G.delta_u = 1;
  } else {
    G.delta_u = (uint32_t)std::min(4294967295.0, std::max(1.0, std::floor(delta)));
    G.inv_delta = 0.0f;
  }
  G.delta_scale = scale;
  return B2_SUCCESS;
}
b2_status srv_tune_graph(b2_server s, int32_t gid);
}  // namespace
}  // namespace b2

extern "C" b2_status b2_server_add_graph(b2_server s, b2_graph g, int32_t* graph_id) {
  if (!s || !g || !graph_id) return B2_INVALID_ARGUMENT;
  if (g->has_negative) return B2_INVALID_WEIGHT;
  if (g->n <= 0 || g->n > 0x7fffffff) return B2_NOT_SUPPORTED;
  std::lock_guard<std::mutex> lock(s->mu);
  SrvGraph G;
  G.g = g;
  G.n = (uint32_t)g->n;
  G.isf = g->weight_type == B2_W_F32;
  G.big = G.n >= s->big_n;
  G.tuned = false;
  b2_status st = set_bucket_width(G, s->o.delta_scale > 0 ? s->o.delta_scale : 4.0);
  if (st != B2_SUCCESS) return st;
  s->graphs.push_back(G);
  *graph_id = (int32_t)s->graphs.size() - 1;
  if (s->o.autotune) {
    if (!s->pending.empty() || !s->running.empty()) return B2_SUCCESS;   // busy: keep the defaults
    st = srv_tune_graph(s, *graph_id);
    if (st != B2_SUCCESS) {
      s->graphs.pop_back();
      return st;
    }
  }
  return B2_SUCCESS;
}

extern "C" b2_status b2_server_graph_config(b2_server s, int32_t graph_id, int32_t* cluster_team,
                                            double* delta_scale, int32_t* tuned) {
  if (!s) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  if (graph_id < 0 || graph_id >= (int32_t)s->graphs.size()) return B2_INVALID_ARGUMENT;
  const SrvGraph& G = s->graphs[graph_id];
  if (cluster_team) *cluster_team = G.big ? 1 : 0;
  if (delta_scale) *delta_scale = G.delta_scale;
  if (tuned) *tuned = G.tuned ? 1 : 0;
  return B2_SUCCESS;
}

namespace b2 {
namespace {
b2_status srv_submit(b2_server s, int32_t graph_id, uint32_t source, void* out_dist, int32_t* out_pred,
                     uint64_t t_submit, bool check_ptrs, uint64_t* ticket) {
  if (graph_id < 0 || graph_id >= (int32_t)s->graphs.size()) return B2_INVALID_ARGUMENT;
  const SrvGraph& G = s->graphs[graph_id];
  if (source >= G.n) return B2_INVALID_ARGUMENT;
  if (check_ptrs && (!mapped_or_device(out_dist) || (out_pred && !mapped_or_device(out_pred))))
    return B2_INVALID_ARGUMENT;
  if (slot_bytes(G.n, out_pred != nullptr) > s->alloc.cap()) return B2_OUT_OF_MEMORY;   // can never be admitted
  SrvQuery q;
  q.ticket = s->next_ticket++;
  q.gid = graph_id;
  q.source = source;
  q.out_dist = out_dist;
  q.out_pred = out_pred;
  q.t_submit = t_submit;
  s->pending.push_back(q);
  *ticket = q.ticket;
  return B2_SUCCESS;
}
}  // namespace
}  // namespace b2

extern "C" b2_status b2_server_submit(b2_server s, int32_t graph_id, uint32_t source, void* out_dist,
                                      int32_t* out_pred, uint64_t* ticket) {
  if (!s || !out_dist || !ticket) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  return srv_submit(s, graph_id, source, out_dist, out_pred, now_ns(), true, ticket);
}

extern "C" b2_status b2_server_cancel(b2_server s, uint64_t ticket) {
  if (!s) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
    if (it->ticket == ticket) {
      b2_completion c;
      memset(&c, 0, sizeof(c));
      c.ticket = ticket;
      c.graph_id = it->gid;
      c.source = it->source;
      c.status = B2_CANCELLED;
      c.latency_us = (double)(now_ns() - it->t_submit) * 1e-3;
      s->done.push_back(c);
      s->pending.erase(it);
      return B2_SUCCESS;
    }
  }
  return B2_NOT_SUPPORTED;   // unknown, or already running (a running query is never interrupted)
}

extern "C" b2_status b2_server_progress(b2_server s, int32_t wait_all) {
  if (!s) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  b2_status st = srv_progress(s);
  if (st != B2_SUCCESS || !wait_all) return st;
  const uint64_t t0 = now_ns();
  while (!s->pending.empty() || !s->running.empty()) {
    st = srv_progress(s);
    if (st != B2_SUCCESS) return st;
    if (s->pending.empty() && !s->running.empty()) {
      bool any_busy = false;
      for (auto& ln : s->lanes) any_busy |= ln.busy;
      if (!any_busy) srv_reap(s);   // kernels ended: every record is final
      if (!any_busy && !s->running.empty()) {
        // a kernel ended without publishing a record: report, do not spin
        for (auto& q : s->running) {
          b2_completion c;
          memset(&c, 0, sizeof(c));
          c.ticket = q.ticket;
          c.graph_id = q.gid;
          c.source = q.source;
          c.status = B2_DEVICE_ERROR;
          s->done.push_back(c);
          s->alloc.release(q.off, q.bytes);
          s->free_recs.push_back(q.rec);
        }
        s->running.clear();
      }
    }
    if ((double)(now_ns() - t0) * 1e-6 > 4.0 * s->o.timeout_ms + 60000.0) return B2_TIMEOUT;
  }
  return B2_SUCCESS;
}

extern "C" b2_status b2_server_poll(b2_server s, b2_completion* out, int32_t capacity, int32_t* count) {
  if (!s || !count || capacity < 0 || (capacity > 0 && !out)) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  srv_reap(s);
  const int32_t k = std::min<int32_t>(capacity, (int32_t)s->done.size());
  for (int32_t i = 0; i < k; ++i) out[i] = s->done[i];
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *count = k;
  return B2_SUCCESS;
}

extern "C" b2_status b2_server_info(b2_server s, b2_server_info_t* info) {
  if (!s || !info) return B2_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  memset(info, 0, sizeof(*info));
  info->graphs = (int32_t)s->graphs.size();
  info->pending = (int64_t)s->pending.size();
  info->running = (int64_t)s->running.size();
  info->completed_unpolled = (int64_t)s->done.size();
  info->arena_bytes = s->alloc.cap();
  info->arena_used = s->alloc.used();
  info->blocks = s->grid_cap;
  return B2_SUCCESS;
}

extern "C" size_t b2_server_slot_bytes(int64_t n, int32_t with_pred) {
  if (n <= 0 || n > 0x7fffffff) return 0;
  return slot_bytes((uint32_t)n, with_pred != 0);
}

// ---------------------------------------------------------------------------
// Load generator: Poisson arrivals (exponential gaps, seeded), uniform graph
// and source per query, results into a page-locked host pool.  Latency is
// measured from each query's scheduled arrival to the moment its result is
// in host memory, so queueing delay counts.  mode 1 answers the same stream
// one query at a time with the full-GPU delta-stepping solve and a
// device-to-host copy (the sequential baseline).
namespace b2 {
namespace {
uint64_t checksum_words(const uint32_t* p, uint32_t n) {
  uint64_t h = 0x9E3779B97F4A7C15ull;
  for (uint32_t i = 0; i < n; ++i) h = (h ^ p[i]) * 0x100000001B3ull + i;
  return h;
}
double pct(std::vector<double>& v, double q) {
  if (v.empty()) return 0.0;
  const size_t k = std::min(v.size() - 1, (size_t)std::floor(q * (double)(v.size() - 1) + 0.5));
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}
}  // namespace
}  // namespace b2

extern "C" void b2_load_opts_default(b2_load_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->queries = 1024;
  o->rate_qps = 0.0;
  o->seed = 1;
  o->host_result_bytes = (size_t)1 << 30;
}

extern "C" b2_status b2_server_run_load(b2_server s, const b2_load_opts* opts, b2_load_report* rep) {
  if (!s || !opts || !rep || opts->queries <= 0) return B2_INVALID_ARGUMENT;
  const b2_load_opts& o = *opts;
  std::vector<int32_t> gids;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->graphs.empty() || !s->pending.empty() || !s->running.empty()) return B2_INVALID_ARGUMENT;
    if (o.graph_ids && o.n_graph_ids > 0) {
      for (int32_t i = 0; i < o.n_graph_ids; ++i) {
        if (o.graph_ids[i] < 0 || o.graph_ids[i] >= (int32_t)s->graphs.size()) return B2_INVALID_ARGUMENT;
        gids.push_back(o.graph_ids[i]);
      }
    } else {
      for (int32_t i = 0; i < (int32_t)s->graphs.size(); ++i) gids.push_back(i);
    }
  }
  const int64_t Q = o.queries;
  std::mt19937_64 rng(o.seed);
  std::vector<double> arrival((size_t)Q);
  std::vector<int32_t> qg((size_t)Q);
  std::vector<uint32_t> qs((size_t)Q);
  double t = 0.0;
  for (int64_t i = 0; i < Q; ++i) {
    if (o.rate_qps > 0) {
      const double u = ((double)(rng() >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      t += -std::log(u) / o.rate_qps;
    }
    arrival[i] = t;
    qg[i] = gids[rng() % gids.size()];
    qs[i] = (uint32_t)(rng() % s->graphs[qg[i]].n);
  }
  uint32_t max_n = 0;
  for (int32_t g : gids) max_n = std::max(max_n, s->graphs[g].n);
  const bool pred = o.with_pred != 0;
  const size_t per_n = pred ? 8 : 4;
  size_t pool = std::max(o.host_result_bytes, (size_t)max_n * per_n + 512);
  char* host = nullptr;
  B2_CUDA_TRY(cudaHostAlloc((void**)&host, pool, cudaHostAllocMapped));
  RangeAlloc hp;
  hp.reset(pool & ~(size_t)255);
  std::vector<double> lat;
  lat.reserve((size_t)Q);
  int64_t completed = 0, failed = 0;
  unsigned long long redges = 0;
  b2_status status = B2_SUCCESS;
  const uint64_t t0 = now_ns();
  uint64_t t_last = t0;
  if (o.mode == 1) {
    // one query at a time: full-GPU solve, copy to host, next
    void* d_dist = nullptr;
    int32_t* d_pred = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaMalloc(&d_dist, (size_t)max_n * 4);
    if (e == cudaSuccess && pred) e = cudaMalloc((void**)&d_pred, (size_t)max_n * 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) status = from_cuda(e);
    b2_sssp_opts so;
    b2_sssp_opts_default(&so);
    so.timeout_ms = s->o.timeout_ms;
    // (the plain solver's own Near-Far delta: this mode is the one-at-a-time baseline)
    so.collect_reach = 1;
    for (int64_t i = 0; i < Q && status == B2_SUCCESS; ++i) {
      const uint64_t due = t0 + (uint64_t)(arrival[i] * 1e9);
      while (now_ns() < due) std::this_thread::yield();
      const SrvGraph& G = s->graphs[qg[i]];
      b2_stats stt;
      b2_status r = b2_sssp_delta(G.g, qs[i], d_dist, d_pred, &so, st, &stt);
      if (r == B2_SUCCESS) {
        e = cudaMemcpyAsync(host, d_dist, (size_t)G.n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && pred)
          e = cudaMemcpyAsync(host + (size_t)G.n * 4, d_pred, (size_t)G.n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { status = from_cuda(e); break; }
        redges += stt.reached_edges;
        if (o.checksums) o.checksums[i] = checksum_words((const uint32_t*)host, G.n);
      } else {
        ++failed;
      }
      t_last = now_ns();
      lat.push_back((double)(t_last - due) * 1e-3);
      ++completed;
    }
    if (st) cudaStreamDestroy(st);
    cudaFree(d_dist);
    cudaFree(d_pred);
  } else {
    struct Live { int64_t idx; size_t off, bytes; };
    std::map<uint64_t, Live> live;
    int64_t next = 0;
    std::vector<b2_completion> buf(1024);
    const double limit_s = (arrival.back() + 60.0) + 4.0 * s->o.timeout_ms * 1e-3 + 600.0;
    while (completed < Q && status == B2_SUCCESS) {
      bool acted = false;
      {
        std::lock_guard<std::mutex> lock(s->mu);
        const uint64_t tn = now_ns();
        while (next < Q && t0 + (uint64_t)(arrival[next] * 1e9) <= tn) {
          const SrvGraph& G = s->graphs[qg[next]];
          const size_t need = (size_t)G.n * per_n;
          size_t off = 0;
          if (!hp.alloc(need, &off)) break;                 // host pool full: back-pressure
          uint64_t tk = 0;
          char* out = host + off;
          b2_status r = srv_submit(s, qg[next], qs[next], out, pred ? (int32_t*)(out + (size_t)G.n * 4) : nullptr,
                                   t0 + (uint64_t)(arrival[next] * 1e9), false, &tk);
          if (r != B2_SUCCESS) { hp.release(off, need); status = r; break; }
          live[tk] = Live{next, off, need};
          ++next;
          acted = true;
        }
        if (status != B2_SUCCESS) break;
        status = srv_progress(s);
        const int32_t k = std::min<int32_t>((int32_t)buf.size(), (int32_t)s->done.size());
        for (int32_t j = 0; j < k; ++j) buf[j] = s->done[j];
        s->done.erase(s->done.begin(), s->done.begin() + k);
        for (int32_t j = 0; j < k; ++j) {
          const b2_completion& c = buf[j];
          auto it = live.find(c.ticket);
          if (it == live.end()) continue;
          const Live L = it->second;
          live.erase(it);
          if (c.status != B2_SUCCESS) ++failed;
          redges += c.reached_edges;
          lat.push_back(c.latency_us);
          if (o.checksums) o.checksums[L.idx] = checksum_words((const uint32_t*)(host + L.off), s->graphs[qg[L.idx]].n);
          hp.release(L.off, L.bytes);
          ++completed;
          acted = true;
        }
        t_last = now_ns();
      }
      if ((double)(t_last - t0) * 1e-9 > limit_s) { status = B2_TIMEOUT; break; }
      if (!acted) std::this_thread::yield();
    }
    if (status != B2_SUCCESS) {
      std::lock_guard<std::mutex> lock(s->mu);
      s->pending.clear();
      srv_drain_running(s);
      s->done.clear();
    }
  }
  cudaFreeHost(host);
  memset(rep, 0, sizeof(*rep));
  rep->completed = completed;
  rep->failed = failed;
  rep->elapsed_s = (double)(t_last - t0) * 1e-9;
  rep->qps = rep->elapsed_s > 0 ? (double)completed / rep->elapsed_s : 0.0;
  double sum = 0.0, mx = 0.0;
  for (double x : lat) { sum += x; mx = std::max(mx, x); }
  rep->mean_us = lat.empty() ? 0.0 : sum / (double)lat.size();
  rep->max_us = mx;
  rep->p50_us = pct(lat, 0.50);
  rep->p99_us = pct(lat, 0.99);
  rep->reached_edges = redges;
  rep->gteps = rep->elapsed_s > 0 ? (double)redges / rep->elapsed_s * 1e-9 : 0.0;
  if (o.query_graph) for (int64_t i = 0; i < Q; ++i) o.query_graph[i] = qg[i];
  if (o.query_source) for (int64_t i = 0; i < Q; ++i) o.query_source[i] = qs[i];
  return status;
}
