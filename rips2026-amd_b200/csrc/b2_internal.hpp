// Host-side internals of libb200sssp: resident graph handle, solver
// workspace, error helpers.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/b200sssp.h"

namespace b2 {

#define B2_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ::b2::from_cuda(_e);      \
  } while (0)

inline b2_status from_cuda(cudaError_t e) {
  if (e == cudaSuccess) return B2_SUCCESS;
  if (e == cudaErrorMemoryAllocation) return B2_OUT_OF_MEMORY;
  if (e == cudaErrorInvalidValue) return B2_INVALID_ARGUMENT;
  return B2_CUDA_ERROR;
}

// Number of ring buckets in the delta-stepping window (aligned windows of
// kRing consecutive buckets; buckets past the window go to the far pile).
constexpr int kRing = 16;
// Edges per hub chunk (vertices with out-degree >= hub_degree are split into
// chunks of this many edges that any warp of the grid may take).
constexpr uint32_t kHubChunk = 256;

// One 256-edge chunk of a high-degree vertex's phase range.
struct HubEntry {
  uint32_t v;
  uint32_t chunk;  // chunk index within v's edge range of the phase
};

// Control block of one persistent solve (device memory).  The manager step
// (last block to arrive at a grid barrier) is the only writer of the phase
// record; counters are written by all blocks during a phase.
struct PhaseRec {
  uint32_t kind;        // PhaseKind
  uint32_t phase;       // monotone phase id (also the near-queue dedup stamp base)
  uint32_t fq;          // frontier queue id (QueueId)
  uint32_t fcount;      // entries in the frontier queue
  uint32_t push_q;      // near queue receiving same-bucket pushes
  uint32_t stamp;       // dedup stamp for those pushes
  uint32_t hub_in;      // hub list consumed this phase
  uint32_t hub_in_count;
  uint32_t hub_in_chunks;
  uint32_t hub_out;     // hub list produced this phase
  uint32_t cur;         // current bucket (delta)
  uint32_t win;         // window base bucket (delta)
  uint32_t far_sel;     // far pile being appended to (delta)
  uint32_t iter;        // BF iteration being executed
  uint32_t heavy;       // 1: relax the heavy suffix (w > delta) of each frontier vertex
  uint32_t hround;      // stamp of the current heavy round (members dedup)
  uint32_t aux;         // BF: round role (0 normal, 2 commit-before-probe, 1 probe); FINAL: source buffer
  uint32_t dq;          // bucket width (uint32 graphs)
  uint32_t dinv;        // float bits of 1/width (float graphs)
  uint32_t dbase;       // distance key at which bucket dbase_b starts (0 until re-based)
  uint32_t dbase_b;
  uint32_t dense;       // 0: read the frontier queue; kDenseNear / kDenseSlot: sweep the stamps
  uint32_t fstamp;      // stamp value marking the frontier's vertices in a sweep
};

// One entry per executed phase when tracing is on (manager-written).
struct TraceEntry {
  uint32_t kind;        // PhaseKind | heavy << 8
  uint32_t fcount;      // frontier entries
  uint32_t hub_chunks;  // hub chunks consumed
  uint32_t cur;         // bucket (delta) or round (BF)
  unsigned long long t_ns;  // end of the phase, ns since the first barrier
};
constexpr uint32_t kTraceCap = 4096;

enum PhaseKind : uint32_t {
  kPhaseInit = 0,
  kPhaseProcess = 1,   // relax a frontier (+ hub chunks of the previous phase)
  kPhaseCommit = 2,    // BF: dist_cur[v] = dist_next[v] for v in frontier
  kPhaseSplit = 3,     // delta: move far-pile entries into the new window
  kPhaseProbe = 4,     // delta: count valid pending entries (max_iters cut)
  kPhaseFinal = 5,     // write outputs
  kPhaseDone = 6,
  kPhaseLocal = 7,     // delta: block 0 alone runs small light sub-phases (bucket fusion)
  kPhasePull = 8,      // delta: heavy pass in the pull direction (unsettled vertices scan in-edges)
};

// How a delta-stepping relaxation phase finds its frontier.  A large near
// frontier is the set of vertices whose push stamp equals the previous phase's
// stamp; a large window-slot frontier is the set whose bucket stamp equals the
// current bucket.  Sweeping those stamps in vertex order replaces random queue
// order with ordered access to labels, row pointers and rows.
enum DenseKind : uint32_t {
  kDenseOff = 0,
  kDenseNear = 1,
  kDenseSlot = 2,
};

enum QueueId : uint32_t {
  kQNear0 = 0,
  kQNear1 = 1,
  kQFar0 = 2,
  kQFar1 = 3,
  kQMembers = 4,  // vertices settled in the current heavy round
  kQSlot0 = 5,    // kQSlot0 + s, s < kRing
  kQNone = 0xFFFFFFFFu,
};

struct Control {
  // grid barrier (must stay first; see b2_common.cuh GridBarrier)
  uint32_t bar_arrive;
  uint32_t bar_gen;
  uint32_t error;
  uint32_t error_site;
  PhaseRec rec;
  // counters produced during phases
  uint32_t near_count[2];
  uint32_t far_count[2];
  uint32_t slot_count[kRing];
  uint32_t far_min;        // lower bound of buckets in the active far pile
  uint32_t far_min_next;   // exact min of the kept entries during a split
  uint32_t hub_count[2];   // chunk entries in each hub list
  uint32_t work_next;      // dynamic work counter of the running phase
  uint32_t bucket_valid;   // a valid vertex was processed in the current bucket
  uint32_t probe_valid;    // PROBE phase result
  uint32_t members_count;  // entries in the heavy-round member list
  uint32_t trace_n;
  uint32_t stamp_ctr;      // next dedup stamp (manager and local loop)
  uint32_t local_q;        // LOCAL phase: queue holding the next frontier
  uint32_t local_iters;    // LOCAL phase: sub-phases run inside it
  uint32_t fusion_off;     // a LOCAL sub-phase scanned too many edges: no more fusion this solve
  uint32_t local_total;    // sub-phases run by all LOCAL phases
  unsigned long long member_heavy;       // heavy out-edges of the current bucket's members (push cost)
  uint32_t cur_min_key;                  // smallest label processed in the current bucket (pull bound)
  uint32_t heavy_pulls;                  // heavy passes run by pull
  uint32_t delta_updates;
  // results
  uint32_t iterations;
  uint32_t converged;
  uint32_t negative_cycle;
  uint32_t phases;
  uint32_t first_unchanged;
  uint32_t done;
  unsigned long long t_start;   // globaltimer at the first barrier (solve budget)
  unsigned long long edges;
  unsigned long long improvements;
  unsigned long long pushes;
};

// Progress record in mapped host memory.  The solve's manager step writes it
// after every finished round / bucket (`rounds` last, with a system-scope
// release); the calling thread polls it while the kernel runs.
struct ProgressBoard {
  uint32_t rounds;
  uint32_t changed;
  unsigned long long t_ns;   // end of the round, ns after the solve's start
};

// ---- asynchronous ADDS worklist (b2_adds.cu) ------------------------------
// Buckets of one window epoch: slot s holds global bucket W + s.  Each slot is
// an append-only queue with its own counters on a 128-byte line.
constexpr int kAddsSlots = 32;
struct alignas(128) AddsSlot {
  unsigned long long claim;   // (epoch << 32) | entries claimed by warps
  uint32_t reserved;          // entries reserved by writers
  uint32_t extra;             // hub chunks spawned by this bucket's entries
  uint32_t done;              // entries and hub chunks finished
  uint32_t pad[27];
};
static_assert(sizeof(AddsSlot) == 128, "slot line");

struct alignas(128) AddsControl {
  // grid barrier (start of the solve only); must stay first
  uint32_t bar_arrive;
  uint32_t bar_gen;
  uint32_t error;
  uint32_t error_site;
  uint32_t pad0[28];
  AddsSlot slot[kAddsSlots];
  // window epoch: written by the one warp that prepares a split while every
  // other warp waits; `epoch` is written last
  uint32_t state_unused;
  uint32_t epoch;
  uint32_t head_unused;
  uint32_t W;                 // global number of slot 0's bucket
  uint32_t kbase;             // distance key at which slot 0 starts
  uint32_t dq;                // bucket width (uint32 graphs)
  uint32_t dinv;              // float bits of 1 / width (float graphs)
  uint32_t far_sel;           // far pile receiving pushes past the window
  uint32_t far_count[2];
  uint32_t far_min_key;       // smallest key pushed into the far pile this epoch
  uint32_t active;            // buckets from head on that warps may take entries from
  uint32_t pad1[20];
  unsigned long long hub_claim;   // hub chunks claimed
  unsigned long long hub_reserved;
  // (epoch << 32) | position: the first bucket of the epoch not yet retired
  // (0 .. kAddsSlots), or an AddsHead mark.  Every change of the window --
  // retiring a bucket, ending the epoch, finishing the solve -- is a
  // compare-and-swap of this one word, so a warp acting on a stale epoch fails.
  unsigned long long head;
  uint32_t pad2[26];
  uint32_t split_cursor;
  uint32_t split_done;
  uint32_t split_total;
  uint32_t trace_n;
  // statistics
  unsigned long long edges;
  unsigned long long improvements;
  unsigned long long pushes;
  unsigned long long entries;     // entries taken from bucket queues
  unsigned long long hub_chunks;
  unsigned long long t_start;
  uint32_t buckets;               // non-empty buckets retired
  uint32_t epochs;
  uint32_t delta_updates;
  uint32_t max_active;
  unsigned long long epoch_entries;
  uint32_t epoch_buckets;
  uint32_t converged;
};

// Marks in the position half of AddsControl::head.
enum AddsHead : uint32_t {
  kAddsPrep = 0xFFFFFFF0u,    // one warp prepares the next epoch; everyone else waits
  kAddsSplit = 0xFFFFFFF1u,   // every warp routes far-pile entries into the new window
  kAddsDone = 0xFFFFFFF2u,    // no work is left: labels are final
};

// Per-graph solver workspace, sized for n vertices (allocated on first use).
struct Workspace {
  size_t n = 0;
  bool pred = false;
  void* dist_a = nullptr;     // 4n or 8n bytes
  void* dist_b = nullptr;     // BF second buffer
  uint32_t* pstamp = nullptr; // near-queue dedup stamps
  uint32_t* bstamp = nullptr; // min bucket pushed (delta)
  uint32_t* farflag = nullptr;
  uint32_t* hstamp = nullptr; // heavy-round member stamps
  uint32_t* lightcnt = nullptr; // per vertex: edges with weight <= delta (sorted prefix)
  uint32_t light_key_valid = 0;
  uint32_t light_key = 0;     // delta (uint32) or its float bits the counts were built for
  uint32_t* in_lightcnt = nullptr;  // the same for the incoming rows (pull heavy pass)
  uint32_t in_light_key_valid = 0;
  uint32_t in_light_key = 0;
  TraceEntry* trace = nullptr;
  uint32_t trace_n = 0;       // entries recorded by the last traced solve
  uint32_t* queues = nullptr; // (5 + kRing) * n ids
  HubEntry* hubs = nullptr;   // 2 * hub_cap
  size_t hub_cap = 0;
  Control* ctl = nullptr;
  Control* h_ctl = nullptr;   // pinned mirror for the result read-back
  unsigned long long* reach = nullptr;   // [reached vertices, their out-edges] of the last solve
  uint32_t phase_epoch = 0;
  size_t bytes = 0;
  ProgressBoard* board_h = nullptr;  // mapped pinned progress record (first solve with a callback)
  ProgressBoard* board_d = nullptr;  // its device address
  // ADDS worklist (allocated on the first b2_sssp_adds solve)
  void* adds_q = nullptr;           // kAddsSlots rings of adds_cap 64-bit words, then 2 far piles of adds_cap u32
  size_t adds_cap = 0;
  void* adds_hub = nullptr;         // ring of 16-byte hub-chunk slots {position tag, entry}
  size_t adds_hub_cap = 0;
  uint32_t* adds_qb = nullptr;      // per vertex: global bucket it is queued in (unprocessed), else ~0
  AddsControl* adds_ctl = nullptr;
  AddsControl* adds_h_ctl = nullptr;
  bool adds_dirty = true;           // queue entries must be reset to empty before the next solve
};

}  // namespace b2

struct b2_graph_s {
  int64_t n = 0;
  int64_t m = 0;
  int32_t weight_type = B2_W_U32;
  int device = 0;
  uint64_t* rowptr = nullptr;   // outgoing, n + 1
  uint2* edges = nullptr;       // (dst, weight bits), m
  uint32_t* in_rowptr32 = nullptr;  // reserved
  uint64_t* in_rowptr = nullptr;    // incoming CSR (internal ids), rows sorted by weight; built on
  uint2* in_edges = nullptr;        // first use by a solve that may pull its heavy pass
  double mean_weight = 1.0;     // over weights > 0
  double mean_degree = 0.0;
  int32_t max_degree = 0;
  bool has_negative = false;
  bool rows_sorted = false;     // each adjacency list ordered by weight
  // Degree order: internal vertex id i is the input vertex perm[i] (ids
  // sorted by out-degree, descending); null when ids are the input's.
  uint32_t* perm = nullptr;     // device, internal -> input id
  uint32_t* inv = nullptr;      // device, input -> internal id
  std::vector<uint32_t> inv_host;   // host copy of inv (source ids of solves and queries)
  size_t graph_bytes = 0;
  float features[24] = {};      // schedule-policy features (computed on first use)
  bool features_valid = false;
  uint64_t pol_version = 0;     // policy decision cache: valid when equal to the
  double pol_mult = 1.0;        // active policy's version
  uint32_t pol_fusion = 0;      // bucket-fusion threshold (0: off)
  float pol_pull = 8.0f;        // push/pull switch point (0: push only)
  bool pol_outside = false;     // the graph's features lie outside the training range: fixed schedule
  b2::Workspace ws;
  std::mutex mu;   // one solve at a time per handle
};

namespace b2 {
b2_status ensure_workspace(b2_graph g, bool pred);
void free_adds_workspace(Workspace& w);
// Asynchronous ADDS worklist solve (b2_adds.cu).
b2_status run_adds(b2_graph g, uint32_t source, void* d_dist, int32_t* d_pred, const b2_sssp_opts* o,
                   cudaStream_t st, b2_stats* stats);
// Live progress: prepare the board before a launch (null when no callback),
// then poll it until `done` has completed, calling o.progress for each new
// round in order; finish_progress reports what the kernel published last.
b2_status progress_begin(b2_graph g, const b2_sssp_opts& o, ProgressBoard** board_d);
void progress_poll(b2_graph g, const b2_sssp_opts& o, cudaEvent_t done, int32_t max_iters, uint32_t* reported);
void progress_finish(b2_graph g, const b2_sssp_opts& o, int32_t max_iters, uint32_t final_rounds, int32_t last_changed,
                     uint32_t* reported);
// stats->reached / reached_edges from a solve's labels (keys, or key|pred words when pred).
b2_status collect_reach(b2_graph g, const void* labels, bool pred, bool isf, cudaStream_t st, b2_stats* stats);
b2_status ensure_incoming(b2_graph g, cudaStream_t st);
// Internal id of input vertex `v` (identity unless the graph is in degree order).
inline uint32_t internal_id(b2_graph g, uint32_t v) { return g->inv_host.empty() ? v : g->inv_host[v]; }
// Learned schedule: delta multiplier (x Near-Far delta), bucket-fusion
// threshold (0: off) and push/pull switch point (pull_fraction; 0: push only)
// for g.  B2_NOT_SUPPORTED when no policy is active.
b2_status policy_decide(b2_graph g, double* delta_mult, uint32_t* fusion_threshold, float* pull_fraction);
b2_status graph_from_device_outgoing(int64_t n, int64_t m, const uint64_t* rowptr, const uint2* edges,
                                     int weight_type, b2_graph* out);
}  // namespace b2
