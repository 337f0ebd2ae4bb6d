// Deterministic synthetic graphs (host memory) and the RIPSCSR1 file format.
//
// Random numbers come from a counter-based hash (the splitmix64 finalizer of
// Steele, Lea and Flood applied to seed, stream and index), so every edge is a
// pure function of (seed, index): results do not depend on the thread count,
// and a numpy restatement can reproduce small cases bit for bit.
//
// All generators return OUTGOING CSR with columns sorted within each row, no
// self-loops and no duplicate arcs.
//   ER   : arcs drawn as (u, v) uniform pairs, u != v, first m distinct kept;
//          weight U{wmin..wmax}; float weight w / (wmax + 1).
//   RMAT : scale, edge factor, (a, b, c, d) quadrant recursion with 32-bit
//          thresholds per level, vertex ids scrambled by an odd affine map
//          mod 2^scale, symmetrised, deduplicated; one weight per undirected
//          pair, U{wmin..wmax}; float weight w / (wmax + 1).
//   Grid : rows x cols 4-neighbour bidirectional lattice plus
//          round(frac * lattice_arcs) random long-range pairs added in both
//          directions; every arc weight ceil(exp(mu + sigma * z)), z standard
//          normal by Box-Muller; float weight w / (max_w + 1).
// RIPSCSR1 layout follows the reference converter
// (HIP_kernel/bellman_ford/src/gr_to_csr.cpp:34-57): magic, 10 uint64 header
// words, int64 rowptr, int32 colind, float values, incoming orientation.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/b200sssp.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + i);
}
inline uint32_t bounded(uint32_t r32, uint64_t range) { return (uint32_t)(((uint64_t)r32 * range) >> 32); }

int n_threads() {
  unsigned h = std::thread::hardware_concurrency();
  if (const char* e = std::getenv("B2_GEN_THREADS")) h = (unsigned)std::max(1, atoi(e));
  return (int)std::max(1u, std::min(h, 64u));
}

template <typename F>
void parallel_for(int64_t n, F&& f) {
  const int T = n_threads();
  if (T == 1 || n < 4096) { f(0, n, 0); return; }
  std::vector<std::thread> th;
  const int64_t chunk = (n + T - 1) / T;
  for (int t = 0; t < T; ++t) {
    const int64_t lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([&, lo, hi, t] { f(lo, hi, t); });
  }
  for (auto& x : th) x.join();
}

bool alloc_csr(b2_host_csr* g, int64_t n, int64_t m, bool fw) {
  memset(g, 0, sizeof(*g));
  g->n = n;
  g->m = m;
  g->rowptr = (int64_t*)malloc((size_t)(n + 1) * 8);
  g->colind = (int32_t*)malloc(std::max<size_t>((size_t)m, 1) * 4);
  g->weights = (uint32_t*)malloc(std::max<size_t>((size_t)m, 1) * 4);
  g->fweights = fw ? (float*)malloc(std::max<size_t>((size_t)m, 1) * 4) : nullptr;
  return g->rowptr && g->colind && g->weights && (!fw || g->fweights);
}

// Build CSR from arcs given as (src, dst) pairs in `keys` (src << 32 | dst):
// counting sort by source, per-row sort, dedup.  Weights assigned afterwards.
b2_status csr_from_arcs(int64_t n, std::vector<uint64_t>& keys, b2_host_csr* g) {
  std::vector<std::atomic<uint32_t>> deg((size_t)n);
  for (auto& d : deg) d.store(0, std::memory_order_relaxed);
  parallel_for((int64_t)keys.size(), [&](int64_t lo, int64_t hi, int) {
    for (int64_t i = lo; i < hi; ++i) deg[keys[i] >> 32].fetch_add(1, std::memory_order_relaxed);
  });
  std::vector<int64_t> start((size_t)n + 1, 0);
  for (int64_t v = 0; v < n; ++v) start[v + 1] = start[v] + deg[v].load(std::memory_order_relaxed);
  std::vector<std::atomic<int64_t>> cur((size_t)n);
  for (int64_t v = 0; v < n; ++v) cur[v].store(start[v], std::memory_order_relaxed);
  std::vector<uint32_t> dst(keys.size());
  parallel_for((int64_t)keys.size(), [&](int64_t lo, int64_t hi, int) {
    for (int64_t i = lo; i < hi; ++i) {
      const uint64_t k = keys[i];
      dst[cur[k >> 32].fetch_add(1, std::memory_order_relaxed)] = (uint32_t)k;
    }
  });
  std::vector<uint64_t>().swap(keys);
  std::vector<int64_t> kept((size_t)n, 0);
  parallel_for(n, [&](int64_t lo, int64_t hi, int) {
    for (int64_t v = lo; v < hi; ++v) {
      uint32_t* a = dst.data() + start[v];
      uint32_t* b = dst.data() + start[v + 1];
      std::sort(a, b);
      kept[v] = std::unique(a, b) - a;
    }
  });
  int64_t m = 0;
  for (int64_t v = 0; v < n; ++v) m += kept[v];
  if (!alloc_csr(g, n, m, true)) return B2_OUT_OF_MEMORY;
  g->rowptr[0] = 0;
  for (int64_t v = 0; v < n; ++v) g->rowptr[v + 1] = g->rowptr[v] + kept[v];
  parallel_for(n, [&](int64_t lo, int64_t hi, int) {
    for (int64_t v = lo; v < hi; ++v)
      for (int64_t j = 0; j < kept[v]; ++j) g->colind[g->rowptr[v] + j] = (int32_t)dst[start[v] + j];
  });
  return B2_SUCCESS;
}

}  // namespace

extern "C" void b2_host_csr_free(b2_host_csr* g) {
  if (!g) return;
  free(g->rowptr);
  free(g->colind);
  free(g->weights);
  free(g->fweights);
  memset(g, 0, sizeof(*g));
}

extern "C" b2_status b2_gen_er(int64_t n, int64_t m, uint32_t wmin, uint32_t wmax, uint64_t seed,
                               b2_host_csr* out) {
  if (!out || n < 2 || m < 0 || m > n * (n - 1) || wmax < wmin) return B2_INVALID_ARGUMENT;
  if (n >= ((int64_t)1 << 31)) return B2_NOT_SUPPORTED;
  memset(out, 0, sizeof(*out));
  // Candidate i -> (u, v); the first m distinct arcs in candidate order win.
  std::unordered_set<uint64_t> seen;
  seen.reserve((size_t)m * 2 + 16);
  std::vector<uint64_t> keys;
  std::vector<uint64_t> cand_of;   // candidate index of each accepted arc
  keys.reserve((size_t)m);
  cand_of.reserve((size_t)m);
  for (uint64_t i = 0; (int64_t)keys.size() < m; ++i) {
    const uint64_t r = rnd(seed, 1, i);
    const uint32_t u = bounded((uint32_t)(r >> 32), (uint64_t)n);
    const uint32_t v = bounded((uint32_t)r, (uint64_t)n);
    if (u == v) continue;
    const uint64_t k = ((uint64_t)u << 32) | v;
    if (seen.insert(k).second) { keys.push_back(k); cand_of.push_back(i); }
  }
  // weight is a function of the accepted arc's candidate index
  std::unordered_map<uint64_t, uint32_t> wmap;
  wmap.reserve((size_t)m * 2 + 16);
  const uint64_t range = (uint64_t)wmax - wmin + 1;
  for (size_t j = 0; j < keys.size(); ++j)
    wmap[keys[j]] = wmin + bounded((uint32_t)(rnd(seed, 2, cand_of[j]) >> 32), range);
  std::vector<uint64_t> copy = keys;
  b2_status s = csr_from_arcs(n, copy, out);
  if (s != B2_SUCCESS) return s;
  for (int64_t v = 0; v < n; ++v)
    for (int64_t e = out->rowptr[v]; e < out->rowptr[v + 1]; ++e) {
      const uint32_t w = wmap[((uint64_t)v << 32) | (uint32_t)out->colind[e]];
      out->weights[e] = w;
      out->fweights[e] = (float)w / (float)((double)wmax + 1.0);
    }
  return B2_SUCCESS;
}

extern "C" b2_status b2_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                                 uint32_t wmin, uint32_t wmax, uint64_t seed, b2_host_csr* out) {
  if (!out || scale < 2 || scale > 30 || edge_factor < 1 || wmax < wmin) return B2_INVALID_ARGUMENT;
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) return B2_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  const int64_t n = (int64_t)1 << scale;
  const int64_t mg = (int64_t)edge_factor * n;
  const uint64_t ta = (uint64_t)std::floor(a * 4294967296.0);
  const uint64_t tab = (uint64_t)std::floor((a + b) * 4294967296.0);
  const uint64_t tabc = (uint64_t)std::floor((a + b + c) * 4294967296.0);
  const uint64_t mask = (uint64_t)n - 1;
  const uint64_t mulA = (mix64(seed ^ 0x5bd1e995ull) | 1ull) & mask;
  const uint64_t addB = mix64(seed ^ 0x27d4eb2full) & mask;
  auto perm = [&](uint64_t x) { return (x * (mulA ? mulA : 1ull) + addB) & mask; };
  // pass 1: count kept arcs per thread chunk (self-loops dropped), pass 2: fill
  std::vector<uint64_t> keys;
  {
    std::vector<int64_t> per(64, 0);
    auto gen_edge = [&](int64_t i, uint32_t* pu, uint32_t* pv) {
      uint64_t u = 0, v = 0;
      for (int l = 0; l < scale; l += 2) {
        const uint64_t r = rnd(seed, 3, (uint64_t)i * 16 + (uint64_t)(l >> 1));
        for (int h = 0; h < 2 && l + h < scale; ++h) {
          const uint64_t r32 = h == 0 ? (r >> 32) : (r & 0xffffffffull);
          const int bu = r32 >= tab ? 1 : 0;
          const int bv = (r32 >= ta && r32 < tab) || r32 >= tabc ? 1 : 0;
          u = (u << 1) | (uint64_t)bu;
          v = (v << 1) | (uint64_t)bv;
        }
      }
      *pu = (uint32_t)perm(u);
      *pv = (uint32_t)perm(v);
    };
    const int T = n_threads();
    const int64_t chunk = (mg + T - 1) / T;
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
      th.emplace_back([&, t] {
        int64_t cnt = 0;
        for (int64_t i = t * chunk; i < std::min(mg, (t + 1) * chunk); ++i) {
          uint32_t u, v;
          gen_edge(i, &u, &v);
          cnt += (u != v) ? 2 : 0;
        }
        per[t] = cnt;
      });
    for (auto& x : th) x.join();
    th.clear();
    std::vector<int64_t> off(T + 1, 0);
    for (int t = 0; t < T; ++t) off[t + 1] = off[t] + per[t];
    keys.resize((size_t)off[T]);
    for (int t = 0; t < T; ++t)
      th.emplace_back([&, t] {
        int64_t p = off[t];
        for (int64_t i = t * chunk; i < std::min(mg, (t + 1) * chunk); ++i) {
          uint32_t u, v;
          gen_edge(i, &u, &v);
          if (u == v) continue;
          keys[p++] = ((uint64_t)u << 32) | v;
          keys[p++] = ((uint64_t)v << 32) | u;
        }
      });
    for (auto& x : th) x.join();
  }
  b2_status s = csr_from_arcs(n, keys, out);
  if (s != B2_SUCCESS) return s;
  const uint64_t range = (uint64_t)wmax - wmin + 1;
  const float fden = (float)((double)wmax + 1.0);
  parallel_for(n, [&](int64_t lo, int64_t hi, int) {
    for (int64_t u = lo; u < hi; ++u)
      for (int64_t e = out->rowptr[u]; e < out->rowptr[u + 1]; ++e) {
        const uint64_t v = (uint64_t)out->colind[e];
        const uint64_t x = (uint64_t)u < v ? (uint64_t)u : v, y = (uint64_t)u < v ? v : (uint64_t)u;
        const uint32_t w = wmin + bounded((uint32_t)(rnd(seed, 4, (x << 32) | y) >> 32), range);
        out->weights[e] = w;
        out->fweights[e] = (float)w / fden;
      }
  });
  return B2_SUCCESS;
}

extern "C" b2_status b2_gen_grid(int32_t rows, int32_t cols, double shortcut_frac, double mu,
                                 double sigma, uint64_t seed, b2_host_csr* out) {
  if (!out || rows < 1 || cols < 1 || shortcut_frac < 0 || !(sigma >= 0)) return B2_INVALID_ARGUMENT;
  const int64_t n = (int64_t)rows * cols;
  if (n < 2 || n >= ((int64_t)1 << 31)) return B2_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  const int64_t lattice = 2 * ((int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols);
  const int64_t pairs = (int64_t)std::llround(shortcut_frac * (double)lattice);
  std::vector<uint64_t> keys((size_t)(lattice + 2 * pairs));
  parallel_for(n, [&](int64_t lo, int64_t hi, int) {
    for (int64_t v = lo; v < hi; ++v) {
      const int64_t r = v / cols, cc = v % cols;
      // arcs of v in a fixed slot order so the fill is thread-independent
      const int64_t right_base = 0;
      (void)right_base;
      int64_t idx;
      // horizontal arcs: slot 2*(r*(cols-1)+cc) (+0 right, +1 left)
      if (cc + 1 < cols) {
        idx = 2 * (r * (cols - 1) + cc);
        keys[idx] = ((uint64_t)v << 32) | (uint64_t)(v + 1);
        keys[idx + 1] = ((uint64_t)(v + 1) << 32) | (uint64_t)v;
      }
      if (r + 1 < rows) {
        idx = 2 * (int64_t)rows * (cols - 1) + 2 * (r * cols + cc);
        keys[idx] = ((uint64_t)v << 32) | (uint64_t)(v + cols);
        keys[idx + 1] = ((uint64_t)(v + cols) << 32) | (uint64_t)v;
      }
    }
  });
  for (int64_t p = 0; p < pairs; ++p) {
    uint32_t u, v;
    uint64_t k = 0;
    do {
      const uint64_t r = rnd(seed, 5, (uint64_t)p * 1024 + k++);
      u = bounded((uint32_t)(r >> 32), (uint64_t)n);
      v = bounded((uint32_t)r, (uint64_t)n);
    } while (u == v);
    keys[lattice + 2 * p] = ((uint64_t)u << 32) | v;
    keys[lattice + 2 * p + 1] = ((uint64_t)v << 32) | u;
  }
  b2_status s = csr_from_arcs(n, keys, out);
  if (s != B2_SUCCESS) return s;
  std::vector<uint32_t> tmax(64, 0);
  parallel_for(n, [&](int64_t lo, int64_t hi, int t) {
    uint32_t mx = 0;
    for (int64_t u = lo; u < hi; ++u)
      for (int64_t e = out->rowptr[u]; e < out->rowptr[u + 1]; ++e) {
        const uint64_t key = ((uint64_t)u << 32) | (uint32_t)out->colind[e];
        const uint64_t r1 = rnd(seed, 6, key), r2 = rnd(seed, 7, key);
        const double u1 = ((double)(r1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
        const double u2 = (double)(r2 >> 11) * (1.0 / 9007199254740992.0);         // [0, 1)
        const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
        double w = std::ceil(std::exp(mu + sigma * z));
        if (!(w >= 1.0)) w = 1.0;
        if (w > 2147483647.0) w = 2147483647.0;
        out->weights[e] = (uint32_t)w;
        mx = std::max(mx, (uint32_t)w);
      }
    tmax[t] = std::max(tmax[t], mx);
  });
  uint32_t maxw = 0;
  for (uint32_t x : tmax) maxw = std::max(maxw, x);
  const float fden = (float)((double)maxw + 1.0);
  parallel_for(out->m, [&](int64_t lo, int64_t hi, int) {
    for (int64_t e = lo; e < hi; ++e) out->fweights[e] = (float)out->weights[e] / fden;
  });
  return B2_SUCCESS;
}

extern "C" b2_status b2_host_csr_transpose(const b2_host_csr* in, b2_host_csr* out) {
  if (!in || !out || in->n < 1) return B2_INVALID_ARGUMENT;
  const int64_t n = in->n, m = in->m;
  if (!alloc_csr(out, n, m, in->fweights != nullptr)) { b2_host_csr_free(out); return B2_OUT_OF_MEMORY; }
  std::vector<int64_t> cnt((size_t)n + 1, 0);
  for (int64_t e = 0; e < m; ++e) cnt[(size_t)in->colind[e] + 1]++;
  out->rowptr[0] = 0;
  for (int64_t v = 0; v < n; ++v) out->rowptr[v + 1] = out->rowptr[v] + cnt[v + 1];
  std::vector<int64_t> cur(out->rowptr, out->rowptr + n);
  for (int64_t u = 0; u < n; ++u)   // rows visited in order -> stable, sorted columns
    for (int64_t e = in->rowptr[u]; e < in->rowptr[u + 1]; ++e) {
      const int64_t p = cur[in->colind[e]]++;
      out->colind[p] = (int32_t)u;
      out->weights[p] = in->weights ? in->weights[e] : 0u;
      if (in->fweights) out->fweights[p] = in->fweights[e];
    }
  return B2_SUCCESS;
}

// ---- RIPSCSR1 --------------------------------------------------------------
static const char kMagic[8] = {'R', 'I', 'P', 'S', 'C', 'S', 'R', '1'};

extern "C" b2_status b2_csrbin_write(const char* path, int64_t n, int64_t nnz, const int64_t* rowptr,
                                     const int32_t* colind, const float* values) {
  if (!path || n < 0 || nnz < 0 || !rowptr || (nnz && (!colind || !values))) return B2_INVALID_ARGUMENT;
  FILE* f = fopen(path, "wb");
  if (!f) return B2_INVALID_ARGUMENT;
  uint64_t hdr[10] = {1, 1, (uint64_t)n, (uint64_t)n, (uint64_t)nnz, (uint64_t)nnz, (uint64_t)nnz,
                      (uint64_t)n + 1, (uint64_t)nnz, (uint64_t)nnz};
  bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(hdr, 8, 10, f) == 10 &&
            fwrite(rowptr, 8, (size_t)n + 1, f) == (size_t)n + 1 &&
            fwrite(colind, 4, (size_t)nnz, f) == (size_t)nnz && fwrite(values, 4, (size_t)nnz, f) == (size_t)nnz;
  ok = (fclose(f) == 0) && ok;
  return ok ? B2_SUCCESS : B2_INVALID_ARGUMENT;
}

extern "C" b2_status b2_csrbin_read(const char* path, b2_host_csr* out) {
  if (!path || !out) return B2_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "rb");
  if (!f) return B2_INVALID_ARGUMENT;
  char magic[8];
  uint64_t h[10];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kMagic, 8) != 0 || fread(h, 8, 10, f) != 10) {
    fclose(f);
    return B2_INVALID_ARGUMENT;
  }
  // h: version, orientation, rows, cols, declared, loaded, nnz, rowptr_count, colind_count, values_count
  if (h[0] != 1 || h[1] != 1 || h[2] != h[3] || h[7] != h[2] + 1 || h[8] != h[6] || h[9] != h[6] ||
      h[2] >= (1ull << 31)) {
    fclose(f);
    return B2_INVALID_ARGUMENT;
  }
  const int64_t n = (int64_t)h[2], m = (int64_t)h[6];
  if (!alloc_csr(out, n, m, true)) { fclose(f); b2_host_csr_free(out); return B2_OUT_OF_MEMORY; }
  bool ok = fread(out->rowptr, 8, (size_t)n + 1, f) == (size_t)n + 1 &&
            fread(out->colind, 4, (size_t)m, f) == (size_t)m && fread(out->fweights, 4, (size_t)m, f) == (size_t)m;
  fclose(f);
  if (!ok || out->rowptr[0] != 0 || out->rowptr[n] != m) { b2_host_csr_free(out); return B2_INVALID_ARGUMENT; }
  for (int64_t e = 0; e < m; ++e) out->weights[e] = 0u;  // float file: uint32 view unused
  return B2_SUCCESS;
}
