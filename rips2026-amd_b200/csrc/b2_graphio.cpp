// Graph files of the reference's drivers, read and written on the host.
//
// DIMACS shortest-path text (.gr): "c" comment lines, one "p <kind> n m"
// problem line, "a u v w" arc lines with 1-based ids.  Read as an INCOMING
// CSR with float weights under the rules of the reference's converter
// (HIP_kernel/bellman_ford/src/gr_to_csr.cpp:124-230): trailing CR/LF are
// stripped, empty and "c" lines skipped, lines of any other kind ignored; a
// problem line needs n in [1, 2^31 - 1] and m >= 0 and starts the graph over
// (the count of arc lines read keeps running); an arc line needs a problem
// line before it, endpoints in [1, n] and a finite weight (stored as float);
// each row lists its columns in increasing order, arcs repeated between the
// same pair are reduced to their smallest weight, self-loops stay.
// b2_dimacs_to_csrbin writes the converter's RIPSCSR1 file (declared arcs =
// the problem line's m, loaded arcs = arc lines read) byte for byte.
//
// Galois / Lonestar binary .gr, version 1, the input of the ADDS port
// (HIP_kernel/faster_GPU_algo/Charlotte_ADS_Float_Attempt/csr_graph.cpp:153-291):
// little-endian uint64 {version = 1, edge data bytes (0 or 4), n, m}, uint64
// row END offsets [n], uint32 destinations [m], 4 bytes of padding when m is
// odd, then the edge data [m].  Read as an OUTGOING CSR; no edge data means
// weight 1; 4-byte data are floats (the port's reading) or uint32.  The port's
// checks apply: n in [1, 2^31 - 1], m < 2^31, offsets monotone and ending at
// m, destinations < n, float weights finite and non-negative.
#include <algorithm>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "b200sssp.h"

namespace {

struct InArc {
  int32_t row;   // head (incoming row)
  int32_t col;   // tail
  float w;
};

bool alloc_host(b2_host_csr* g, int64_t n, int64_t m) {
  memset(g, 0, sizeof(*g));
  g->n = n;
  g->m = m;
  const size_t mm = std::max<size_t>((size_t)m, 1);
  g->rowptr = (int64_t*)malloc((size_t)(n + 1) * 8);
  g->colind = (int32_t*)malloc(mm * 4);
  g->weights = (uint32_t*)malloc(mm * 4);
  g->fweights = (float*)malloc(mm * 4);
  return g->rowptr && g->colind && g->weights && g->fweights;
}

struct Dimacs {
  int64_t n = 0;
  int64_t declared = 0;
  int64_t loaded = 0;
  std::vector<InArc> arcs;
};

b2_status parse_dimacs(const char* path, Dimacs& d) {
  FILE* f = fopen(path, "r");
  if (!f) return B2_INVALID_ARGUMENT;
  char* line = nullptr;
  size_t cap = 0;
  ssize_t len;
  b2_status st = B2_SUCCESS;
  bool have_problem = false;
  while (st == B2_SUCCESS && (len = getline(&line, &cap, f)) != -1) {
    while (len > 0 && (line[len - 1] == '\n' || line[len - 1] == '\r')) line[--len] = '\0';
    if (len == 0 || line[0] == 'c') continue;
    if (line[0] == 'p') {
      char kind[32] = {};
      long long n = 0, m = 0;
      if (sscanf(line, "p %31s %lld %lld", kind, &n, &m) != 3 || n <= 0 || n > INT32_MAX || m < 0) {
        st = B2_INVALID_ARGUMENT;
        break;
      }
      d.n = n;
      d.declared = m;
      d.arcs.clear();
      have_problem = true;
    } else if (line[0] == 'a') {
      long long u = 0, v = 0;
      double w = 0.0;
      if (!have_problem || sscanf(line, "a %lld %lld %lf", &u, &v, &w) != 3) {
        st = B2_INVALID_ARGUMENT;
      } else if (u <= 0 || u > d.n || v <= 0 || v > d.n) {
        st = B2_INVALID_INDEX;
      } else if (!std::isfinite(w)) {
        st = B2_INVALID_WEIGHT;
      } else {
        d.arcs.push_back({(int32_t)(v - 1), (int32_t)(u - 1), (float)w});
        ++d.loaded;
      }
    }
  }
  free(line);
  fclose(f);
  if (st == B2_SUCCESS && !have_problem) st = B2_INVALID_ARGUMENT;
  return st;
}

// Incoming CSR from the arcs: counting sort by row, then each row by
// (column, weight); the first arc of every column run is its smallest.
b2_status build_incoming(Dimacs& d, b2_host_csr* out) {
  const int64_t n = d.n;
  std::vector<int64_t> start((size_t)n + 1, 0);
  for (const InArc& a : d.arcs) ++start[(size_t)a.row + 1];
  for (int64_t r = 0; r < n; ++r) start[r + 1] += start[r];
  std::vector<InArc> by_row(d.arcs.size());
  {
    std::vector<int64_t> pos(start.begin(), start.end() - 1);
    for (const InArc& a : d.arcs) by_row[(size_t)pos[a.row]++] = a;
  }
  d.arcs.clear();
  d.arcs.shrink_to_fit();
  int64_t nnz = 0;
  for (int64_t r = 0; r < n; ++r) {
    auto b = by_row.begin() + start[r], e = by_row.begin() + start[r + 1];
    std::sort(b, e, [](const InArc& x, const InArc& y) { return x.col != y.col ? x.col < y.col : x.w < y.w; });
    for (auto it = b; it != e; ++it)
      if (it == b || it->col != (it - 1)->col) ++nnz;
  }
  if (!alloc_host(out, n, nnz)) {
    b2_host_csr_free(out);
    return B2_OUT_OF_MEMORY;
  }
  int64_t k = 0;
  for (int64_t r = 0; r < n; ++r) {
    out->rowptr[r] = k;
    for (int64_t i = start[r]; i < start[r + 1]; ++i) {
      const InArc& a = by_row[(size_t)i];
      if (i > start[r] && a.col == by_row[(size_t)i - 1].col) continue;
      out->colind[k] = a.col;
      out->fweights[k] = a.w;
      out->weights[k] = 0u;   // float file: the uint32 view is unused
      ++k;
    }
  }
  out->rowptr[n] = k;
  return B2_SUCCESS;
}

bool write_all(FILE* f, const void* p, size_t bytes) { return bytes == 0 || fwrite(p, 1, bytes, f) == bytes; }

}  // namespace

extern "C" b2_status b2_dimacs_read(const char* path, b2_host_csr* out, int64_t* declared_arcs,
                                    int64_t* loaded_arcs) {
  if (!path || !out) return B2_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  Dimacs d;
  b2_status st = parse_dimacs(path, d);
  if (st != B2_SUCCESS) return st;
  if (declared_arcs) *declared_arcs = d.declared;
  if (loaded_arcs) *loaded_arcs = d.loaded;
  return build_incoming(d, out);
}

extern "C" b2_status b2_dimacs_to_csrbin(const char* gr_path, const char* csrbin_path, int64_t* nnz_out) {
  if (!gr_path || !csrbin_path) return B2_INVALID_ARGUMENT;
  Dimacs d;
  b2_status st = parse_dimacs(gr_path, d);
  if (st != B2_SUCCESS) return st;
  b2_host_csr g;
  const int64_t declared = d.declared, loaded = d.loaded;
  st = build_incoming(d, &g);
  if (st != B2_SUCCESS) return st;
  FILE* f = fopen(csrbin_path, "wb");
  if (!f) {
    b2_host_csr_free(&g);
    return B2_INVALID_ARGUMENT;
  }
  static const char kMagic[8] = {'R', 'I', 'P', 'S', 'C', 'S', 'R', '1'};
  const uint64_t n = (uint64_t)g.n, nnz = (uint64_t)g.m;
  const uint64_t hdr[10] = {1, 1, n, n, (uint64_t)declared, (uint64_t)loaded, nnz, n + 1, nnz, nnz};
  bool ok = write_all(f, kMagic, 8) && write_all(f, hdr, sizeof(hdr)) && write_all(f, g.rowptr, (n + 1) * 8) &&
            write_all(f, g.colind, nnz * 4) && write_all(f, g.fweights, nnz * 4);
  ok = (fclose(f) == 0) && ok;
  if (nnz_out) *nnz_out = (int64_t)nnz;
  b2_host_csr_free(&g);
  return ok ? B2_SUCCESS : B2_INVALID_ARGUMENT;
}

extern "C" b2_status b2_lonestar_read(const char* path, int32_t data_is_float, b2_host_csr* out) {
  if (!path || !out) return B2_INVALID_ARGUMENT;
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "rb");
  if (!f) return B2_INVALID_ARGUMENT;
  uint64_t h[4];
  b2_status st = B2_SUCCESS;
  if (fread(h, 8, 4, f) != 4 || h[0] != 1 || (h[1] != 0 && h[1] != 4) || h[2] == 0 || h[2] > (uint64_t)INT32_MAX ||
      h[3] > (uint64_t)INT32_MAX) {
    fclose(f);
    return B2_INVALID_ARGUMENT;
  }
  const int64_t n = (int64_t)h[2], m = (int64_t)h[3];
  const bool has_data = h[1] == 4;
  std::vector<uint64_t> ends((size_t)n);
  std::vector<uint32_t> dst((size_t)m), data(has_data ? (size_t)m : 0);
  uint32_t pad = 0;
  bool ok = fread(ends.data(), 8, (size_t)n, f) == (size_t)n && fread(dst.data(), 4, (size_t)m, f) == (size_t)m &&
            ((m & 1) == 0 || !has_data || fread(&pad, 4, 1, f) == 1) &&
            (!has_data || fread(data.data(), 4, (size_t)m, f) == (size_t)m);
  fclose(f);
  if (!ok) return B2_INVALID_ARGUMENT;   // truncated
  if (!alloc_host(out, n, m)) {
    b2_host_csr_free(out);
    return B2_OUT_OF_MEMORY;
  }
  out->rowptr[0] = 0;
  for (int64_t v = 0; v < n && st == B2_SUCCESS; ++v) {
    if (ends[v] > (uint64_t)m || (int64_t)ends[v] < out->rowptr[v]) {
      st = B2_INVALID_ROWPTR;
      break;
    }
    out->rowptr[v + 1] = (int64_t)ends[v];
    for (int64_t e = out->rowptr[v]; e < out->rowptr[v + 1]; ++e) {
      if (dst[e] >= (uint64_t)n) { st = B2_INVALID_INDEX; break; }
      out->colind[e] = (int32_t)dst[e];
      if (!has_data) {
        out->fweights[e] = 1.0f;
        out->weights[e] = 1u;
      } else if (data_is_float) {
        float w;
        memcpy(&w, &data[e], 4);
        if (!std::isfinite(w) || w < 0.0f) { st = B2_INVALID_WEIGHT; break; }
        out->fweights[e] = w;
        out->weights[e] = 0u;   // float file: the uint32 view is unused
      } else {
        out->weights[e] = data[e];
        out->fweights[e] = (float)data[e];
      }
    }
  }
  if (st == B2_SUCCESS && out->rowptr[n] != m) st = B2_INVALID_ROWPTR;
  if (st != B2_SUCCESS) b2_host_csr_free(out);
  return st;
}

extern "C" b2_status b2_lonestar_write(const char* path, const b2_host_csr* g, int32_t data_is_float) {
  if (!path || !g || g->n <= 0 || g->n > INT32_MAX || g->m < 0 || g->m > INT32_MAX || !g->rowptr ||
      (g->m && !g->colind) || (g->m && !(data_is_float ? (const void*)g->fweights : (const void*)g->weights)))
    return B2_INVALID_ARGUMENT;
  const int64_t n = g->n, m = g->m;
  if (g->rowptr[0] != 0 || g->rowptr[n] != m) return B2_INVALID_ROWPTR;
  for (int64_t v = 0; v < n; ++v)
    if (g->rowptr[v + 1] < g->rowptr[v]) return B2_INVALID_ROWPTR;
  for (int64_t e = 0; e < m; ++e)
    if (g->colind[e] < 0 || g->colind[e] >= n) return B2_INVALID_INDEX;
  FILE* f = fopen(path, "wb");
  if (!f) return B2_INVALID_ARGUMENT;
  const uint64_t h[4] = {1, 4, (uint64_t)n, (uint64_t)m};
  bool ok = write_all(f, h, sizeof(h));
  for (int64_t v = 0; v < n && ok; ++v) {
    const uint64_t end = (uint64_t)g->rowptr[v + 1];
    ok = write_all(f, &end, 8);
  }
  for (int64_t e = 0; e < m && ok; ++e) {
    const uint32_t d = (uint32_t)g->colind[e];
    ok = write_all(f, &d, 4);
  }
  const uint32_t pad = 0;
  if (ok && (m & 1)) ok = write_all(f, &pad, 4);
  if (ok) ok = write_all(f, data_is_float ? (const void*)g->fweights : (const void*)g->weights, (size_t)m * 4);
  ok = (fclose(f) == 0) && ok;
  return ok ? B2_SUCCESS : B2_INVALID_ARGUMENT;
}
