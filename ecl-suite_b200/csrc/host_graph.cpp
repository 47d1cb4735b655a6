// ECLgraph file I/O, host-side CSR validation and seeded synthetic generators.
//
// File format (library/ECLgraph.h:41-102): little-endian int32 nodes, int32
// edges, int32 nindex[nodes+1], int32 nlist[edges], then optionally int32
// eweight[edges].  A file that ends after nlist has no weights.  No magic,
// no version.  The same byte layout is read and written here; errors become
// status codes instead of exit(-1).
//
// Generators draw every random number from a counter-based hash of
// (seed, stream, index), so the graph is identical for any OpenMP thread count.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <omp.h>

#include "ecl_b200.h"
#include "host_util.h"

namespace {

using ecl::host::mix64;
using ecl::host::unit_double;

// Pair-symmetric weight in [1, wmax): keyed on the unordered pair.
inline int32_t pair_weight(uint64_t wseed, int32_t u, int32_t v, int32_t wmax) {
  const uint32_t lo = (uint32_t)std::min(u, v), hi = (uint32_t)std::max(u, v);
  const uint64_t h = mix64(mix64(wseed ^ 0x6a09e667f3bcc909ull) ^ (((uint64_t)lo << 32) | hi));
  return 1 + (int32_t)(h % (uint64_t)(wmax - 1));
}

// Builds a sorted, duplicate-free, self-loop-free CSR from a list of directed
// (src, dst) pairs.  The pair order in `src`/`dst` does not matter.
ecl_status build_csr(int32_t n, const std::vector<int32_t>& src, const std::vector<int32_t>& dst, ecl_graph* out) {
  const int64_t m_in = (int64_t)src.size();
  std::vector<int64_t> cnt((size_t)n + 1, 0);
  {
    std::atomic<int64_t>* acnt = reinterpret_cast<std::atomic<int64_t>*>(cnt.data());
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m_in; e++) {
      if (src[e] != dst[e]) acnt[src[e]].fetch_add(1, std::memory_order_relaxed);
    }
  }
  std::vector<int64_t> off((size_t)n + 1, 0);
  for (int32_t v = 0; v < n; v++) off[v + 1] = off[v] + cnt[v];
  const int64_t total = off[n];
  std::vector<int32_t> adj((size_t)std::max<int64_t>(total, 1));
  {
    std::vector<int64_t> pos(off.begin(), off.end() - 1);
    std::atomic<int64_t>* apos = reinterpret_cast<std::atomic<int64_t>*>(pos.data());
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m_in; e++) {
      if (src[e] != dst[e]) adj[apos[src[e]].fetch_add(1, std::memory_order_relaxed)] = dst[e];
    }
  }
  std::vector<int32_t> deg((size_t)n);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < n; v++) {
    int32_t* b = adj.data() + off[v];
    int32_t* e = adj.data() + off[v + 1];
    std::sort(b, e);
    deg[v] = (int32_t)(std::unique(b, e) - b);
  }
  int64_t m = 0;
  for (int32_t v = 0; v < n; v++) m += deg[v];
  if (m > INT32_MAX) return ECL_ERR_UNSUPPORTED;
  out->nodes = n;
  out->edges = (int32_t)m;
  out->nindex = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  out->nlist = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  out->eweight = nullptr;
  if (!out->nindex || !out->nlist) return ECL_ERR_OOM;
  out->nindex[0] = 0;
  for (int32_t v = 0; v < n; v++) out->nindex[v + 1] = out->nindex[v] + deg[v];
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < n; v++) {
    memcpy(out->nlist + out->nindex[v], adj.data() + off[v], sizeof(int32_t) * (size_t)deg[v]);
  }
  return ECL_OK;
}

ecl_status attach_pair_weights(ecl_graph* g, uint64_t wseed, int32_t wmax) {
  if (wseed == 0) return ECL_OK;
  if (wmax < 2) return ECL_ERR_INVALID_ARG;
  g->eweight = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max(g->edges, 1));
  if (!g->eweight) return ECL_ERR_OOM;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < g->nodes; v++) {
    for (int32_t i = g->nindex[v]; i < g->nindex[v + 1]; i++) g->eweight[i] = pair_weight(wseed, v, g->nlist[i], wmax);
  }
  return ECL_OK;
}

}  // namespace

extern "C" {

ecl_status ecl_graph_read(const char* path, ecl_graph* out) {
  if (!path || !out) return ECL_ERR_INVALID_ARG;
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "rb");
  if (!f) return ECL_ERR_IO;
  int32_t hdr[2];
  if (fread(hdr, sizeof(int32_t), 2, f) != 2) {
    fclose(f);
    return ECL_ERR_IO;
  }
  // Same lower bounds as readECLgraph (ECLgraph.h:57).
  if (hdr[0] < 1 || hdr[1] < 0) {
    fclose(f);
    return ECL_ERR_BAD_GRAPH;
  }
  out->nodes = hdr[0];
  out->edges = hdr[1];
  out->nindex = (int32_t*)malloc(sizeof(int32_t) * ((size_t)out->nodes + 1));
  out->nlist = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max(out->edges, 1));
  out->eweight = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max(out->edges, 1));
  if (!out->nindex || !out->nlist || !out->eweight) {
    fclose(f);
    ecl_graph_free(out);
    return ECL_ERR_OOM;
  }
  ecl_status st = ECL_OK;
  if (fread(out->nindex, sizeof(int32_t), (size_t)out->nodes + 1, f) != (size_t)out->nodes + 1) st = ECL_ERR_IO;
  if (st == ECL_OK && fread(out->nlist, sizeof(int32_t), (size_t)out->edges, f) != (size_t)out->edges) st = ECL_ERR_IO;
  if (st == ECL_OK) {
    // Weights are optional: zero entries read means "no weights"; a partial
    // block is an error (ECLgraph.h:66-72).
    const size_t cnt = out->edges ? fread(out->eweight, sizeof(int32_t), (size_t)out->edges, f) : 0;
    if (cnt == 0) {
      free(out->eweight);
      out->eweight = nullptr;
    } else if (cnt != (size_t)out->edges) {
      st = ECL_ERR_IO;
    }
  }
  fclose(f);
  if (st != ECL_OK) ecl_graph_free(out);
  return st;
}

ecl_status ecl_graph_write(const char* path, const ecl_graph* g) {
  if (!path || !g) return ECL_ERR_INVALID_ARG;
  if (g->nodes < 1 || g->edges < 0) return ECL_ERR_BAD_GRAPH;  // ECLgraph.h:80
  FILE* f = fopen(path, "wb");
  if (!f) return ECL_ERR_IO;
  bool ok = fwrite(&g->nodes, sizeof(int32_t), 1, f) == 1 && fwrite(&g->edges, sizeof(int32_t), 1, f) == 1 &&
            fwrite(g->nindex, sizeof(int32_t), (size_t)g->nodes + 1, f) == (size_t)g->nodes + 1 &&
            fwrite(g->nlist, sizeof(int32_t), (size_t)g->edges, f) == (size_t)g->edges;
  if (ok && g->eweight) ok = fwrite(g->eweight, sizeof(int32_t), (size_t)g->edges, f) == (size_t)g->edges;
  ok = (fclose(f) == 0) && ok;
  return ok ? ECL_OK : ECL_ERR_IO;
}

void ecl_graph_free(ecl_graph* g) {
  if (!g) return;
  free(g->nindex);
  free(g->nlist);
  free(g->eweight);
  g->nindex = g->nlist = g->eweight = nullptr;
}

ecl_status ecl_graph_validate(const ecl_graph_view* g, int32_t require_symmetric, int32_t forbid_self_loops) {
  if (!g) return ECL_ERR_INVALID_ARG;
  if (g->location != ECL_HOST) return ECL_ERR_INVALID_ARG;
  if (g->nodes < 1 || g->edges < 0) return ECL_ERR_BAD_GRAPH;
  if (!g->nindex || (g->edges > 0 && !g->nlist)) return ECL_ERR_INVALID_ARG;
  const int32_t n = g->nodes;
  if (g->nindex[0] != 0 || g->nindex[n] != g->edges) return ECL_ERR_BAD_GRAPH;
  int bad = 0;
  int unsorted = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : bad, unsorted)
  for (int32_t v = 0; v < n; v++) {
    const int32_t b = g->nindex[v], e = g->nindex[v + 1];
    if (e < b) {
      bad |= 1;
      continue;
    }
    int32_t prev = INT32_MIN;
    for (int32_t i = b; i < e; i++) {
      const int32_t u = g->nlist[i];
      if (u < 0 || u >= n) bad |= 1;
      if (forbid_self_loops && u == v) bad |= 1;
      if (u < prev) unsorted |= 1;
      prev = u;
    }
  }
  if (bad) return ECL_ERR_BAD_GRAPH;
  if (!require_symmetric) return ECL_OK;
  if (!unsorted) {
    // Sorted lists: binary-search the reverse entry of every edge, counting
    // multiplicities so that duplicated entries must be mirrored as often.
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : bad)
    for (int32_t v = 0; v < n; v++) {
      const int32_t b = g->nindex[v], e = g->nindex[v + 1];
      for (int32_t i = b; i < e && !bad; i++) {
        const int32_t u = g->nlist[i];
        const int32_t* ub = g->nlist + g->nindex[u];
        const int32_t* ue = g->nlist + g->nindex[u + 1];
        const auto rng = std::equal_range(ub, ue, v);
        const auto fwd = std::equal_range(g->nlist + b, g->nlist + e, u);
        if ((rng.second - rng.first) != (fwd.second - fwd.first)) bad |= 1;
      }
    }
    return bad ? ECL_ERR_BAD_GRAPH : ECL_OK;
  }
  // Unsorted lists: compare the sorted edge multiset with its transpose.
  std::vector<uint64_t> fwd((size_t)g->edges), rev((size_t)g->edges);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int32_t v = 0; v < n; v++) {
    for (int32_t i = g->nindex[v]; i < g->nindex[v + 1]; i++) {
      const uint64_t u = (uint32_t)g->nlist[i];
      fwd[i] = ((uint64_t)(uint32_t)v << 32) | u;
      rev[i] = (u << 32) | (uint32_t)v;
    }
  }
  std::sort(fwd.begin(), fwd.end());
  std::sort(rev.begin(), rev.end());
  return fwd == rev ? ECL_OK : ECL_ERR_BAD_GRAPH;
}

ecl_status ecl_graph_from_mm(const char* path, int32_t symmetrise, ecl_graph* out) {
  if (!path || !out) return ECL_ERR_INVALID_ARG;
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "rt");
  if (!f) return ECL_ERR_IO;
  char line[1024];
  if (!fgets(line, sizeof(line), f)) {
    fclose(f);
    return ECL_ERR_IO;
  }
  // banner checks of scripts/mm2ecl_real.cpp:63-72
  if (!strstr(line, "%%MatrixMarket") || !strstr(line, "matrix") || !strstr(line, "coordinate") ||
      (!strstr(line, "general") && !strstr(line, "symmetric")) ||
      (!strstr(line, "integer") && !strstr(line, "pattern") && !strstr(line, "real"))) {
    fclose(f);
    return ECL_ERR_BAD_GRAPH;
  }
  const bool intw = strstr(line, "integer") != nullptr, realw = strstr(line, "real") != nullptr;
  bool got = false;
  while (fgets(line, sizeof(line), f)) {
    if (line[0] != '%') {
      got = true;
      break;
    }
  }
  int nodes = 0, cols = 0;
  long long nnz = -1;
  if (!got || sscanf(line, "%d %d %lld", &nodes, &cols, &nnz) != 3 || nodes < 1 || nnz < 0 || nodes != cols ||
      nnz > INT32_MAX) {
    fclose(f);
    return ECL_ERR_BAD_GRAPH;
  }
  struct Entry {
    int s, d;
    double w;
    bool operator<(const Entry& o) const { return s != o.s ? s < o.s : (d != o.d ? d < o.d : w < o.w); }
  };
  std::vector<Entry> e;
  e.reserve((size_t)nnz * (symmetrise ? 2 : 1));
  for (long long k = 0; k < nnz; k++) {
    int s_ = 0, d_ = 0;
    double w = 0;
    const int want = (intw || realw) ? 3 : 2;
    const int got_ = (want == 3) ? fscanf(f, "%d %d %lf", &s_, &d_, &w) : fscanf(f, "%d %d", &s_, &d_);
    if (got_ != want || s_ < 1 || s_ > nodes || d_ < 1 || d_ > nodes) {
      fclose(f);
      return ECL_ERR_BAD_GRAPH;
    }
    e.push_back(Entry{s_ - 1, d_ - 1, w});
    if (symmetrise && s_ != d_) e.push_back(Entry{d_ - 1, s_ - 1, w});
  }
  fclose(f);
  if (e.size() > (size_t)INT32_MAX) return ECL_ERR_UNSUPPORTED;
  std::sort(e.begin(), e.end());
  const int m = (int)e.size();
  out->nodes = nodes;
  out->edges = m;
  out->nindex = (int32_t*)calloc((size_t)nodes + 1, sizeof(int32_t));
  out->nlist = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max(m, 1));
  if (intw || realw) out->eweight = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max(m, 1));
  if (!out->nindex || !out->nlist || ((intw || realw) && !out->eweight)) {
    ecl_graph_free(out);
    return ECL_ERR_OOM;
  }
  for (int i = 0; i < m; i++) {
    out->nindex[e[i].s + 1] = i + 1;
    out->nlist[i] = e[i].d;
    if (intw) out->eweight[i] = (int32_t)e[i].w;
    if (realw) out->eweight[i] = (int32_t)(e[i].w * 100);
  }
  for (int i = 1; i <= nodes; i++) out->nindex[i] = std::max(out->nindex[i - 1], out->nindex[i]);  // empty rows
  return ECL_OK;
}

ecl_status ecl_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                        int32_t symmetrise, uint64_t weight_seed, int32_t weight_max, ecl_graph* out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1) return ECL_ERR_INVALID_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return ECL_ERR_INVALID_ARG;
  memset(out, 0, sizeof(*out));
  const int32_t n = (int32_t)1 << scale;
  const int64_t samples = (int64_t)edge_factor * n;
  const int64_t stored = symmetrise ? 2 * samples : samples;
  if (stored > (int64_t)INT32_MAX * 2) return ECL_ERR_UNSUPPORTED;
  std::vector<int32_t> src((size_t)stored), dst((size_t)stored);
  const double ab = a + b, abc = a + b + c;
  const uint64_t base = mix64(seed ^ 0x243f6a8885a308d3ull);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < samples; e++) {
    uint64_t h = mix64(base + (uint64_t)e * 0x9e3779b97f4a7c15ull);
    int32_t s = 0, d = 0;
    for (int32_t l = 0; l < scale; l++) {
      h = mix64(h + (uint64_t)l + 1);
      const double u = unit_double(h);
      const int32_t bit = 1 << (scale - 1 - l);
      if (u < a) {
      } else if (u < ab) {
        d |= bit;
      } else if (u < abc) {
        s |= bit;
      } else {
        s |= bit;
        d |= bit;
      }
    }
    src[e] = s;
    dst[e] = d;
    if (symmetrise) {
      src[samples + e] = d;
      dst[samples + e] = s;
    }
  }
  ecl_status st = build_csr(n, src, dst, out);
  if (st == ECL_OK) st = attach_pair_weights(out, weight_seed, weight_max);
  if (st != ECL_OK) ecl_graph_free(out);
  return st;
}

ecl_status ecl_gen_grid(int32_t rows, int32_t cols, double delete_frac, uint64_t seed, uint64_t weight_seed,
                        int32_t weight_max, ecl_graph* out) {
  if (!out || rows < 1 || cols < 1 || delete_frac < 0 || delete_frac > 1) return ECL_ERR_INVALID_ARG;
  if ((int64_t)rows * cols > INT32_MAX) return ECL_ERR_UNSUPPORTED;
  memset(out, 0, sizeof(*out));
  const int32_t n = rows * cols;
  const int64_t hcount = (int64_t)rows * (cols - 1);
  const uint64_t base = mix64(seed ^ 0x13198a2e03707344ull);
  // Undirected edge ids: horizontal (r,c)-(r,c+1) -> r*(cols-1)+c;
  // vertical (r,c)-(r+1,c) -> hcount + r*cols + c.
  auto kept = [&](int64_t id) { return unit_double(mix64(base + (uint64_t)id)) >= delete_frac; };
  std::vector<int32_t> deg((size_t)n, 0);
#pragma omp parallel for schedule(static)
  for (int32_t v = 0; v < n; v++) {
    const int32_t r = v / cols, c = v % cols;
    int32_t d = 0;
    if (r > 0 && kept(hcount + (int64_t)(r - 1) * cols + c)) d++;
    if (c > 0 && kept((int64_t)r * (cols - 1) + c - 1)) d++;
    if (c + 1 < cols && kept((int64_t)r * (cols - 1) + c)) d++;
    if (r + 1 < rows && kept(hcount + (int64_t)r * cols + c)) d++;
    deg[v] = d;
  }
  int64_t m = 0;
  for (int32_t v = 0; v < n; v++) m += deg[v];
  if (m > INT32_MAX) return ECL_ERR_UNSUPPORTED;
  out->nodes = n;
  out->edges = (int32_t)m;
  out->nindex = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  out->nlist = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  if (!out->nindex || !out->nlist) {
    ecl_graph_free(out);
    return ECL_ERR_OOM;
  }
  out->nindex[0] = 0;
  for (int32_t v = 0; v < n; v++) out->nindex[v + 1] = out->nindex[v] + deg[v];
#pragma omp parallel for schedule(static)
  for (int32_t v = 0; v < n; v++) {
    const int32_t r = v / cols, c = v % cols;
    int32_t* p = out->nlist + out->nindex[v];
    // Ascending neighbour order: up, left, right, down.
    if (r > 0 && kept(hcount + (int64_t)(r - 1) * cols + c)) *p++ = v - cols;
    if (c > 0 && kept((int64_t)r * (cols - 1) + c - 1)) *p++ = v - 1;
    if (c + 1 < cols && kept((int64_t)r * (cols - 1) + c)) *p++ = v + 1;
    if (r + 1 < rows && kept(hcount + (int64_t)r * cols + c)) *p++ = v + cols;
  }
  ecl_status st = attach_pair_weights(out, weight_seed, weight_max);
  if (st != ECL_OK) ecl_graph_free(out);
  return st;
}

ecl_status ecl_gen_er(int32_t n, double p, uint64_t seed, int32_t symmetrise, uint64_t weight_seed, int32_t weight_min,
                      int32_t weight_max, ecl_graph* out) {
  if (!out || n < 1 || p < 0 || p > 1) return ECL_ERR_INVALID_ARG;
  if (weight_seed != 0 && weight_max < weight_min) return ECL_ERR_INVALID_ARG;
  memset(out, 0, sizeof(*out));
  const uint64_t base = mix64(seed ^ 0xa4093822299f31d0ull);
  // Row i samples its candidate columns by geometric skipping; row i draws
  // from its own stream, so rows are independent of the thread schedule.
  // symmetrise=0: candidates are all j != i; symmetrise=1: j > i only.
  std::vector<std::vector<int32_t>> rows((size_t)n);
  const double lq = (p < 1.0) ? std::log1p(-p) : 0.0;
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < n; i++) {
    if (p <= 0.0) continue;
    uint64_t h = mix64(base + (uint64_t)i * 0x9e3779b97f4a7c15ull);
    int64_t j = symmetrise ? (int64_t)i + 1 : 0;
    std::vector<int32_t>& r = rows[i];
    while (true) {
      if (p < 1.0) {
        h = mix64(h + 1);
        const double u = 1.0 - unit_double(h);  // (0, 1]
        j += (int64_t)std::floor(std::log(u) / lq);
      }
      if (j >= n) break;
      if (j != i) r.push_back((int32_t)j);
      j++;
    }
  }
  std::vector<int32_t> src, dst;
  size_t total = 0;
  for (int32_t i = 0; i < n; i++) total += rows[i].size();
  src.reserve(symmetrise ? 2 * total : total);
  dst.reserve(symmetrise ? 2 * total : total);
  for (int32_t i = 0; i < n; i++) {
    for (int32_t j : rows[i]) {
      src.push_back(i);
      dst.push_back(j);
      if (symmetrise) {
        src.push_back(j);
        dst.push_back(i);
      }
    }
  }
  rows.clear();
  ecl_status st = build_csr(n, src, dst, out);
  if (st == ECL_OK && weight_seed != 0) {
    out->eweight = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max(out->edges, 1));
    if (!out->eweight) st = ECL_ERR_OOM;
    if (st == ECL_OK) {
      const uint64_t span = (uint64_t)((int64_t)weight_max - weight_min + 1);
      const uint64_t ws = mix64(weight_seed ^ 0x082efa98ec4e6c89ull);
#pragma omp parallel for schedule(dynamic, 1024)
      for (int32_t v = 0; v < out->nodes; v++) {
        for (int32_t k = out->nindex[v]; k < out->nindex[v + 1]; k++) {
          const int32_t u = out->nlist[k];
          uint64_t key;
          if (symmetrise) {
            key = ((uint64_t)(uint32_t)std::min(u, v) << 32) | (uint32_t)std::max(u, v);
          } else {
            key = ((uint64_t)(uint32_t)v << 32) | (uint32_t)u;
          }
          out->eweight[k] = weight_min + (int32_t)(mix64(ws ^ key) % span);
        }
      }
    }
  }
  if (st != ECL_OK) ecl_graph_free(out);
  return st;
}

}  // extern "C"
