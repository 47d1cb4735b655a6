/* Seeded synthetic graph generators -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C restatement of the product's generators (ecl_gen_rmat,
 * ecl_gen_grid, ecl_gen_er), so that the bench's reference arm and the tests
 * can build the benchmark graphs without loading the product library.  The
 * graphs are the same byte for byte; tests/test_oracle.py checks that on
 * every generator and parameter kind.
 *
 * Every random number is a counter-based hash of (seed, stream, index): the
 * SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014) as a bijective
 * mixer and the top 53 bits as a double in [0, 1).  The CSR has sorted,
 * duplicate-free rows and no self-loops.  Weights are keyed on the unordered
 * pair (R-MAT, grid) or on the pair the ER row drew, so symmetric graphs get
 * symmetric weights. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

static uint64_t gen_mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

static double gen_unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

static int32_t gen_pair_weight(uint64_t wseed, int32_t u, int32_t v, int32_t wmax) {
  const uint32_t lo = (uint32_t)(u < v ? u : v), hi = (uint32_t)(u < v ? v : u);
  const uint64_t h = gen_mix64(gen_mix64(wseed ^ 0x6a09e667f3bcc909ull) ^ (((uint64_t)lo << 32) | hi));
  return 1 + (int32_t)(h % (uint64_t)(wmax - 1));
}

static int gen_cmp_int(const void* a, const void* b) {
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

static void gen_sort_row(int32_t* b, int64_t len) {
  if (len < 32) { /* insertion sort: most rows are short */
    for (int64_t i = 1; i < len; i++) {
      const int32_t x = b[i];
      int64_t j = i - 1;
      while (j >= 0 && b[j] > x) {
        b[j + 1] = b[j];
        j--;
      }
      b[j + 1] = x;
    }
  } else {
    qsort(b, (size_t)len, sizeof(int32_t), gen_cmp_int);
  }
}

/* The generated graph; arrays are malloc'ed and released by gen_free. */
typedef struct {
  int32_t nodes, edges;
  int32_t* nindex;
  int32_t* nlist;
  int32_t* eweight;
} gen_graph;

void gen_free(gen_graph* g) {
  free(g->nindex);
  free(g->nlist);
  free(g->eweight);
  memset(g, 0, sizeof(*g));
}

/* CSR with sorted, unique rows from (src, dst) pairs; self-loops dropped. */
static int gen_build_csr(int32_t n, int64_t m_in, const int32_t* src, const int32_t* dst, gen_graph* out) {
  int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  if (!cnt) return 3;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m_in; e++)
    if (src[e] != dst[e]) __atomic_fetch_add(&cnt[src[e]], 1, __ATOMIC_RELAXED);
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * ((size_t)n + 1));
  off[0] = 0;
  for (int32_t v = 0; v < n; v++) off[v + 1] = off[v] + cnt[v];
  const int64_t total = off[n];
  int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  for (int32_t v = 0; v < n; v++) cnt[v] = off[v];
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m_in; e++)
    if (src[e] != dst[e]) adj[__atomic_fetch_add(&cnt[src[e]], 1, __ATOMIC_RELAXED)] = dst[e];
  int32_t* deg = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < n; v++) {
    int32_t* b = adj + off[v];
    const int64_t len = off[v + 1] - off[v];
    gen_sort_row(b, len);
    int64_t k = 0;
    for (int64_t i = 0; i < len; i++)
      if (i == 0 || b[i] != b[i - 1]) b[k++] = b[i];
    deg[v] = (int32_t)k;
  }
  int64_t m = 0;
  for (int32_t v = 0; v < n; v++) m += deg[v];
  if (m > INT32_MAX) {
    free(cnt), free(off), free(adj), free(deg);
    return 7;
  }
  out->nodes = n;
  out->edges = (int32_t)m;
  out->nindex = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  out->nlist = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  out->eweight = NULL;
  out->nindex[0] = 0;
  for (int32_t v = 0; v < n; v++) out->nindex[v + 1] = out->nindex[v] + deg[v];
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < n; v++)
    memcpy(out->nlist + out->nindex[v], adj + off[v], sizeof(int32_t) * (size_t)deg[v]);
  free(cnt), free(off), free(adj), free(deg);
  return 0;
}

static int gen_pair_weights(gen_graph* g, uint64_t wseed, int32_t wmax) {
  if (wseed == 0) return 0;
  if (wmax < 2) return 1;
  g->eweight = (int32_t*)malloc(sizeof(int32_t) * (size_t)(g->edges > 0 ? g->edges : 1));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < g->nodes; v++)
    for (int32_t i = g->nindex[v]; i < g->nindex[v + 1]; i++)
      g->eweight[i] = gen_pair_weight(wseed, v, g->nlist[i], wmax);
  return 0;
}

/* R-MAT: edge_factor * 2^scale samples, each descending `scale` quadrant
 * levels with probabilities (a, b, c, 1 - a - b - c). */
int gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, int32_t symmetrise,
             uint64_t weight_seed, int32_t weight_max, gen_graph* out) {
  memset(out, 0, sizeof(*out));
  if (scale < 1 || scale > 30 || edge_factor < 1) return 1;
  const int32_t n = (int32_t)1 << scale;
  const int64_t samples = (int64_t)edge_factor * n;
  const int64_t stored = symmetrise ? 2 * samples : samples;
  int32_t* src = (int32_t*)malloc(sizeof(int32_t) * (size_t)stored);
  int32_t* dst = (int32_t*)malloc(sizeof(int32_t) * (size_t)stored);
  if (!src || !dst) {
    free(src), free(dst);
    return 3;
  }
  const double ab = a + b, abc = a + b + c;
  const uint64_t base = gen_mix64(seed ^ 0x243f6a8885a308d3ull);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < samples; e++) {
    uint64_t h = gen_mix64(base + (uint64_t)e * 0x9e3779b97f4a7c15ull);
    int32_t s = 0, d = 0;
    for (int32_t l = 0; l < scale; l++) {
      h = gen_mix64(h + (uint64_t)l + 1);
      const double u = gen_unit(h);
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
  int st = gen_build_csr(n, stored, src, dst, out);
  free(src), free(dst);
  if (st == 0) st = gen_pair_weights(out, weight_seed, weight_max);
  if (st) gen_free(out);
  return st;
}

/* rows x cols 4-neighbour grid; each undirected edge is deleted with
 * probability delete_frac (a hash of its id). */
int gen_grid(int32_t rows, int32_t cols, double delete_frac, uint64_t seed, uint64_t weight_seed, int32_t weight_max,
             gen_graph* out) {
  memset(out, 0, sizeof(*out));
  if (rows < 1 || cols < 1 || (int64_t)rows * cols > INT32_MAX) return 1;
  const int32_t n = rows * cols;
  const int64_t hcount = (int64_t)rows * (cols - 1);
  const uint64_t base = gen_mix64(seed ^ 0x13198a2e03707344ull);
#define GEN_KEPT(id) (gen_unit(gen_mix64(base + (uint64_t)(id))) >= delete_frac)
  int32_t* deg = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
#pragma omp parallel for schedule(static)
  for (int32_t v = 0; v < n; v++) {
    const int32_t r = v / cols, c = v % cols;
    int32_t d = 0;
    if (r > 0 && GEN_KEPT(hcount + (int64_t)(r - 1) * cols + c)) d++;
    if (c > 0 && GEN_KEPT((int64_t)r * (cols - 1) + c - 1)) d++;
    if (c + 1 < cols && GEN_KEPT((int64_t)r * (cols - 1) + c)) d++;
    if (r + 1 < rows && GEN_KEPT(hcount + (int64_t)r * cols + c)) d++;
    deg[v] = d;
  }
  int64_t m = 0;
  for (int32_t v = 0; v < n; v++) m += deg[v];
  out->nodes = n;
  out->edges = (int32_t)m;
  out->nindex = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  out->nlist = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  out->nindex[0] = 0;
  for (int32_t v = 0; v < n; v++) out->nindex[v + 1] = out->nindex[v] + deg[v];
  free(deg);
#pragma omp parallel for schedule(static)
  for (int32_t v = 0; v < n; v++) {
    const int32_t r = v / cols, c = v % cols;
    int32_t* p = out->nlist + out->nindex[v];
    if (r > 0 && GEN_KEPT(hcount + (int64_t)(r - 1) * cols + c)) *p++ = v - cols;
    if (c > 0 && GEN_KEPT((int64_t)r * (cols - 1) + c - 1)) *p++ = v - 1;
    if (c + 1 < cols && GEN_KEPT((int64_t)r * (cols - 1) + c)) *p++ = v + 1;
    if (r + 1 < rows && GEN_KEPT(hcount + (int64_t)r * cols + c)) *p++ = v + cols;
  }
#undef GEN_KEPT
  const int st = gen_pair_weights(out, weight_seed, weight_max);
  if (st) gen_free(out);
  return st;
}

/* Erdos-Renyi G(n, p) by geometric skipping over each row's candidate
 * columns (all j != i, or j > i when symmetrising); weights uniform in
 * [weight_min, weight_max]. */
int gen_er(int32_t n, double p, uint64_t seed, int32_t symmetrise, uint64_t weight_seed, int32_t weight_min,
           int32_t weight_max, gen_graph* out) {
  memset(out, 0, sizeof(*out));
  if (n < 1 || p < 0 || p > 1) return 1;
  const uint64_t base = gen_mix64(seed ^ 0xa4093822299f31d0ull);
  const double lq = (p < 1.0) ? log1p(-p) : 0.0;
  /* pass 1 counts each row's draws, pass 2 repeats them into place */
  int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  for (int pass = 0; pass < 2; pass++) {
    int32_t* src = NULL;
    int32_t* dst = NULL;
    int64_t total = 0;
    if (pass == 1) {
      for (int32_t i = 0; i < n; i++) {
        const int64_t c = cnt[i];
        cnt[i] = total;
        total += c;
      }
      cnt[n] = total;
      const int64_t stored = symmetrise ? 2 * total : total;
      src = (int32_t*)malloc(sizeof(int32_t) * (size_t)(stored > 0 ? stored : 1));
      dst = (int32_t*)malloc(sizeof(int32_t) * (size_t)(stored > 0 ? stored : 1));
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t i = 0; i < n; i++) {
      if (p <= 0.0) continue;
      uint64_t h = gen_mix64(base + (uint64_t)i * 0x9e3779b97f4a7c15ull);
      int64_t j = symmetrise ? (int64_t)i + 1 : 0;
      int64_t k = pass == 1 ? cnt[i] : 0;
      while (1) {
        if (p < 1.0) {
          h = gen_mix64(h + 1);
          const double u = 1.0 - gen_unit(h);
          j += (int64_t)floor(log(u) / lq);
        }
        if (j >= n) break;
        if (j != i) {
          if (pass == 1) {
            src[k] = i;
            dst[k] = (int32_t)j;
            if (symmetrise) {
              src[cnt[n] + k] = (int32_t)j;
              dst[cnt[n] + k] = i;
            }
          }
          k++;
        }
        j++;
      }
      if (pass == 0) cnt[i] = k;
    }
    if (pass == 1) {
      const int64_t stored = symmetrise ? 2 * total : total;
      const int st = gen_build_csr(n, stored, src, dst, out);
      free(src), free(dst);
      if (st) {
        free(cnt);
        gen_free(out);
        return st;
      }
    }
  }
  free(cnt);
  if (weight_seed != 0) {
    if (weight_max < weight_min) {
      gen_free(out);
      return 1;
    }
    out->eweight = (int32_t*)malloc(sizeof(int32_t) * (size_t)(out->edges > 0 ? out->edges : 1));
    const uint64_t span = (uint64_t)((int64_t)weight_max - weight_min + 1);
    const uint64_t ws = gen_mix64(weight_seed ^ 0x082efa98ec4e6c89ull);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t v = 0; v < out->nodes; v++) {
      for (int32_t k = out->nindex[v]; k < out->nindex[v + 1]; k++) {
        const int32_t u = out->nlist[k];
        uint64_t key;
        if (symmetrise)
          key = ((uint64_t)(uint32_t)(u < v ? u : v) << 32) | (uint32_t)(u < v ? v : u);
        else
          key = ((uint64_t)(uint32_t)v << 32) | (uint32_t)u;
        out->eweight[k] = weight_min + (int32_t)(gen_mix64(ws ^ key) % span);
      }
    }
  }
  return 0;
}
