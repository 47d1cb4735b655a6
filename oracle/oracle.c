/*
 * CPU oracle for the race-free ECL-Suite hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * (ecl-suite_b200/) never links, loads or calls it and has no CPU fallback.
 *
 * Each function restates, in plain serial C, the RESULT that the reference's
 * race-free CUDA code computes (see the per-function citations; paths are
 * relative to the ECL-Suite project).  Parity pins:
 *  - orc_mst / orc_apsp follow the reference's own CPU routines cpuMST and
 *    FW_cpu; tests/golden fixtures were produced by those routines, compiled
 *    from the reference sources (oracle/Makefile, oracle/ref_*.cu).
 *  - orc_cc / orc_mis / orc_gc / orc_scc restate the fixpoint the reference
 *    GPU kernels converge to; tests/golden fixtures hold the reference GPU
 *    build's outputs on the same inputs (generated on a B200 by
 *    tests/golden/make_golden.py).
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off: the MIS priority is an
 * fp32 expression that must round exactly like the device code).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MIS_IN 0xfe
#define ORC_MIS_OUT 0x00
#define ORC_INF (0x7fffffff / 2)

/* Integer hash of ECL-MIS-atomic.cu:109-114 and ECL-GC-atomic.cu:70-75. */
static unsigned int orc_hash(unsigned int val) {
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  return (val >> 16) ^ val;
}

/* ------------------------------------------------------------------ CC */

static int uf_find(int* parent, int v) {
  while (parent[v] != v) {
    parent[v] = parent[parent[v]];
    v = parent[v];
  }
  return v;
}

/* ECL-CC-atomic.cu:114-153 hooks v only along entries nlist[i] < v, always
 * larger root under smaller root, and flatten (:250-264) leaves the root, so
 * label[v] = min id in v's component of {(v,u): u in list(v), u < v}. */
void orc_cc(int n, int m, const int* nindex, const int* nlist, int* label) {
  (void)m;
  for (int v = 0; v < n; v++) label[v] = v;
  for (int v = 0; v < n; v++) {
    for (int i = nindex[v]; i < nindex[v + 1]; i++) {
      const int u = nlist[i];
      if (u < v) {
        int a = uf_find(label, v), b = uf_find(label, u);
        if (a != b) {
          if (a < b) label[b] = a;
          else label[a] = b;
        }
      }
    }
  }
  for (int v = 0; v < n; v++) label[v] = uf_find(label, v);
}

/* The reference's CC self-check (ECL-CC-atomic.cu:373-393), iteratively:
 * adjacent vertices share a label, labels are non-negative, every label is
 * the label of exactly one connected piece.  Returns 0 when all pass. */
int orc_verify_cc(int n, int m, const int* nindex, const int* nlist, const int* label) {
  (void)m;
  if (n < 1) return 4;
  for (int v = 0; v < n; v++) {
    if (label[v] < 0) return 2;
    for (int i = nindex[v]; i < nindex[v + 1]; i++)
      if (label[nlist[i]] != label[v]) return 1;
  }
  char* seen = (char*)calloc((size_t)n, 1);
  char* used = (char*)calloc((size_t)n, 1);
  int* stack = (int*)malloc(sizeof(int) * (size_t)n);
  int rc = 0;
  for (int s = 0; s < n && rc == 0; s++) {
    if (seen[s]) continue;
    if (label[s] >= n || used[label[s]]) { rc = 3; break; }
    used[label[s]] = 1;
    int top = 0;
    stack[top++] = s;
    seen[s] = 1;
    while (top > 0 && rc == 0) {
      const int v = stack[--top];
      if (label[v] != label[s]) rc = 3;
      for (int i = nindex[v]; i < nindex[v + 1]; i++) {
        const int u = nlist[i];
        if (!seen[u]) { seen[u] = 1; stack[top++] = u; }
      }
    }
  }
  free(seen); free(used); free(stack);
  return rc;
}

/* ----------------------------------------------------------------- MIS */

/* Priority byte of ECL-MIS-atomic.cu:118-136, in IEEE fp32 with the same
 * operation order: avg = (float)edges/nodes, scaledavg = 126*avg,
 * x = deg - hash(v)*2^-32, res = round-half-even(scaledavg/(avg+x)),
 * byte = (2*res)|1; degree-0 vertices get IN (0xfe). */
void orc_mis_priority(int n, int m, const int* nindex, unsigned char* prio) {
  const float avg = (float)m / (float)n;
  const float scaledavg = 126.0f * avg;
  for (int v = 0; v < n; v++) {
    unsigned char val = ORC_MIS_IN;
    const int degree = nindex[v + 1] - nindex[v];
    if (degree > 0) {
      const float h = (float)orc_hash((unsigned)v) * 0.00000000023283064365386962890625f;
      const float x = (float)degree - h;
      const float q = scaledavg / (avg + x);
      const int res = (int)rintf(q);
      val = (unsigned char)((res + res) | 1);
    }
    prio[v] = val;
  }
}

/* findmins (ECL-MIS-atomic.cu:72-104) lets v join once every undecided
 * neighbour has a lower (byte, id) and no neighbour is in; with fixed
 * priorities that is the sequential greedy MIS in descending (byte, id)
 * order.  status[v] = 0xfe (in) or 0 (out). */
void orc_mis(int n, int m, const int* nindex, const int* nlist, unsigned char* status) {
  unsigned char* prio = (unsigned char*)malloc((size_t)n);
  orc_mis_priority(n, m, nindex, prio);
  int count[256] = {0};
  for (int v = 0; v < n; v++) count[prio[v]]++;
  int start[257];
  start[256] = n;
  for (int b = 255; b >= 0; b--) start[b] = start[b + 1] - count[b];
  /* order[] ascending by (byte, id); walk it backwards. */
  int* order = (int*)malloc(sizeof(int) * (size_t)n);
  int fill[256];
  for (int b = 0; b < 256; b++) fill[b] = start[b];
  for (int v = 0; v < n; v++) order[fill[prio[v]]++] = v;
  for (int v = 0; v < n; v++) status[v] = (prio[v] == ORC_MIS_IN) ? ORC_MIS_IN : 1;
  for (int k = n - 1; k >= 0; k--) {
    const int v = order[k];
    if (status[v] != 1) continue;
    int blocked = 0;
    for (int i = nindex[v]; i < nindex[v + 1]; i++)
      if (status[nlist[i]] == ORC_MIS_IN) { blocked = 1; break; }
    status[v] = blocked ? ORC_MIS_OUT : ORC_MIS_IN;
  }
  free(order);
  free(prio);
}

/* MIS self-check of ECL-MIS-atomic.cu:216-231. */
int orc_verify_mis(int n, int m, const int* nindex, const int* nlist, const unsigned char* status) {
  (void)m;
  for (int v = 0; v < n; v++) {
    if (status[v] != ORC_MIS_IN && status[v] != ORC_MIS_OUT) return 1;
    int any_in = 0;
    for (int i = nindex[v]; i < nindex[v + 1]; i++)
      if (status[nlist[i]] == ORC_MIS_IN) any_in = 1;
    if (status[v] == ORC_MIS_IN && any_in) return 2;
    if (status[v] == ORC_MIS_OUT && !any_in) return 3;
  }
  return 0;
}

/* ------------------------------------------------------------------ GC */

/* Priority of ECL-GC-atomic.cu:102: u outranks v iff deg(u) > deg(v), or
 * equal degrees and hash(u) > hash(v), or both equal and u > v. */
static int gc_outranks(const int* nindex, int u, int v) {
  const int du = nindex[u + 1] - nindex[u], dv = nindex[v + 1] - nindex[v];
  if (du != dv) return du > dv;
  const unsigned hu = orc_hash((unsigned)u), hv = orc_hash((unsigned)v);
  if (hu != hv) return hu > hv;
  return u > v;
}

static const int* g_sort_nindex;
static int gc_cmp_desc(const void* a, const void* b) {
  const int u = *(const int*)a, v = *(const int*)b;
  if (u == v) return 0;
  return gc_outranks(g_sort_nindex, u, v) ? -1 : 1;
}

/* init/runLarge/runSmall (ECL-GC-atomic.cu:78-303) give v the smallest colour
 * not used by its higher-priority list entries (the shortcuts only decide a
 * colour early when no undecided higher-priority neighbour can take it), i.e.
 * first-fit greedy in descending priority order. */
void orc_gc(int n, int m, const int* nindex, const int* nlist, int* color) {
  (void)m;
  int* order = (int*)malloc(sizeof(int) * (size_t)n);
  for (int v = 0; v < n; v++) order[v] = v;
  g_sort_nindex = nindex;
  qsort(order, (size_t)n, sizeof(int), gc_cmp_desc);
  int* stamp = (int*)malloc(sizeof(int) * ((size_t)n + 2));
  for (int v = 0; v < n + 2; v++) stamp[v] = -1;
  for (int v = 0; v < n; v++) color[v] = -1;
  for (int k = 0; k < n; k++) {
    const int v = order[k];
    for (int i = nindex[v]; i < nindex[v + 1]; i++) {
      const int u = nlist[i];
      if (gc_outranks(nindex, u, v) && color[u] >= 0 && color[u] <= n) stamp[color[u]] = v;
    }
    int c = 0;
    while (stamp[c] == v) c++;
    color[v] = c;
  }
  free(stamp);
  free(order);
}

/* GC self-check of ECL-GC-atomic.cu:375-381; returns the colour count in
 * *ncolors (max colour + 1). */
int orc_verify_gc(int n, int m, const int* nindex, const int* nlist, const int* color, int* ncolors) {
  (void)m;
  int mx = -1;
  for (int v = 0; v < n; v++) {
    if (color[v] < 0) return 1;
    if (color[v] > mx) mx = color[v];
    for (int i = nindex[v]; i < nindex[v + 1]; i++)
      if (nlist[i] != v && color[nlist[i]] == color[v]) return 2;
  }
  if (ncolors) *ncolors = mx + 1;
  return 0;
}

/* ----------------------------------------------------------------- MST */

static int cmp_u64(const void* a, const void* b) {
  const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return (x > y) - (x < y);
}

/* cpuMST (ECL-MST_10-atomic.cu:112-154): Kruskal over the v<n copies sorted
 * by (weight, edge index), union-find, in_mst[j] = 1 for the accepted
 * entries.  Returns the total weight. */
uint64_t orc_mst(int n, int m, const int* nindex, const int* nlist, const int* eweight, unsigned char* in_mst) {
  memset(in_mst, 0, (size_t)m);
  int cnt = 0;
  for (int v = 0; v < n; v++)
    for (int j = nindex[v]; j < nindex[v + 1]; j++)
      if (nlist[j] > v) cnt++;
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(cnt > 0 ? cnt : 1));
  int* src = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  int k = 0;
  for (int v = 0; v < n; v++)
    for (int j = nindex[v]; j < nindex[v + 1]; j++) {
      src[j] = v;
      if (nlist[j] > v) keys[k++] = ((uint64_t)(uint32_t)eweight[j] << 32) | (uint32_t)j;
    }
  qsort(keys, (size_t)cnt, sizeof(uint64_t), cmp_u64);
  int* parent = (int*)malloc(sizeof(int) * (size_t)n);
  for (int v = 0; v < n; v++) parent[v] = v;
  uint64_t total = 0;
  int left = n - 1;
  for (int p = 0; p < cnt && left > 0; p++) {
    const int j = (int)(keys[p] & 0xffffffffu);
    const int a = uf_find(parent, src[j]), b = uf_find(parent, nlist[j]);
    if (a != b) {
      in_mst[j] = 1;
      total += (uint64_t)(uint32_t)eweight[j];
      if (a > b) parent[b] = a;
      else parent[a] = b;
      left--;
    }
  }
  free(parent);
  free(src);
  free(keys);
  return total;
}

/* ----------------------------------------------------------------- SCC */

/* ECL-SCC_10-atomic.cu propagates max in-reachable and max out-reachable ids
 * until they agree; the label it reports, readFirst(iomax[v]) (:318), is the
 * largest vertex id of v's SCC.  Restated with an iterative Tarjan. */
void orc_scc(int n, int m, const int* nindex, const int* nlist, int* label) {
  (void)m;
  int* index = (int*)malloc(sizeof(int) * (size_t)n);
  int* low = (int*)malloc(sizeof(int) * (size_t)n);
  int* stk = (int*)malloc(sizeof(int) * (size_t)n);
  char* on = (char*)calloc((size_t)n, 1);
  int* cs_v = (int*)malloc(sizeof(int) * (size_t)n);
  int* cs_i = (int*)malloc(sizeof(int) * (size_t)n);
  for (int v = 0; v < n; v++) index[v] = -1;
  int counter = 0, sp = 0;
  for (int s = 0; s < n; s++) {
    if (index[s] >= 0) continue;
    int cp = 0;
    cs_v[cp] = s;
    cs_i[cp] = nindex[s];
    cp++;
    index[s] = low[s] = counter++;
    stk[sp++] = s;
    on[s] = 1;
    while (cp > 0) {
      const int v = cs_v[cp - 1];
      if (cs_i[cp - 1] < nindex[v + 1]) {
        const int w = nlist[cs_i[cp - 1]++];
        if (index[w] < 0) {
          index[w] = low[w] = counter++;
          stk[sp++] = w;
          on[w] = 1;
          cs_v[cp] = w;
          cs_i[cp] = nindex[w];
          cp++;
        } else if (on[w] && index[w] < low[v]) {
          low[v] = index[w];
        }
      } else {
        cp--;
        if (cp > 0) {
          const int p = cs_v[cp - 1];
          if (low[v] < low[p]) low[p] = low[v];
        }
        if (low[v] == index[v]) {
          int mx = -1, q = sp;
          do {
            q--;
            if (stk[q] > mx) mx = stk[q];
          } while (stk[q] != v);
          while (sp > q) {
            const int w = stk[--sp];
            on[w] = 0;
            label[w] = mx;
          }
        }
      }
    }
  }
  free(index); free(low); free(stk); free(on); free(cs_v); free(cs_i);
}

/* ---------------------------------------------------------------- APSP */

/* FW_cpu (ECL-APSP-atomic.cu:533-570) on an n x n matrix with leading
 * dimension ld: 0 diagonal, INF = INT_MAX/2 elsewhere, then every list entry
 * j of row i writes eweight[j] at (i, nlist[j]) in CSR order (the last
 * duplicate wins, a self-loop overwrites the 0), then the k-i-j triple loop. */
void orc_apsp(int n, int m, const int* nindex, const int* nlist, const int* eweight, int* dist, long ld) {
  (void)m;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) dist[(long)i * ld + j] = (i == j) ? 0 : ORC_INF;
  for (int i = 0; i < n; i++)
    for (int j = nindex[i]; j < nindex[i + 1]; j++) dist[(long)i * ld + nlist[j]] = eweight[j];
  for (int k = 0; k < n; k++)
    for (int i = 0; i < n; i++) {
      const int dik = dist[(long)i * ld + k];
      int* row = dist + (long)i * ld;
      const int* krow = dist + (long)k * ld;
      for (int j = 0; j < n; j++) {
        const int s = dik + krow[j];
        if (row[j] > s) row[j] = s;
      }
    }
}

/* Rows `rows[0..nrows)` of the same closure as orc_apsp, by Dijkstra from
 * each requested source, for matrices too large for the O(n^3) restatement.
 * The arc weight of (i, j) is the LAST list entry i -> j, as the matrix fill
 * of ECL-APSP-atomic.cu:74-83 leaves it; the graph must have no self-loops
 * (then the closure's diagonal is 0) and non-negative weights.  Unreachable
 * entries are ORC_INF.  out is nrows x n. */
void orc_apsp_rows(int n, int m, const int* nindex, const int* nlist, const int* eweight, const int* rows, int nrows,
                   int* out) {
  (void)m;
  long long* d = (long long*)malloc(sizeof(long long) * (size_t)n);
  int* heap = (int*)malloc(sizeof(int) * (size_t)(m + n + 1)); /* lazy-deletion heap of (vertex) keyed by d */
  long long* hk = (long long*)malloc(sizeof(long long) * (size_t)(m + n + 1));
  int* last = (int*)malloc(sizeof(int) * (size_t)n); /* entry index of the last i -> j, per j (scratch) */
  for (int j = 0; j < n; j++) last[j] = -1;
  for (int r = 0; r < nrows; r++) {
    const int s = rows[r];
    for (int j = 0; j < n; j++) d[j] = -1;
    int hs = 0;
    d[s] = 0;
    heap[hs] = s;
    hk[hs++] = 0;
    while (hs > 0) {
      /* pop min */
      const int v = heap[0];
      const long long dv = hk[0];
      hs--;
      heap[0] = heap[hs];
      hk[0] = hk[hs];
      for (int i = 0;;) {
        int c = 2 * i + 1;
        if (c >= hs) break;
        if (c + 1 < hs && hk[c + 1] < hk[c]) c++;
        if (hk[c] >= hk[i]) break;
        const int tv = heap[i];
        const long long tk = hk[i];
        heap[i] = heap[c];
        hk[i] = hk[c];
        heap[c] = tv;
        hk[c] = tk;
        i = c;
      }
      if (dv > d[v] && d[v] >= 0) continue; /* stale */
      /* last duplicate of each arc wins */
      for (int e = nindex[v]; e < nindex[v + 1]; e++) last[nlist[e]] = e;
      for (int e = nindex[v]; e < nindex[v + 1]; e++) {
        const int u = nlist[e];
        if (last[u] != e) continue;
        const long long nd = dv + eweight[e];
        if (d[u] < 0 || nd < d[u]) {
          d[u] = nd;
          int i = hs++;
          heap[i] = u;
          hk[i] = nd;
          while (i > 0) {
            const int p = (i - 1) / 2;
            if (hk[p] <= hk[i]) break;
            const int tv = heap[i];
            const long long tk = hk[i];
            heap[i] = heap[p];
            hk[i] = hk[p];
            heap[p] = tv;
            hk[p] = tk;
            i = p;
          }
        }
      }
      for (int e = nindex[v]; e < nindex[v + 1]; e++) last[nlist[e]] = -1;
    }
    for (int j = 0; j < n; j++) out[(long)r * n + j] = (d[j] < 0 || d[j] > ORC_INF) ? ORC_INF : (int)d[j];
  }
  free(d);
  free(heap);
  free(hk);
  free(last);
}
