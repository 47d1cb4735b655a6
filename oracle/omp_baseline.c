/*
 * OpenMP CPU baselines for CC, MIS, GC and SCC -- TEST / BASELINE
 * INFRASTRUCTURE ONLY (the reference has no CPU solver for these four codes;
 * its CPU routines are cpuMST and FW_cpu, which bench.py times directly).
 *
 * Only tests/ and the cpu_baseline / --impl reference legs of bench.py load
 * this (it is linked into oracle/_build/liboracle.so).  Each function is a
 * plain multi-threaded rendering of the same algorithm family the reference
 * uses and returns exactly the serial oracle's result (tests/test_oracle.py
 * checks that): shared words are accessed with GCC __atomic builtins only.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OMP_MIS_IN 0xfe
#define OMP_MIS_OUT 0x00

void orc_mis_priority(int n, int m, const int* nindex, unsigned char* prio);

static inline int ald(const int* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
static inline void ast(int* p, int v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
static inline int acas(int* p, int expected, int desired) {
  __atomic_compare_exchange_n(p, &expected, desired, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
  return expected;
}
static inline void amax(int* p, int v) {
  int cur = ald(p);
  while (cur < v) {
    const int seen = acas(p, cur, v);
    if (seen == cur) return;
    cur = seen;
  }
}

int omp_threads(void) { return omp_get_max_threads(); }

/* ------------------------------------------------------------------ CC */

/* Root of v with path halving (parents point at smaller ids). */
static int cc_find(int* parent, int v) {
  int p = ald(&parent[v]);
  while (p != v) {
    const int gp = ald(&parent[p]);
    if (gp != p) ast(&parent[v], gp);
    v = p;
    p = ald(&parent[v]);
  }
  return v;
}

/* Union-find over the entries u < v of every list (ECL-CC-atomic.cu:114-153
 * semantics), larger root hooked under the smaller by CAS; the flattened
 * roots are the component minima.  Same result as orc_cc. */
void omp_cc(int n, int m, const int* nindex, const int* nlist, int* label) {
  (void)m;
#pragma omp parallel for schedule(static)
  for (int v = 0; v < n; v++) label[v] = v;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int v = 0; v < n; v++) {
    for (int i = nindex[v]; i < nindex[v + 1]; i++) {
      const int u = nlist[i];
      if (u >= v || u < 0) continue;
      int a = v, b = u;
      for (;;) {
        a = cc_find(label, a);
        b = cc_find(label, b);
        if (a == b) break;
        if (a < b) {
          const int t = a;
          a = b;
          b = t;
        }
        if (acas(&label[a], a, b) == a) break;
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int v = 0; v < n; v++) ast(&label[v], cc_find(label, v));
}

/* ------------------------------------------------------------------ MIS */

/* Sweeps over a shrinking list of undecided vertices, updating in place: v
 * joins once no undecided neighbour outranks it in (priority byte, id) and no
 * neighbour is in; it leaves once a neighbour is in (ECL-MIS-atomic.cu:72-104).
 * With fixed priorities the fixpoint is the greedy MIS in descending order,
 * whatever the interleaving -- the same set as orc_mis. */
void omp_mis(int n, int m, const int* nindex, const int* nlist, unsigned char* status) {
  unsigned char* prio = (unsigned char*)malloc((size_t)n);
  int* wl = (int*)malloc(sizeof(int) * (size_t)n);
  int* wl2 = (int*)malloc(sizeof(int) * (size_t)n);
  orc_mis_priority(n, m, nindex, prio);
  int size = 0;
  for (int v = 0; v < n; v++) {
    status[v] = prio[v];
    if (prio[v] & 1) wl[size++] = v;
  }
  while (size > 0) {
    int next = 0;
#pragma omp parallel
    {
      const int nt = omp_get_num_threads(), t = omp_get_thread_num();
      const int lo = (int)((long long)size * t / nt), hi = (int)((long long)size * (t + 1) / nt);
      int* keep = (int*)malloc(sizeof(int) * (size_t)(hi - lo + 1));
      int nk = 0;
      for (int k = lo; k < hi; k++) {
        const int v = wl[k];
        const unsigned char b = prio[v];
        int verdict = 1; /* join */
        for (int i = nindex[v]; i < nindex[v + 1]; i++) {
          const int u = nlist[i];
          const unsigned char su = __atomic_load_n(&status[u], __ATOMIC_RELAXED);
          if (su == OMP_MIS_IN) {
            verdict = 2; /* out */
            break;
          }
          if ((su & 1) && (su > b || (su == b && u > v))) verdict = 0; /* wait */
        }
        if (verdict == 1)
          __atomic_store_n(&status[v], (unsigned char)OMP_MIS_IN, __ATOMIC_RELAXED);
        else if (verdict == 2)
          __atomic_store_n(&status[v], (unsigned char)OMP_MIS_OUT, __ATOMIC_RELAXED);
        else
          keep[nk++] = v;
      }
      const int at = __atomic_fetch_add(&next, nk, __ATOMIC_RELAXED);
      memcpy(wl2 + at, keep, sizeof(int) * (size_t)nk);
      free(keep);
    }
    int* t = wl;
    wl = wl2;
    wl2 = t;
    size = next;
  }
  free(prio);
  free(wl);
  free(wl2);
}

/* ------------------------------------------------------------------ GC */

static inline unsigned gc_hash(unsigned val) {
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  return (val >> 16) ^ val;
}

/* u outranks v in (degree, hash, id) (ECL-GC-atomic.cu:102). */
static inline int gc_higher(const int* nindex, int u, int v) {
  const int du = nindex[u + 1] - nindex[u], dv = nindex[v + 1] - nindex[v];
  if (du != dv) return du > dv;
  const unsigned hu = gc_hash((unsigned)u), hv = gc_hash((unsigned)v);
  if (hu != hv) return hu > hv;
  return u > v;
}

/* First-fit greedy in priority order as topological waves: cnt[v] counts
 * v's uncoloured higher-priority neighbours; a wave colours every vertex
 * whose count is zero (smallest colour none of its higher neighbours uses)
 * and releases its lower neighbours.  Same colouring as orc_gc. */
void omp_gc(int n, int m, const int* nindex, const int* nlist, int* color) {
  (void)m;
  int* cnt = (int*)malloc(sizeof(int) * (size_t)n);
  int* wave = (int*)malloc(sizeof(int) * (size_t)n);
  int* next = (int*)malloc(sizeof(int) * (size_t)n);
  int size = 0;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int v = 0; v < n; v++) {
    int c = 0;
    for (int i = nindex[v]; i < nindex[v + 1]; i++) {
      const int u = nlist[i];
      if (u != v && gc_higher(nindex, u, v)) c++;
    }
    cnt[v] = c;
    color[v] = -1;
  }
  for (int v = 0; v < n; v++)
    if (cnt[v] == 0) wave[size++] = v;
  while (size > 0) {
    int nsize = 0;
#pragma omp parallel
    {
      int cap = 64;
      unsigned long long* used = (unsigned long long*)calloc((size_t)cap, 8);
      int* rel = (int*)malloc(sizeof(int) * 1024);
      int nrel = 0, relcap = 1024;
#pragma omp for schedule(dynamic, 64)
      for (int k = 0; k < size; k++) {
        const int v = wave[k];
        const int deg = nindex[v + 1] - nindex[v];
        const int words = deg / 64 + 1;
        if (words > cap) {
          free(used);
          cap = words;
          used = (unsigned long long*)calloc((size_t)cap, 8);
        }
        for (int i = nindex[v]; i < nindex[v + 1]; i++) {
          const int u = nlist[i];
          if (u == v || !gc_higher(nindex, u, v)) continue;
          const int c = ald(&color[u]);
          if (c < 64 * words) used[c >> 6] |= 1ull << (c & 63);
        }
        int c = 0;
        while (used[c >> 6] & (1ull << (c & 63))) c++;
        for (int w = 0; w < words; w++) used[w] = 0;
        ast(&color[v], c);
        for (int i = nindex[v]; i < nindex[v + 1]; i++) {
          const int w = nlist[i];
          if (w == v || gc_higher(nindex, w, v)) continue;
          if (__atomic_sub_fetch(&cnt[w], 1, __ATOMIC_ACQ_REL) == 0) {
            if (nrel == relcap) {
              relcap *= 2;
              rel = (int*)realloc(rel, sizeof(int) * (size_t)relcap);
            }
            rel[nrel++] = w;
          }
        }
      }
      const int at = __atomic_fetch_add(&nsize, nrel, __ATOMIC_RELAXED);
      memcpy(next + at, rel, sizeof(int) * (size_t)nrel);
      free(rel);
      free(used);
    }
    int* t = wave;
    wave = next;
    next = t;
    size = nsize;
  }
  free(cnt);
  free(wave);
  free(next);
}

/* ------------------------------------------------------------------ SCC */

/* Max-id propagation with trimming (the family of ECL-SCC_10-atomic.cu:
 * 132-214): per round, in-max travels forward and out-max backward along the
 * live edges to a fixpoint; a vertex whose two values agree is labelled with
 * them (the largest id of its SCC); edges whose ends disagree are dropped and
 * the rest start over.  Same labels as orc_scc. */
void omp_scc(int n, int m, const int* nindex, const int* nlist, int* label) {
  (void)m;
  char* in = (char*)calloc((size_t)n, 1);
  char* out = (char*)calloc((size_t)n, 1);
  int* imax = (int*)malloc(sizeof(int) * (size_t)n);
  int* omax = (int*)malloc(sizeof(int) * (size_t)n);
  for (int v = 0; v < n; v++)
    for (int i = nindex[v]; i < nindex[v + 1]; i++)
      if (nlist[i] != v) {
        in[nlist[i]] = 1;
        out[v] = 1;
      }
  long long ne = 0;
  for (int v = 0; v < n; v++)
    if (in[v] && out[v])
      for (int i = nindex[v]; i < nindex[v + 1]; i++) {
        const int w = nlist[i];
        if (w != v && in[w] && out[w]) ne++;
      }
  int* es = (int*)malloc(sizeof(int) * (size_t)(ne + 1));
  int* ed = (int*)malloc(sizeof(int) * (size_t)(ne + 1));
  ne = 0;
  for (int v = 0; v < n; v++)
    if (in[v] && out[v])
      for (int i = nindex[v]; i < nindex[v + 1]; i++) {
        const int w = nlist[i];
        if (w != v && in[w] && out[w]) {
          es[ne] = v;
          ed[ne] = w;
          ne++;
        }
      }
#pragma omp parallel for schedule(static)
  for (int v = 0; v < n; v++) {
    imax[v] = v;
    omax[v] = v;
    label[v] = -1;
  }
  for (;;) {
    int changed = 1;
    while (changed) {
      changed = 0;
#pragma omp parallel for schedule(static) reduction(| : changed)
      for (long long k = 0; k < ne; k++) {
        const int v = es[k], w = ed[k];
        const int iv = ald(&imax[v]), ow = ald(&omax[w]);
        if (ald(&imax[w]) < iv) {
          amax(&imax[w], iv);
          changed = 1;
        }
        if (ald(&omax[v]) < ow) {
          amax(&omax[v], ow);
          changed = 1;
        }
      }
    }
    long long keep = 0;
    for (long long k = 0; k < ne; k++) {
      const int v = es[k], w = ed[k];
      if (imax[v] != omax[v] && imax[v] == imax[w] && omax[v] == omax[w]) {
        es[keep] = v;
        ed[keep] = w;
        keep++;
      }
    }
    int again = 0;
#pragma omp parallel for schedule(static) reduction(| : again)
    for (int v = 0; v < n; v++) {
      if (label[v] >= 0) continue;
      if (imax[v] == omax[v]) {
        label[v] = imax[v];
      } else {
        imax[v] = v;
        omax[v] = v;
        again = 1;
      }
    }
    ne = keep;
    if (!again) break;
  }
  free(in);
  free(out);
  free(imax);
  free(omax);
  free(es);
  free(ed);
}
