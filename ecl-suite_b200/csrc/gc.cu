// Graph colouring (ECL-GC contract).
//
// Result contract (src/racefree/egr-input/GC/ECL-GC-atomic.cu): a vertex's
// colour is chosen among [0, r] where r is its number of higher-priority list
// entries, priority being (degree, hash, id) (:102).  init/runLarge/runSmall
// (:78-303) only fix a colour once it is the smallest colour not taken by a
// decided higher-priority neighbour and no undecided higher-priority
// neighbour can still take it, which yields the first-fit greedy colouring in
// descending priority order -- a schedule-independent result.
//
// B200 design (Jones-Plassmann with window shortcutting):
//  * gc_init compacts each vertex's higher-priority entries into hl[] at the
//    vertex's own CSR offset (lane-serial for short lists, warp ballot +
//    popc compaction for long ones) and sets state[v] = (lo=0, hi=r).
//  * state[v] is one 32-bit word (lo << 16 | hi): lo = smallest colour v can
//    still get, hi = r, an upper bound.  lo == hi means decided (colour lo).
//    r <= sqrt(edges) < 46341, so 16 bits each suffice.
//  * gc_run is ONE persistent launch.  Each undecided vertex scans its hl
//    list once per sweep, building two 64-bit masks over the colour window
//    [lo, lo+64): colours of decided neighbours, and the union of the
//    possible-colour windows of undecided neighbours.  The first free colour
//    c in the window is v's colour as soon as no undecided neighbour can
//    take it; otherwise lo advances to c.  Long lists are scanned by the
//    whole warp with the masks OR-reduced by __reduce_or_sync.
#include "runtime.cuh"

namespace ecl {
namespace {

using namespace dev;

constexpr int kTPB = 256;
constexpr int kLaneMax = 32;

__device__ __forceinline__ bool gc_outranks(int du, unsigned hu, int u, int dv, unsigned hv, int v) {
  if (du != dv) return du > dv;
  if (hu != hv) return hu > hv;
  return u > v;
}

__global__ void __launch_bounds__(kTPB) gc_init(int n, int m, const int* __restrict__ nindex,
                                                const int* __restrict__ nlist, int* __restrict__ hl,
                                                int* __restrict__ hc, unsigned* __restrict__ state,
                                                int* __restrict__ color, Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    const int v = base + lane;
    int beg = 0, end = 0;
    if (v < n) {
      beg = __ldg(&nindex[v]);
      end = __ldg(&nindex[v + 1]);
      if (beg < 0 || end < beg || end > m) {
        raise(status, ECL_ERR_BAD_GRAPH, v);
        beg = end = 0;
      }
    }
    const int dv = end - beg;
    const unsigned hv = ecl_hash((unsigned)v);
    int cnt = 0;
    const bool big = dv > kLaneMax;
    if (v < n && !big) {
      for (int i = beg; i < end; i++) {
        const int u = __ldg(&nlist[i]);
        if ((unsigned)u >= (unsigned)n) {
          raise(status, ECL_ERR_BAD_GRAPH, u);
          continue;
        }
        const int du = __ldg(&nindex[u + 1]) - __ldg(&nindex[u]);
        if (gc_outranks(du, ecl_hash((unsigned)u), u, dv, hv, v)) hl[beg + cnt++] = u;
      }
    }
    unsigned todo = __ballot_sync(kFull, big);
    while (todo) {
      const int who = __ffs(todo) - 1;
      todo &= todo - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      const int wdv = wend - wbeg;
      const unsigned whv = ecl_hash((unsigned)wv);
      int wcnt = 0;
      for (int i0 = wbeg; i0 < wend; i0 += 32) {
        const int i = i0 + lane;
        bool keep = false;
        int u = 0;
        if (i < wend) {
          u = __ldg(&nlist[i]);
          if ((unsigned)u < (unsigned)n) {
            const int du = __ldg(&nindex[u + 1]) - __ldg(&nindex[u]);
            keep = gc_outranks(du, ecl_hash((unsigned)u), u, wdv, whv, wv);
          } else {
            raise(status, ECL_ERR_BAD_GRAPH, u);
          }
        }
        const unsigned bal = __ballot_sync(kFull, keep);
        if (keep) hl[wbeg + wcnt + __popc(bal & ((1u << lane) - 1))] = u;
        wcnt += __popc(bal);
      }
      if (lane == who) cnt = wcnt;
    }
    if (v < n) {
      if (cnt > 0xffff) raise(status, ECL_ERR_UNSUPPORTED, v);
      hc[v] = cnt;
      state[v] = (unsigned)cnt & 0xffffu;  // lo = 0, hi = cnt; cnt == 0 means decided colour 0
      if (cnt == 0) color[v] = 0;
    }
  }
}

// Folds neighbour state s into the masks of window [lo, lo+64).
__device__ __forceinline__ void gc_fold(unsigned s, int lo, unsigned long long& used, unsigned long long& cover) {
  const int slo = (int)(s >> 16), shi = (int)(s & 0xffffu);
  if (slo == shi) {
    const int d = slo - lo;
    if (d >= 0 && d < 64) used |= 1ull << d;
  } else {
    const int a = max(slo, lo) - lo, b = min(shi, lo + 63) - lo;
    if (a <= b) {
      const unsigned long long hiMask = (b >= 63) ? ~0ull : ((1ull << (b + 1)) - 1);
      cover |= hiMask & ~((1ull << a) - 1);
    }
  }
}

// Applies one scan's result to v.  Returns true when v is still undecided.
__device__ __forceinline__ bool gc_apply(int v, int lo, int hi, unsigned long long used, unsigned long long cover,
                                         unsigned* state, int* color) {
  if (used == ~0ull) {  // the whole window is taken by decided neighbours
    const int nlo = lo + 64;  // <= hi: 64 + lo decided neighbours exist
    if (nlo >= hi) {
      color[v] = hi;
      st(&state[v], ((unsigned)hi << 16) | (unsigned)hi);
      return false;
    }
    st(&state[v], ((unsigned)nlo << 16) | (unsigned)hi);
    return true;
  }
  const int c = __ffsll((long long)~used) - 1;
  const int col = lo + c;
  if (((cover >> c) & 1ull) == 0 || col == hi) {
    color[v] = col;
    st(&state[v], ((unsigned)col << 16) | (unsigned)col);
    return false;
  }
  if (col != lo) st(&state[v], ((unsigned)col << 16) | (unsigned)hi);
  return true;
}

__global__ void __launch_bounds__(kTPB) gc_run(int n, const int* __restrict__ nindex, const int* __restrict__ hl,
                                               const int* __restrict__ hc, unsigned* __restrict__ state,
                                               int* __restrict__ color, Status* __restrict__ status,
                                               int max_sweeps) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  int sweep = 0;
  for (;; sweep++) {
    bool missing = false;
    for (int base = warp * 32; base < n; base += nwarps * 32) {
      const int v = base + lane;
      unsigned s = 0;
      if (v < n) s = ld(&state[v]);
      const int lo = (int)(s >> 16), hi = (int)(s & 0xffffu);
      const bool und = (v < n) && lo != hi;
      if (!__any_sync(kFull, und)) continue;
      int beg = 0, cnt = 0;
      if (und) {
        beg = __ldg(&nindex[v]);
        cnt = __ldg(&hc[v]);
      }
      const bool big = und && cnt > kLaneMax;
      if (und && !big) {
        unsigned long long used = 0, cover = 0;
        for (int i = beg; i < beg + cnt; i++) gc_fold(ld(&state[__ldg(&hl[i])]), lo, used, cover);
        missing |= gc_apply(v, lo, hi, used, cover, state, color);
      }
      unsigned todo = __ballot_sync(kFull, big);
      while (todo) {
        const int who = __ffs(todo) - 1;
        todo &= todo - 1;
        const int wv = __shfl_sync(kFull, v, who);
        const int wbeg = __shfl_sync(kFull, beg, who);
        const int wend = wbeg + __shfl_sync(kFull, cnt, who);
        const int wlo = __shfl_sync(kFull, lo, who);
        const int whi = __shfl_sync(kFull, hi, who);
        unsigned long long used = 0, cover = 0;
        for (int i = wbeg + lane; i < wend; i += 32) gc_fold(ld(&state[__ldg(&hl[i])]), wlo, used, cover);
        const unsigned ul = __reduce_or_sync(kFull, (unsigned)used);
        const unsigned uh = __reduce_or_sync(kFull, (unsigned)(used >> 32));
        const unsigned cl = __reduce_or_sync(kFull, (unsigned)cover);
        const unsigned ch = __reduce_or_sync(kFull, (unsigned)(cover >> 32));
        if (lane == who) {
          used = ((unsigned long long)uh << 32) | ul;
          cover = ((unsigned long long)ch << 32) | cl;
          missing |= gc_apply(wv, wlo, whi, used, cover, state, color);
        }
      }
    }
    if (!__any_sync(kFull, missing)) break;
    if (sweep >= max_sweeps) {
      if (lane == 0) raise(status, ECL_ERR_NO_CONVERGENCE, warp);
      break;
    }
  }
  if (lane == 0) fetch_max(&status->rounds, sweep + 1);
}

void gc_layout(Carve& c, int n, int m, int** hl, int** hc, unsigned** state) {
  *hl = c.take<int>((size_t)(m > 0 ? m : 1));
  *hc = c.take<int>((size_t)n);
  *state = c.take<unsigned>((size_t)n);
}

}  // namespace

size_t gc_workspace_bytes(int n, int m) {
  Carve c;
  int *hl, *hc;
  unsigned* state;
  gc_layout(c, n, m, &hl, &hc, &state);
  return c.bytes();
}

}  // namespace ecl

extern "C" ecl_status ecl_gc(const ecl_graph_view* g, int32_t* color_out, ecl_opts* opts) {
  using namespace ecl;
  ecl_opts local{};
  if (!opts) opts = &local;
  if (!color_out) return ECL_ERR_INVALID_ARG;
  Solve s(g, opts);
  GraphNeeds needs;
  needs.symmetric = true;
  needs.no_self_loops = true;
  ecl_status st = s.begin(needs, g ? gc_workspace_bytes(g->nodes, g->edges) : 0);
  if (st != ECL_OK) return s.finish(st);
  int* color = s.output(color_out, (size_t)s.n);
  if (!color) return s.finish(ECL_ERR_OOM);
  Carve c{s.ws};
  int *hl, *hc;
  unsigned* state;
  gc_layout(c, s.n, s.m, &hl, &hc, &state);
  const int grid = s.dev.sms * (s.dev.max_threads_per_sm / kTPB);
  // Warps sweep asynchronously, so one warp may sweep many times while it
  // waits on a vertex owned by a slower warp: the cap is a fixed backstop
  // (GC cannot stall -- priorities form a DAG), not a per-graph bound.
  const int max_sweeps = opts->max_rounds > 0 ? opts->max_rounds : (1 << 22);

  s.start_timer();
  ECL_LAUNCH(gc_init, grid, kTPB, 0, s.stream, s.n, s.m, s.nindex, s.nlist, hl, hc, state, color, s.status);
  s.mark();
  ECL_LAUNCH(gc_run, grid, kTPB, 0, s.stream, s.n, s.nindex, hl, hc, state, color, s.status, max_sweeps);
  s.mark();
  s.stop_timer();
  return s.finish();
}

extern "C" ecl_status ecl_compute_gc(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist,
                                     int32_t* color) {
  ecl_graph_view g{nodes, edges, nidx, nlist, nullptr, ECL_HOST, 0};
  ecl_opts o{};
  return ecl_gc(&g, color, &o);
}
