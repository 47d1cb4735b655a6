// Strongly connected components (ECL-SCC contract).
//
// Result contract (src/racefree/mesh-input/ECL-SCC_10-atomic.cu): the
// reference keeps, per vertex, the largest id that reaches it (in-max) and the
// largest id it reaches (out-max) within the current edge set, propagates both
// to a fixpoint (:132-172), retires vertices whose two values agree, drops
// edges whose endpoints disagree (:175-195), resets the rest (:198-214) and
// repeats.  A vertex retires exactly when the largest id of its SCC reaches it
// and is reached by it, so the label it reports, readFirst(iomax[v]) (:318),
// is the largest vertex id of v's SCC -- schedule independent.
//
// B200 design:
//  * scc_mark / scc_build trim first: a vertex with no in-entry or no
//    out-entry (self-loops ignored) is its own SCC and contributes no edge;
//    only edges between two untrimmed vertices enter the int2 worklist
//    (warp-aggregated appends).  Both passes are degree-binned (lane / warp /
//    256-entry chunk records), so hub rows spread over all warps;
//  * scc_solve runs EVERY propagation sweep and every trimming round in one
//    cooperative persistent launch, separated by bounded grid barriers (the
//    reference pays a host round trip per propagation launch, :283-287);
//    in-max / out-max live in two int arrays updated with fetch_max, and each
//    sweep jumps through imax[imax[v]] / omax[omax[w]] (both still valid
//    bounds) so values travel many hops per sweep;
//  * the final labels are written by the same launch (label = in-max).
#include "csr_bins.cuh"
#include "grid_sync.cuh"
#include "solvers.cuh"

namespace ecl {
namespace {

using namespace dev;

constexpr int kTPB = 256;
constexpr int kMaxSweeps = 1 << 16;

struct SCCCtl {
  GridBarrier bar;
  int nedges;       // initial worklist size
  int sizes[2];     // unused slot for alignment
  int pad[61];
  int changed[kMaxSweeps];   // per-sweep "something moved" flags
};

struct SCCRound {
  int size;
  int again;
};

// A vertex is live (can be in a non-trivial SCC) iff it has an in-entry and an
// out-entry other than self-loops.  scc_mark sets hasin[w] for every entry
// w != v (plain relaxed stores of 1: idempotent) and hasout[v] for every v
// with such an entry; rows longer than kBinChunk go to chunk records.
__device__ __forceinline__ void scc_mark_entry(bool valid, int v, int w, int n, int* hasin, bool& out,
                                               Status* status) {
  if (!valid) return;
  if ((unsigned)w >= (unsigned)n) {
    raise(status, ECL_ERR_BAD_GRAPH, w);
  } else if (w != v) {
    st(&hasin[w], 1);
    out = true;
  }
}

__global__ void __launch_bounds__(kTPB) scc_mark(int n, int m, const int* __restrict__ nindex,
                                                 const int* __restrict__ nlist, int* __restrict__ hasin,
                                                 int* __restrict__ hasout, int* __restrict__ imax,
                                                 int* __restrict__ omax, RowChunks rc, Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    const int v = base + lane;
    int beg = 0, end = 0;
    if (v < n) {
      csr_row(nindex, v, m, beg, end, status);
      imax[v] = v;
      omax[v] = v;
    }
    const int deg = end - beg;
    if (deg > kBinChunk) push_row_chunks(rc, v, beg, end);
    bool out = false;
    const bool lanelvl = deg <= kBinLane;
    const int kmax = __reduce_max_sync(kFull, lanelvl ? deg : 0);
    for (int k = 0; k < kmax; k++) {
      const bool valid = lanelvl && k < deg;
      scc_mark_entry(valid, v, valid ? __ldg(&nlist[beg + k]) : 0, n, hasin, out, status);
    }
    unsigned todo = __ballot_sync(kFull, deg > kBinLane && deg <= kBinChunk);
    while (todo) {
      const int who = __ffs(todo) - 1;
      todo &= todo - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      bool wout = false;
      for (int i = wbeg + lane; i < wend; i += 32) scc_mark_entry(true, wv, __ldg(&nlist[i]), n, hasin, wout, status);
      if (__any_sync(kFull, wout) && lane == who) out = true;
    }
    if (v < n) hasout[v] = (deg <= kBinChunk && out) ? 1 : 0;  // long rows: set by scc_mark_chunks
  }
}

__global__ void __launch_bounds__(kTPB) scc_mark_chunks(int n, const int* __restrict__ nindex,
                                                        const int* __restrict__ nlist, int* __restrict__ hasin,
                                                        int* __restrict__ hasout, RowChunks rc,
                                                        Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int total = *rc.count;
  for (int c = warp; c < total; c += nwarps) {
    const int2 r = rc.rec[c];
    const int end = min(r.y + kBinChunk, __ldg(&nindex[r.x + 1]));
    bool out = false;
    for (int i = r.y + lane; i < end; i += 32) scc_mark_entry(true, r.x, __ldg(&nlist[i]), n, hasin, out, status);
    if (__any_sync(kFull, out) && lane == 0) st(&hasout[r.x], 1);
  }
}

__device__ __forceinline__ bool scc_live(const int* hasin, const int* hasout, int v) {
  return ld(&hasin[v]) != 0 && ld(&hasout[v]) != 0;
}

__global__ void __launch_bounds__(kTPB) scc_build(int n, int m, const int* __restrict__ nindex,
                                                  const int* __restrict__ nlist, const int* __restrict__ hasin,
                                                  const int* __restrict__ hasout, int2* __restrict__ wl,
                                                  SCCCtl* __restrict__ ctl) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    const int v = base + lane;
    int beg = 0, end = 0;
    if (v < n && scc_live(hasin, hasout, v)) {
      beg = __ldg(&nindex[v]);
      end = __ldg(&nindex[v + 1]);
      if (beg < 0 || end < beg || end > m) beg = end = 0;
    }
    const int deg = end - beg;
    const bool lanelvl = deg <= kBinLane;
    const int kmax = __reduce_max_sync(kFull, lanelvl ? deg : 0);
    for (int k = 0; k < kmax; k++) {
      bool keep = false;
      int w = 0;
      if (lanelvl && k < deg) {
        w = __ldg(&nlist[beg + k]);
        keep = w != v && (unsigned)w < (unsigned)n && scc_live(hasin, hasout, w);
      }
      const int at = warp_append(&ctl->nedges, keep);
      if (keep) wl[at] = make_int2(v, w);
    }
    unsigned todo = __ballot_sync(kFull, deg > kBinLane && deg <= kBinChunk);
    while (todo) {
      const int who = __ffs(todo) - 1;
      todo &= todo - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      for (int i0 = wbeg; i0 < wend; i0 += 32) {
        bool keep = false;
        int w = 0;
        if (i0 + lane < wend) {
          w = __ldg(&nlist[i0 + lane]);
          keep = w != wv && (unsigned)w < (unsigned)n && scc_live(hasin, hasout, w);
        }
        const int at = warp_append(&ctl->nedges, keep);
        if (keep) wl[at] = make_int2(wv, w);
      }
    }
  }
}

__global__ void __launch_bounds__(kTPB) scc_build_chunks(int n, const int* __restrict__ nindex,
                                                         const int* __restrict__ nlist, const int* __restrict__ hasin,
                                                         const int* __restrict__ hasout, int2* __restrict__ wl,
                                                         SCCCtl* __restrict__ ctl, RowChunks rc) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int total = *rc.count;
  for (int c = warp; c < total; c += nwarps) {
    const int2 r = rc.rec[c];
    if (!scc_live(hasin, hasout, r.x)) continue;  // warp-uniform
    const int end = min(r.y + kBinChunk, __ldg(&nindex[r.x + 1]));
    for (int i0 = r.y; i0 < end; i0 += 32) {
      bool keep = false;
      int w = 0;
      if (i0 + lane < end) {
        w = __ldg(&nlist[i0 + lane]);
        keep = w != r.x && (unsigned)w < (unsigned)n && scc_live(hasin, hasout, w);
      }
      const int at = warp_append(&ctl->nedges, keep);
      if (keep) wl[at] = make_int2(r.x, w);
    }
  }
}

__global__ void __launch_bounds__(kTPB) scc_solve(int n, int2* __restrict__ wlA, int2* __restrict__ wlB,
                                                  int* __restrict__ imax, int* __restrict__ omax,
                                                  int* __restrict__ label, SCCCtl* __restrict__ ctl,
                                                  SCCRound* __restrict__ rounds, int max_rounds,
                                                  Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int tid = blockIdx.x * kTPB + threadIdx.x;
  const int nthreads = gridDim.x * kTPB;
  int size = ld(&ctl->nedges);
  int sweep = 0;
  int round = 0;
  int2* cur = wlA;
  int2* nxt = wlB;
  for (;; round++) {
    if (round >= max_rounds) {
      raise(status, ECL_ERR_NO_CONVERGENCE, round);
      return;
    }
    // 1. propagate in-max forward and out-max backward to a fixpoint
    while (true) {
      if (sweep >= kMaxSweeps) {
        raise(status, ECL_ERR_NO_CONVERGENCE, -sweep);
        return;
      }
      bool moved = false;
      for (int i = tid; i < size; i += nthreads) {
        const int2 e = cur[i];
        const int v = e.x, w = e.y;
        int iv = ld(&imax[v]);
        if (iv != v) iv = max(iv, ld(&imax[iv]));
        if (ld(&imax[w]) < iv) {
          fetch_max(&imax[w], iv);
          moved = true;
        }
        int ow = ld(&omax[w]);
        if (ow != w) ow = max(ow, ld(&omax[ow]));
        if (ld(&omax[v]) < ow) {
          fetch_max(&omax[v], ow);
          moved = true;
        }
      }
      if (__any_sync(kFull, moved) && lane == 0) st(&ctl->changed[sweep], 1);
      if (!grid_sync(&ctl->bar, status)) return;
      const bool again = ld(&ctl->changed[sweep]) != 0;
      sweep++;
      if (!again) break;
    }
    // 2. keep the edges whose endpoints are unresolved and agree
    for (int i0 = tid - lane; i0 < size; i0 += nthreads) {
      const int i = i0 + lane;
      bool keep = false;
      int2 e = make_int2(0, 0);
      if (i < size) {
        e = cur[i];
        const int iv = ld(&imax[e.x]), ov = ld(&omax[e.x]);
        keep = iv != ov && iv == ld(&imax[e.y]) && ov == ld(&omax[e.y]);
      }
      const int at = warp_append(&rounds[round].size, keep);
      if (keep) nxt[at] = e;
    }
    if (!grid_sync(&ctl->bar, status)) return;
    // 3. retire resolved vertices, reset the rest to their own id
    bool again = false;
    for (int v = tid; v < n; v += nthreads) {
      const int iv = ld(&imax[v]);
      if (iv == ld(&omax[v])) {
        label[v] = iv;
      } else {
        st(&imax[v], v);
        st(&omax[v], v);
        again = true;
      }
    }
    if (__any_sync(kFull, again) && lane == 0) st(&rounds[round].again, 1);
    if (!grid_sync(&ctl->bar, status)) return;
    if (!ld(&rounds[round].again)) break;
    size = ld(&rounds[round].size);
    int2* t = cur;
    cur = nxt;
    nxt = t;
  }
  if (tid == 0) st(&status->rounds, sweep);
}

struct SCCBufs {
  SCCCtl* ctl;
  SCCRound* rounds;
  int* hasin;
  int* hasout;
  int* nchunks;
  int2* chunks;
  int* imax;
  int* omax;
  int2* wlA;
  int2* wlB;
  int max_rounds;
};

void scc_layout(Carve& c, int n, int m, SCCBufs* b) {
  b->ctl = c.take<SCCCtl>(1);
  b->max_rounds = n + 1;
  b->rounds = c.take<SCCRound>((size_t)b->max_rounds);
  b->hasin = c.take<int>((size_t)n);
  b->hasout = c.take<int>((size_t)n);
  b->nchunks = c.take<int>(64);
  b->chunks = c.take<int2>(row_chunk_capacity(m));
  b->imax = c.take<int>((size_t)n);
  b->omax = c.take<int>((size_t)n);
  b->wlA = c.take<int2>((size_t)(m > 0 ? m : 1));
  b->wlB = c.take<int2>((size_t)(m > 0 ? m : 1));
}

}  // namespace

size_t scc_workspace_bytes(int n, int m) {
  Carve c;
  SCCBufs b;
  scc_layout(c, n, m, &b);
  return c.bytes();
}

}  // namespace ecl

namespace ecl {

ecl_status scc_enqueue(const GraphDev& g, int* label, char* ws, Status* status, const DeviceInfo& dev,
                       cudaStream_t stream, int max_rounds, Marker mark) {
  Carve c{ws};
  SCCBufs b;
  scc_layout(c, g.n, g.m, &b);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, scc_solve, kTPB, 0) != cudaSuccess || occ < 1)
    return ECL_ERR_CUDA;
  const int coop_grid = dev.sms * occ;
  const int grid = dev.grid_blocks(kTPB);
  if (max_rounds <= 0 || max_rounds > b.max_rounds) max_rounds = b.max_rounds;

  if (cudaMemsetAsync(b.ctl, 0, sizeof(SCCCtl), stream) != cudaSuccess) return ECL_ERR_CUDA;
  if (cudaMemsetAsync(b.rounds, 0, sizeof(SCCRound) * (size_t)b.max_rounds, stream) != cudaSuccess)
    return ECL_ERR_CUDA;
  if (cudaMemsetAsync(b.hasin, 0, sizeof(int) * (size_t)g.n, stream) != cudaSuccess) return ECL_ERR_CUDA;
  if (cudaMemsetAsync(b.nchunks, 0, sizeof(int), stream) != cudaSuccess) return ECL_ERR_CUDA;
  const RowChunks rc{b.chunks, b.nchunks};
  ECL_LAUNCH(scc_mark, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, b.hasin, b.hasout, b.imax, b.omax, rc,
             status);
  ECL_LAUNCH(scc_mark_chunks, grid, kTPB, 0, stream, g.n, g.nindex, g.nlist, b.hasin, b.hasout, rc, status);
  mark();
  ECL_LAUNCH(scc_build, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, b.hasin, b.hasout, b.wlA, b.ctl);
  ECL_LAUNCH(scc_build_chunks, grid, kTPB, 0, stream, g.n, g.nindex, g.nlist, b.hasin, b.hasout, b.wlA, b.ctl, rc);
  mark();
  ECL_CUDA_TRY(launch_cooperative(scc_solve, coop_grid, kTPB, stream, g.n, b.wlA, b.wlB, b.imax, b.omax, label, b.ctl,
                                  b.rounds, max_rounds, status));
  mark();
  return ECL_OK;
}

}  // namespace ecl

extern "C" ecl_status ecl_scc(const ecl_graph_view* g, int32_t* label_out, ecl_opts* opts) {
  using namespace ecl;
  ecl_opts local{};
  if (!opts) opts = &local;
  if (!label_out) return ECL_ERR_INVALID_ARG;
  Solve s(g, opts);
  ecl_status st = s.begin(GraphNeeds{}, g ? scc_workspace_bytes(g->nodes, g->edges) : 0);
  if (st != ECL_OK) return s.finish(st);
  int* label = s.output(label_out, (size_t)s.n);
  if (!label) return s.finish(ECL_ERR_OOM);
  GraphDev gd;
  gd.n = s.n;
  gd.m = s.m;
  gd.nindex = s.nindex;
  gd.nlist = s.nlist;
  gd.flags = g->flags;
  s.start_timer();
  st = scc_enqueue(gd, label, s.ws, s.status, s.dev, s.stream, opts->max_rounds, Marker{&s});
  s.stop_timer();
  return s.finish(st);
}

extern "C" ecl_status ecl_compute_scc(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist,
                                      int32_t* label) {
  ecl_graph_view g{nodes, edges, nidx, nlist, nullptr, ECL_HOST, 0};
  ecl_opts o{};
  return ecl_scc(&g, label, &o);
}
