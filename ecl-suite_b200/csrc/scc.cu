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
//  * scc_mark trims first: a vertex with no in-entry or no out-entry
//    (self-loops ignored) is its own SCC and contributes no edge.  The same
//    pass writes the int2 edge list in CSR positions -- slot i holds
//    (v, nlist[i]), or a dead slot for a self-loop or a bad id -- so the list
//    costs one streaming store per entry and no separate pass (on R-MAT nearly
//    every edge survives the trim, so compacting it would buy nothing).  Rows
//    are degree-binned (lane / warp / 256-entry chunk records), so hub rows
//    spread over all warps;
//  * scc_solve runs EVERY propagation sweep and every trimming round in one
//    cooperative persistent launch, separated by bounded grid barriers (the
//    reference pays a host round trip per propagation launch, :283-287).
//    In-max and out-max of a vertex share one 64-bit word (in-max high, out-
//    max low), like the reference's iomax, so an edge costs two word loads
//    plus two for the jumps io[in-max(v)] / io[out-max(w)] (both still valid
//    bounds, so values travel many hops per sweep); a raise is a 32-bit
//    atomic max on one half.  Trimmed vertices hold a DEAD word that every
//    sweep skips.  Each lane keeps kSweepBatch edges' loads in flight (a
//    launch knob: 1, 2 or 4; fewer edges a lane leave more lanes resident);
//  * rounds after the first sweep only the surviving edges (the edges whose
//    two ends share both values and are unresolved: io[v] == io[w]); every
//    sweep appends the edges it would keep, and the round's last sweep --
//    which raised nothing, so it read final words -- leaves the next round's
//    list without a separate pass;
//  * the final labels are written by the same launch (label = in-max).
#include "csr_bins.cuh"
#include "grid_sync.cuh"
#include "solvers.cuh"

namespace ecl {
namespace {

using namespace dev;

constexpr int kTPB = 256;
constexpr int kMaxSweeps = 1 << 16;
constexpr int kScanBatch = 4;  // list entries per lane whose loads are issued together

constexpr int kStamps = 256;

struct SCCCtl {
  GridBarrier bar;
  int pad[64];
  // %globaltimer at the start and after each grid barrier (the first
  // kStamps - 1): a time profile of sweeps, compactions and retirements that
  // costs one store per barrier
  unsigned long long stamp[kStamps];
  int changed[kMaxSweeps];   // per-sweep "something moved" flags
  int raised[kMaxSweeps];    // per-sweep counts of raises
  int kept[kMaxSweeps];      // per-sweep sizes of the list of edges a round keeps
  int again[kMaxSweeps];     // per-round "vertices left" flags, indexed by the round's last sweep
};

__device__ __forceinline__ unsigned long long scc_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// In-max (high half) and out-max (low half) of one vertex.
__device__ __forceinline__ unsigned long long io_pack(int in, int out) {
  return ((unsigned long long)(unsigned)in << 32) | (unsigned)out;
}
__device__ __forceinline__ int io_in(unsigned long long x) { return (int)(x >> 32); }
__device__ __forceinline__ int io_out(unsigned long long x) { return (int)(unsigned)x; }

// Raises the in-max (kIn) or out-max half of *p to val when `old`, the word
// last read, is below it; true when it was.  The raise is a 32-bit atomic max
// on that half: a word is read whole and raised per half, the reference's own
// access pattern (readFirst / writeFirstA on iomax, ECL-SCC_10-atomic.cu:145-
// 160), and a max never lowers a value another thread raised meanwhile.
template <bool kIn>
__device__ __forceinline__ bool io_raise(unsigned long long* p, unsigned long long old, int val) {
  if ((kIn ? io_in(old) : io_out(old)) >= val) return false;
  fetch_max(reinterpret_cast<int*>(p) + (kIn ? 1 : 0), val);  // little-endian: high half at +1
  return true;
}

// A vertex is live (can be in a non-trivial SCC) iff it has an in-entry and an
// out-entry other than self-loops.  Both facts share one flag word per vertex
// (kHasIn | kHasOut), so the liveness test is one load; scc_mark ORs kHasIn
// into flags[w] for every entry w != v and kHasOut into flags[v] for every v
// with such an entry; rows longer than bins.chunk go to chunk records.
constexpr int kHasIn = 1, kHasOut = 2;

// Marks kScanBatch entries w[k] (present where valid[k]) of v's list, at CSR
// positions j[k]: v has an out-entry and each w an in-entry (self-loops
// ignored), and slot j[k] of the edge list becomes (v, w) -- or a dead slot
// for a self-loop or an id out of range.  The flag words are read first and
// OR'ed only where kHasIn is still clear: R-MAT sends a large share of all
// entries to a few hub ids, whose words would otherwise take an atomic from
// every one of them.
__device__ __forceinline__ void scc_mark_batch(const bool (&valid)[kScanBatch], int v, const int (&w)[kScanBatch],
                                               const int (&j)[kScanBatch], int n, int* flags, int2* wl, bool& out,
                                               Status* status) {
  int f[kScanBatch];
#pragma unroll
  for (int k = 0; k < kScanBatch; k++)
    f[k] = (valid[k] && (unsigned)w[k] < (unsigned)n && w[k] != v) ? ld(&flags[w[k]]) : kHasIn;
#pragma unroll
  for (int k = 0; k < kScanBatch; k++) {
    if (!valid[k]) continue;
    const bool edge = (unsigned)w[k] < (unsigned)n && w[k] != v;
    if ((unsigned)w[k] >= (unsigned)n) raise(status, ECL_ERR_BAD_GRAPH, w[k]);
    if (edge) {
      if (!(f[k] & kHasIn)) fetch_or(&flags[w[k]], kHasIn);
      out = true;
    }
    __stcs(&wl[j[k]], edge ? make_int2(v, w[k]) : make_int2(-1, -1));
  }
}

__global__ void __launch_bounds__(kTPB) scc_mark(int n, int m, const int* __restrict__ nindex,
                                                 const int* __restrict__ nlist, int* __restrict__ flags,
                                                 int2* __restrict__ wl, RowChunks rc, Bins bins, bool vec,
                                                 Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    const int v = base + lane;
    int beg = 0, end = 0;
    if (v < n) csr_row(nindex, v, m, beg, end, status);
    const int deg = end - beg;
    push_chunks_warp(rc, bins.chunk, deg > bins.chunk, v, beg, end, status);
    bool out = false;
    const bool lanelvl = deg <= bins.lane;
    const int kmax = __reduce_max_sync(kFull, lanelvl ? deg : 0);
    for (int k0 = 0; k0 < kmax; k0 += kScanBatch) {
      int w[kScanBatch], j[kScanBatch];
      bool valid[kScanBatch];
#pragma unroll
      for (int k = 0; k < kScanBatch; k++) {
        valid[k] = lanelvl && k0 + k < deg;
        j[k] = beg + k0 + k;
        w[k] = valid[k] ? __ldg(&nlist[j[k]]) : 0;
      }
      scc_mark_batch(valid, v, w, j, n, flags, wl, out, status);
    }
    unsigned todo = __ballot_sync(kFull, deg > bins.lane && deg <= bins.chunk);
    while (todo) {
      const int who = __ffs(todo) - 1;
      todo &= todo - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      bool wout = false;
      warp_row(wbeg, wend, m, vec, nlist, [&](const int (&j)[4], const int (&w)[4], const bool (&valid)[4]) {
        scc_mark_batch(valid, wv, w, j, n, flags, wl, wout, status);
      });
      if (__any_sync(kFull, wout) && lane == who) out = true;
    }
    if (v < n && deg <= bins.chunk && out) fetch_or(&flags[v], kHasOut);  // long rows: scc_mark_chunks
  }
}

__global__ void __launch_bounds__(kTPB) scc_mark_chunks(int n, int m, const int* __restrict__ nindex,
                                                        const int* __restrict__ nlist, int* __restrict__ flags,
                                                        int2* __restrict__ wl, RowChunks rc, int chunk, bool vec,
                                                        Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int total = chunk_total(rc);
  for (int c = warp; c < total; c += nwarps) {
    const int2 r = rc.rec[c];
    const int end = min(r.y + chunk, __ldg(&nindex[r.x + 1]));
    bool out = false;
    warp_row(r.y, end, m, vec, nlist, [&](const int (&j)[4], const int (&w)[4], const bool (&valid)[4]) {
      scc_mark_batch(valid, r.x, w, j, n, flags, wl, out, status);
    });
    if (__any_sync(kFull, out) && lane == 0) fetch_or(&flags[r.x], kHasOut);
  }
}

// Word of a trimmed vertex: it is its own SCC, and sweeps skip its edges.
constexpr unsigned long long kDead = ~0ull;
// Edges per lane whose loads are issued together in a sweep: a template
// argument (1, 2 or 4), with the blocks per SM the register budget allows.
constexpr int kSweepBatchDefault = 1;  // the measured best at R-MAT-22 (2.16 ms vs 2.24 / 2.40)
template <int kSweepBatch>
struct SweepOcc {
  static constexpr int blocks = kSweepBatch == 1 ? 8 : (kSweepBatch == 2 ? 6 : 4);
};

// Round 0 sweeps the CSR-position edge list of `m0` slots (dead slots have
// x < 0); later rounds sweep the compacted survivors.
template <int kSweepBatch>
__global__ void __launch_bounds__(kTPB, SweepOcc<kSweepBatch>::blocks) scc_solve(int n, int m0, int2* __restrict__ wlA, int2* __restrict__ wlB,
                                                  const int* __restrict__ flags, unsigned long long* __restrict__ io,
                                                  int* __restrict__ label, SCCCtl* __restrict__ ctl,
                                                  int max_rounds,
                                                  Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int tid = blockIdx.x * kTPB + threadIdx.x;
  const int nthreads = gridDim.x * kTPB;
  int nstamp = 0;  // thread 0: stamps written
  if (tid == 0) ctl->stamp[0] = scc_now();
  // 0. live vertices start at (v, v); trimmed ones are DEAD
  for (int v = tid; v < n; v += nthreads)
    io[v] = __ldg(&flags[v]) == (kHasIn | kHasOut) ? io_pack(v, v) : kDead;  // race-free: owned, barrier next
  if (!grid_sync(&ctl->bar, status)) return;
  if (tid == 0 && ++nstamp < kStamps) ctl->stamp[nstamp] = scc_now();
  int size = m0;
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
      int raises = 0;
      // Append the edges this round keeps during the sweep (below) once the
      // last sweep raised few words: the values are then close to final, and
      // few edges look kept.  Earlier, transient agreement makes millions of
      // edges look kept, and their appends would cost more than the
      // separate pass they save.
      const bool spec = sweep > 0 && ld(&ctl->raised[sweep - 1]) <= (m0 >> 6);
      // The jump targets converge on a few vertices (the largest SCC's
      // maximum id first of all), so every thread keeps its last jump of
      // each kind: a repeated target reuses the value instead of loading the
      // same word as every other edge.  A value read earlier is a smaller
      // but still valid bound (in-max and out-max only grow).
      int c_iv = -1, c_in = -1, c_ow = -1, c_out = -1;
      // Whole warps step together over kSweepBatch slices of 32 consecutive
      // slots; in CSR order neighbouring lanes mostly share v, so the out-max
      // raises of v are combined per slice (__match_any_sync + max) into one
      // atomic instead of up to 32 on one address.  Each lane's edge records,
      // then their io words, then the jump words are loaded before any is
      // used.
      for (int i0 = (tid - lane) * kSweepBatch; i0 < size; i0 += nthreads * kSweepBatch) {
        int2 e[kSweepBatch];
#pragma unroll
        for (int k = 0; k < kSweepBatch; k++) {
          const int i = i0 + 32 * k + lane;
          e[k] = i < size ? __ldcs(&cur[i]) : make_int2(-1, -1);
          if ((unsigned)e[k].x >= (unsigned)n || (unsigned)e[k].y >= (unsigned)n) e[k] = make_int2(-1, -1);
        }
        unsigned long long A[kSweepBatch], B[kSweepBatch];
#pragma unroll
        for (int k = 0; k < kSweepBatch; k++) {
          A[k] = e[k].x >= 0 ? ld(&io[e[k].x]) : kDead;
          B[k] = e[k].x >= 0 ? ld(&io[e[k].y]) : kDead;
        }
        // jumps not covered by the memo load only the half they need (in-max
        // is the high word); -1 = not loaded (live values are >= 0)
        int iv[kSweepBatch], ow[kSweepBatch], ji[kSweepBatch], jo[kSweepBatch];
#pragma unroll
        for (int k = 0; k < kSweepBatch; k++) {
          const bool live = A[k] != kDead && B[k] != kDead;
          iv[k] = live ? io_in(A[k]) : -1;
          ow[k] = live ? io_out(B[k]) : -1;
          ji[k] = (live && iv[k] != e[k].x && iv[k] != c_iv) ? ld(reinterpret_cast<const int*>(&io[iv[k]]) + 1) : -1;
          jo[k] = (live && ow[k] != e[k].y && ow[k] != c_ow) ? ld(reinterpret_cast<const int*>(&io[ow[k]])) : -1;
        }
#pragma unroll
        for (int k = 0; k < kSweepBatch; k++) {
          if (iv[k] >= 0 && iv[k] != e[k].x) {
            if (ji[k] >= 0) {
              c_iv = iv[k];
              c_in = ji[k];
            }
            if (iv[k] == c_iv) iv[k] = max(iv[k], c_in);
          }
          if (ow[k] >= 0 && ow[k] != e[k].y) {
            if (jo[k] >= 0) {
              c_ow = ow[k];
              c_out = jo[k];
            }
            if (ow[k] == c_ow) ow[k] = max(ow[k], c_out);
          }
          if (iv[k] >= 0 && io_raise<true>(&io[e[k].y], B[k], iv[k])) raises++;
          const int v = iv[k] >= 0 ? e[k].x : -1;
          const unsigned grp = __match_any_sync(kFull, v);
          const int gow = __reduce_max_sync(grp, ow[k]);
          if (v >= 0 && lane == __ffs(grp) - 1 && io_raise<false>(&io[v], A[k], gow)) raises++;
        }
        // The edges the round keeps (endpoints unresolved and in full
        // agreement), judged by the words this sweep loaded: only the last
        // sweep's list is used, and that sweep raised nothing, so its words
        // were final.  This saves a separate pass over the list and its words.
        if (spec) {
#pragma unroll
          for (int k = 0; k < kSweepBatch; k++) {
            const bool keep = A[k] != kDead && io_in(A[k]) != io_out(A[k]) && A[k] == B[k];
            const int at = warp_append(&ctl->kept[sweep], keep);
            if (keep && at < m0) nxt[at] = e[k];
          }
        }
      }
      // one count per block (a flag per warp would queue at one word)
      __shared__ int s_raises;
      if (threadIdx.x == 0) s_raises = 0;
      __syncthreads();
      const int wr = __reduce_add_sync(kFull, raises);
      if (lane == 0 && wr) atomicAdd(&s_raises, wr);  // shared memory
      __syncthreads();
      if (threadIdx.x == 0 && s_raises) {
        fetch_add(&ctl->raised[sweep], s_raises);
        st(&ctl->changed[sweep], 1);
      }
      if (!grid_sync(&ctl->bar, status)) return;
      if (tid == 0 && ++nstamp < kStamps) ctl->stamp[nstamp] = scc_now();
      const bool again = ld(&ctl->changed[sweep]) != 0;
      sweep++;
      if (!again) {
        if (spec) break;
        // 1b. the last sweep kept no list: keep the edges whose endpoints are
        // unresolved and agree, in a pass of its own
        for (int i0 = tid - lane; i0 < size; i0 += nthreads) {
          const int i = i0 + lane;
          bool keep = false;
          int2 e = make_int2(0, 0);
          if (i < size) {
            e = cur[i];
            if ((unsigned)e.x < (unsigned)n && (unsigned)e.y < (unsigned)n) {
              const unsigned long long A = ld(&io[e.x]);
              keep = A != kDead && io_in(A) != io_out(A) && A == ld(&io[e.y]);
            }
          }
          const int at = warp_append(&ctl->kept[sweep - 1], keep);
          if (keep && at < m0) nxt[at] = e;
        }
        if (!grid_sync(&ctl->bar, status)) return;
        break;
      }
    }
    // 2. retire resolved (and trimmed) vertices, reset the rest to their own id
    bool again = false;
    for (int v = tid; v < n; v += nthreads) {
      const unsigned long long A = ld(&io[v]);
      if (A == kDead) {
        label[v] = v;  // race-free: the output, thread-owned and never read here
      } else if (io_in(A) == io_out(A)) {
        label[v] = io_in(A);  // race-free: as above
      } else {
        st(&io[v], io_pack(v, v));
        again = true;
      }
    }
    if (__any_sync(kFull, again) && lane == 0) st(&ctl->again[sweep - 1], 1);
    if (!grid_sync(&ctl->bar, status)) return;
    if (tid == 0 && ++nstamp < kStamps) ctl->stamp[nstamp] = scc_now();
    if (!ld(&ctl->again[sweep - 1])) break;
    size = min(ld(&ctl->kept[sweep - 1]), m0);
    int2* t = cur;
    cur = nxt;
    nxt = t;
  }
  if (tid == 0) st(&status->rounds, sweep);
}

struct SCCBufs {
  SCCCtl* ctl;
  int* flags;
  int* nchunks;
  int2* chunks;
  unsigned long long* io;
  int2* wlA;
  int2* wlB;
  int max_rounds;
};

void scc_layout(Carve& c, int n, int m, SCCBufs* b) {
  b->ctl = c.take<SCCCtl>(1);
  b->max_rounds = n + 1;
  b->flags = c.take<int>((size_t)n);
  b->nchunks = c.take<int>(64);
  b->chunks = c.take<int2>(row_chunk_capacity(m, kMinChunk));
  b->io = c.take<unsigned long long>((size_t)n);
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
  const int batch = dev.scc_sweep_batch > 0 ? dev.scc_sweep_batch : kSweepBatchDefault;
  void (*solve)(int, int, int2*, int2*, const int*, unsigned long long*, int*, SCCCtl*, int, Status*) =
      batch == 1 ? scc_solve<1> : (batch == 4 ? scc_solve<4> : scc_solve<2>);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, solve, kTPB, 0) != cudaSuccess || occ < 1)
    return ECL_ERR_CUDA;
  const int coop_grid = dev.sms * occ;
  const int grid = dev.grid_blocks(kTPB, g.n, g.m);
  if (max_rounds <= 0 || max_rounds > b.max_rounds) max_rounds = b.max_rounds;

  if (cudaMemsetAsync(b.ctl, 0, sizeof(SCCCtl), stream) != cudaSuccess) return ECL_ERR_CUDA;
  if (cudaMemsetAsync(b.flags, 0, sizeof(int) * (size_t)g.n, stream) != cudaSuccess) return ECL_ERR_CUDA;
  if (cudaMemsetAsync(b.nchunks, 0, sizeof(int), stream) != cudaSuccess) return ECL_ERR_CUDA;
  const RowChunks rc{b.chunks, b.nchunks, (int)row_chunk_capacity(g.m, kMinChunk)};
  // chunk records of 128 entries by default: the mark pass measured faster
  // with them than with 256 (R-MAT-22: 0.65 vs 0.72 ms)
  const Bins bins = bins_of(dev, Bins{kBinLane, kMinChunk});
  const bool vec = (reinterpret_cast<uintptr_t>(g.nlist) & 15) == 0 && dev.row_vec;  // 16-byte row loads
  ECL_LAUNCH(scc_mark, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, b.flags, b.wlA, rc, bins, vec, status);
  ECL_LAUNCH(scc_mark_chunks, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, b.flags, b.wlA, rc, bins.chunk, vec,
             status);
  mark();
  ECL_CUDA_TRY(launch_cooperative(solve, coop_grid, kTPB, stream, g.n, g.m, b.wlA, b.wlB, b.flags, b.io, label, b.ctl,
                                  max_rounds, status));
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
