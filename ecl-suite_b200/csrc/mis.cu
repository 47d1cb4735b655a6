// Maximal independent set (ECL-MIS contract).
//
// Result contract (src/racefree/egr-input/MIS/ECL-MIS-atomic.cu): every
// vertex has a fixed priority byte (:118-136); findmins (:72-104) lets an
// undecided vertex join once every undecided neighbour has a lower
// (byte, id) and none is in.  With fixed priorities the set this converges to
// is the sequential greedy MIS in descending (byte, id) order, independent of
// the schedule, so the set below is bit-identical.
//
// B200 design:
//  * status bytes packed four per 32-bit word in the workspace (4.2 MB at
//    R-MAT-22, resident in the 126 MB L2); every shared access is a
//    device-scope relaxed atomic on the word;
//  * mis_init computes the priority bytes with the reference's fp32 formula
//    using explicit round-to-nearest intrinsics (no contraction);
//  * mis_run is ONE persistent cooperative launch (all blocks co-resident):
//    each warp sweeps its vertex groups until all are decided.  Lists of <= 32 entries are scanned by their own
//    lane with an early exit at the first blocker; longer lists are scanned
//    32 entries per step by the whole warp (two ballots per step); a joining
//    vertex claims itself with one CAS, then clears its neighbours' bytes
//    (fetch_and), so blocked neighbours see OUT without rescanning;
//  * a self-loop (the reference spins forever on one: v never outranks
//    itself) raises ECL_ERR_BAD_GRAPH when it is met; a sweep cap turns any
//    other non-converging input into ECL_ERR_NO_CONVERGENCE.
#include <algorithm>

#include "solvers.cuh"

namespace ecl {
namespace {

using namespace dev;

constexpr int kTPB = 256;
constexpr int kLaneMax = 32;  // default: lists of up to 32 entries per lane (a launch knob)
constexpr int kBatch = 4;  // list entries per lane whose loads are issued together
constexpr unsigned kIn = 0xfe;

__device__ __forceinline__ unsigned byte_of(unsigned word, int v) { return (word >> ((v & 3) * 8)) & 0xffu; }

__device__ __forceinline__ unsigned mis_priority(int v, int degree, float avg, float scaledavg) {
  if (degree <= 0) return kIn;
  // x = degree - hash(v) * 2^-32 ; res = rint(scaledavg / (avg + x))
  const float h = __fmul_rn(__uint2float_rn(ecl_hash((unsigned)v)), 0.00000000023283064365386962890625f);
  const float x = __fsub_rn(__int2float_rn(degree), h);
  const int res = __float2int_rn(__fdiv_rn(scaledavg, __fadd_rn(avg, x)));
  return (unsigned)((res + res) | 1) & 0xffu;
}

// Graph of union vertex v: the last g with vbase[g] <= v (binary search).
__device__ __forceinline__ int union_graph_of(const int* vbase, int ngraphs, int v) {
  int lo = 0, hi = ngraphs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&vbase[mid]) <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// For a union of graphs (vbase != nullptr) every vertex uses ITS graph's
// average degree and its local id, so each graph's bytes are exactly the ones
// a solve of that graph alone computes.
__global__ void __launch_bounds__(kTPB) mis_init(int n, int m, const int* __restrict__ nindex,
                                                 unsigned* __restrict__ st4, int nwords, const int* __restrict__ vbase,
                                                 const float* __restrict__ avgs, int ngraphs,
                                                 Status* __restrict__ status) {
  const float avg1 = __fdiv_rn(__int2float_rn(m), __int2float_rn(n));
  for (int w = blockIdx.x * kTPB + threadIdx.x; w < nwords; w += gridDim.x * kTPB) {
    unsigned word = 0;
    for (int k = 0; k < 4; k++) {
      const int v = 4 * w + k;
      unsigned b = 0;  // padding vertices are OUT
      if (v < n) {
        const int beg = __ldg(&nindex[v]), end = __ldg(&nindex[v + 1]);
        if (beg < 0 || end < beg || end > m) raise(status, ECL_ERR_BAD_GRAPH, v);
        float avg = avg1;
        int local = v;
        if (vbase) {
          const int g = union_graph_of(vbase, ngraphs, v);
          avg = __ldg(&avgs[g]);
          local = v - __ldg(&vbase[g]);
        }
        b = mis_priority(local, end - beg, avg, __fmul_rn(126.0f, avg));
      }
      word |= b << (8 * k);
    }
    st4[w] = word;  // race-free: thread-owned init, no reader in this launch
  }
}

// Outcome of scanning v's list.
enum : int { kWait = 0, kJoin = 1, kOut = 2 };

// Per-neighbour verdict: IN neighbour -> v is out; undecided neighbour with
// a higher (byte, id) -> v must wait; else no constraint.
__device__ __forceinline__ int mis_verdict(unsigned sb, unsigned b, int u, int v) {
  if (sb == kIn) return kOut;
  if ((sb & 1u) && (sb > b || (sb == b && u > v))) return kWait;
  return kJoin;
}

// Claims v as IN if its byte is still the undecided value b.
__device__ __forceinline__ bool mis_claim(unsigned* st4, int v, unsigned b) {
  unsigned* word = &st4[v >> 2];
  const int sh = (v & 3) * 8;
  unsigned cur = ld(word);
  while (byte_of(cur, v) == b) {
    const unsigned want = (cur & ~(0xffu << sh)) | (kIn << sh);
    const unsigned seen = cas(word, cur, want);
    if (seen == cur) return true;
    cur = seen;
  }
  return false;
}

__device__ __forceinline__ void mis_set_out(unsigned* st4, int u) { fetch_and(&st4[u >> 2], ~(0xffu << ((u & 3) * 8))); }

// A joined vertex sets its list entries nlist[i], i = i0, i0 + step, ...
// below end, out.  Their status words are read first (kBatch at a time) and
// only the entries not out yet take the atomic: a low-degree vertex that
// joins mostly neighbours hubs, whose words would otherwise take one atomic
// per joining neighbour.
__device__ __forceinline__ void mis_clear_list(unsigned* st4, const int* nlist, int i0, int end, int step, int n) {
  for (; i0 < end; i0 += step * kBatch) {
    int u[kBatch];
    unsigned w[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      const int i = i0 + k * step;
      u[k] = i < end ? __ldg(&nlist[i]) : -1;
    }
#pragma unroll
    for (int k = 0; k < kBatch; k++) w[k] = (unsigned)u[k] < (unsigned)n ? ld(&st4[u[k] >> 2]) : 0u;
#pragma unroll
    for (int k = 0; k < kBatch; k++)
      if ((unsigned)u[k] < (unsigned)n && byte_of(w[k], u[k]) != 0) mis_set_out(st4, u[k]);
  }
}

__global__ void __launch_bounds__(kTPB) mis_run(int n, int m, const int* __restrict__ nindex,
                                                const int* __restrict__ nlist, unsigned* __restrict__ st4,
                                                Status* __restrict__ status, int max_sweeps, int lane_max) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  int sweep = 0;
  // Bit g: this warp's g-th vertex group is fully decided and is skipped
  // without a load (groups beyond the 64th are re-read every sweep).  Late
  // sweeps then cost only the groups that still wait, not one L2 round trip
  // per group owned.
  unsigned long long done = 0;
  for (;; sweep++) {
    bool missing = false;
    int gi = 0;
    for (int base = warp * 32; base < n; base += nwarps * 32, gi++) {
      if (gi < 64 && ((done >> gi) & 1ull)) continue;
      const int v = base + lane;
      unsigned b = 0;
      if (v < n) b = byte_of(ld(&st4[v >> 2]), v);
      const bool und = (b & 1u) != 0;
      if (!__any_sync(kFull, und)) {
        if (gi < 64) done |= 1ull << gi;
        continue;
      }
      int beg = 0, end = 0;
      if (und) {
        beg = __ldg(&nindex[v]);
        end = __ldg(&nindex[v + 1]);
        if (beg < 0 || end < beg || end > m) beg = end = 0;  // reported by mis_init
      }
      const bool big = und && (end - beg) > lane_max;
      int verdict = kWait;
      if (und && !big) {
        verdict = kJoin;
        // kBatch entries at a time: their index loads, then their status
        // loads, are all in flight before the first verdict is needed
        for (int i0 = beg; i0 < end && verdict == kJoin; i0 += kBatch) {
          int u[kBatch];
          unsigned w[kBatch];
#pragma unroll
          for (int k = 0; k < kBatch; k++) u[k] = i0 + k < end ? __ldg(&nlist[i0 + k]) : -1;
#pragma unroll
          for (int k = 0; k < kBatch; k++) w[k] = (unsigned)u[k] < (unsigned)n ? ld(&st4[u[k] >> 2]) : 0u;
#pragma unroll
          for (int k = 0; k < kBatch; k++) {
            if (i0 + k >= end || verdict != kJoin) continue;
            if ((unsigned)u[k] >= (unsigned)n || u[k] == v) {  // out of range, or a self-loop
              raise(status, ECL_ERR_BAD_GRAPH, u[k]);
              continue;
            }
            const int r = mis_verdict(byte_of(w[k], u[k]), b, u[k], v);
            if (r != kJoin) verdict = r;
          }
        }
        if (verdict == kJoin) {
          if (mis_claim(st4, v, b)) mis_clear_list(st4, nlist, beg, end, 1, n);
        } else if (verdict == kOut) {
          mis_set_out(st4, v);
        }
      }
      // Long lists: the whole warp scans one list, 32 entries per step.
      unsigned todo = __ballot_sync(kFull, big);
      while (todo) {
        const int who = __ffs(todo) - 1;
        todo &= todo - 1;
        const int wv = __shfl_sync(kFull, v, who);
        const int wbeg = __shfl_sync(kFull, beg, who);
        const int wend = __shfl_sync(kFull, end, who);
        const unsigned wb = __shfl_sync(kFull, b, who);
        int wverdict = kJoin;
        for (int i0 = wbeg; i0 < wend; i0 += 32 * kBatch) {
          int u[kBatch];
          unsigned w[kBatch];
#pragma unroll
          for (int k = 0; k < kBatch; k++) {
            const int i = i0 + 32 * k + lane;
            u[k] = i < wend ? __ldg(&nlist[i]) : -1;
          }
#pragma unroll
          for (int k = 0; k < kBatch; k++) w[k] = (unsigned)u[k] < (unsigned)n ? ld(&st4[u[k] >> 2]) : 0u;
          bool out = false, wait = false;
#pragma unroll
          for (int k = 0; k < kBatch; k++) {
            if (i0 + 32 * k + lane >= wend) continue;
            if ((unsigned)u[k] < (unsigned)n && u[k] != wv) {
              const int r = mis_verdict(byte_of(w[k], u[k]), wb, u[k], wv);
              out |= r == kOut;
              wait |= r == kWait;
            } else {
              raise(status, ECL_ERR_BAD_GRAPH, u[k]);
            }
          }
          if (__any_sync(kFull, out)) {
            wverdict = kOut;
            break;
          }
          if (__any_sync(kFull, wait)) {
            wverdict = kWait;
            break;
          }
        }
        if (wverdict == kJoin) {
          bool claimed = false;
          if (lane == 0) claimed = mis_claim(st4, wv, wb);
          if (__shfl_sync(kFull, claimed, 0)) mis_clear_list(st4, nlist, wbeg + lane, wend, 32, n);
        } else if (wverdict == kOut && lane == 0) {
          mis_set_out(st4, wv);
        }
        if (lane == who) verdict = wverdict;
      }
      if (und && verdict == kWait) missing = true;
    }
    if (!__any_sync(kFull, missing)) break;
    if (sweep >= max_sweeps) {
      if (lane == 0) raise(status, ECL_ERR_NO_CONVERGENCE, warp);
      break;
    }
  }
  if (lane == 0) fetch_max(&status->rounds, sweep + 1);
}

__global__ void __launch_bounds__(kTPB) mis_emit(int n, const unsigned* __restrict__ st4,
                                                 unsigned char* __restrict__ out) {
  for (int v = blockIdx.x * kTPB + threadIdx.x; v < n; v += gridDim.x * kTPB) {
    out[v] = (unsigned char)byte_of(st4[v >> 2], v);  // race-free: st4 is final (mis_run finished)
  }
}

void mis_layout(Carve& c, int n, unsigned** st4) { *st4 = c.take<unsigned>((size_t)(n + 3) / 4); }

}  // namespace

size_t mis_workspace_bytes(int n, int m) {
  (void)m;
  Carve c;
  unsigned* st4;
  mis_layout(c, n, &st4);
  return c.bytes();
}

}  // namespace ecl

namespace ecl {

ecl_status mis_enqueue(const GraphDev& g, unsigned char* out, char* ws, Status* status, const DeviceInfo& dev,
                       cudaStream_t stream, int max_sweeps, const UnionInfo* uni, Marker mark) {
  Carve c{ws};
  unsigned* st4;
  mis_layout(c, g.n, &st4);
  const int nwords = (g.n + 3) / 4;
  const int grid = dev.grid_blocks(kTPB, g.n, g.m);
  const int* vbase = uni ? uni->vbase : nullptr;
  const float* avgs = uni ? uni->avg : nullptr;
  const int ngraphs = uni ? uni->ngraphs : 0;
  ECL_LAUNCH(mis_init, grid, kTPB, 0, stream, g.n, g.m, g.nindex, st4, nwords, vbase, avgs, ngraphs, status);
  mark();
  // Warps of mis_run wait (by sweeping) for vertices owned by other warps,
  // so all its blocks must be resident together: a cooperative launch
  // guarantees that even when other solves share the GPU (server slots).
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mis_run, kTPB, 0) != cudaSuccess || occ < 1)
    return ECL_ERR_CUDA;
  ECL_CUDA_TRY(launch_cooperative(mis_run, dev.sms * std::min(occ, dev.max_threads_per_sm / kTPB), kTPB, stream, g.n,
                                  g.m, g.nindex, g.nlist, st4, status, max_sweeps,
                                  bins_of(dev, Bins{kLaneMax, kBinChunk}).lane));
  mark();
  ECL_LAUNCH(mis_emit, grid, kTPB, 0, stream, g.n, st4, out);
  mark();
  return ECL_OK;
}

}  // namespace ecl

extern "C" ecl_status ecl_mis(const ecl_graph_view* g, uint8_t* status_out, ecl_opts* opts) {
  using namespace ecl;
  ecl_opts local{};
  if (!opts) opts = &local;
  if (!status_out) return ECL_ERR_INVALID_ARG;
  Solve s(g, opts);
  GraphNeeds needs;
  needs.symmetric = true;
  needs.no_self_loops = true;
  ecl_status st = s.begin(needs, g ? mis_workspace_bytes(g->nodes, g->edges) : 0);
  if (st != ECL_OK) return s.finish(st);
  unsigned char* out = s.output(status_out, (size_t)s.n);
  if (!out) return s.finish(ECL_ERR_OOM);
  GraphDev gd;
  gd.n = s.n;
  gd.m = s.m;
  gd.nindex = s.nindex;
  gd.nlist = s.nlist;
  gd.flags = g->flags;
  // Warps sweep asynchronously (one may sweep many times while it waits on a
  // slower warp's vertex), so the cap is a fixed backstop against inputs that
  // cannot converge, not a per-graph bound.
  const int max_sweeps = opts->max_rounds > 0 ? opts->max_rounds : (1 << 22);
  s.start_timer();
  st = mis_enqueue(gd, out, s.ws, s.status, s.dev, s.stream, max_sweeps, nullptr, Marker{&s});
  s.stop_timer();
  return s.finish(st);
}

extern "C" ecl_status ecl_compute_mis(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist,
                                      uint8_t* nstat) {
  ecl_graph_view g{nodes, edges, nidx, nlist, nullptr, ECL_HOST, 0};
  ecl_opts o{};
  return ecl_mis(&g, nstat, &o);
}
