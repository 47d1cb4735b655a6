// Minimum spanning forest (ECL-MST contract).
//
// Result contract (src/racefree/egr-input/MST/ECL-MST_10-atomic.cu): each
// undirected edge is represented by its v<n CSR entry j (:203) and ordered by
// the 64-bit key (weight << 32) | j (:248); with unique keys the minimum
// spanning forest is unique, so in_mst[] and the total weight equal cpuMST's
// Kruskal result (:112-154) bit for bit.  Light edges (weight <= a sampled
// threshold) are contracted first, then the rest (:331-360); any threshold
// gives the same forest.
//
// B200 design:
//  * mst_threshold: one block samples 1024 weights on the device and picks
//    the quantile that leaves ~0.75 n light CSR entries (no host round
//    trip).  Fewer light edges than the reference's 3n: on R-MAT-22 the light
//    Boruvka pass then runs on ~1.6 M instead of ~6.4 M edges, and the
//    flattened heavy pass absorbs the rest (factor 3 -> 0.75: MST 6.5 -> 5.0 ms);
//  * mst_scan: builds a worklist of int4 {a, b, weight, j} from the CSR,
//    lane-level for lists <= 32 entries, warp-level up to 256, chunk
//    records beyond; appends are staged per warp in shared memory and
//    reserved in the global list with one atomic per ~kStage entries;
//    the heavy pass drops entries whose endpoints are already joined (the
//    forest is flattened by pointer jumping first, so a root is one load);
//  * mst_boruvka: ALL Boruvka rounds in one cooperative persistent launch
//    (2 bounded grid barriers per round): phase A re-roots each edge, drops
//    intra-component edges and atomicMin's its key into both roots; phase B
//    joins every edge that is the minimum of one of its roots and flags it.
//    Round 0 takes the scan's list as it stands (its entries already join
//    two roots): it publishes the keys and joins along it without re-rooting
//    or copying 10.6 M entries (heavy pass at R-MAT-22: 0.79 -> 0.74 ms).
//    Per warp, every root is found, reset, loaded and min-published once
//    (__match_any_sync groups), and per block every root of a large
//    component once: a shared-memory table of roots takes the key minimums,
//    serves phase B's key reads and ends phase A's finds without a load of
//    the root's word.  Middle rounds give a few hundred large components most
//    of the edges, and per-warp accesses to their words queue at their L2
//    slices (R-MAT-22 light pass: 1.17 -> 0.96 ms).
//    minv is double-buffered so its reset (a streaming pass over the
//    vertices) rides along with phase A instead of costing a third barrier; per-round sizes live in a counter array, so
//    no counter is ever reset concurrently with its use.
#include <cooperative_groups.h>

#include "csr_bins.cuh"
#include "grid_sync.cuh"
#include "solvers.cuh"

namespace ecl {
namespace {

using namespace dev;
typedef unsigned long long u64;

constexpr int kTPB = 256;
// Default degree bins: rows of <= 32 entries per lane, chunk records of 256
// entries (R-MAT's heavy low-id rows share warp groups: keep warp rows short).
constexpr Bins kMstBins{32, 256};
constexpr int kMaxRounds = 64;
constexpr int kSamples = 1024;

struct MSTCtl {
  GridBarrier bar;
  int wlcount[2][kMaxRounds + 2];  // [pass][round] sizes
  int nchunks;
  int threshold;
  int filter;
  int pad;
  u64 total;
  // %globaltimer when each pass started and after each of its barriers
  // (phase A of round r ends at [2r + 1], phase B at [2r + 2]): a per-round
  // time profile that costs one store per barrier.
  u64 stamp[2][2 * kMaxRounds + 2];
};

__device__ __forceinline__ u64 mst_now() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int mst_find(int v, int* parent) {
  int cur = ld(&parent[v]);
  if (cur == v) return v;
  int prev = v, next;
  while (cur != (next = ld(&parent[cur]))) {
    st(&parent[prev], next);
    prev = cur;
    cur = next;
  }
  return cur;
}

__device__ __forceinline__ void mst_join(int a, int b, int* parent) {
  while (true) {
    a = mst_find(a, parent);
    b = mst_find(b, parent);
    if (a == b) return;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    if (cas(&parent[a], a, b) == a) return;
  }
}

// parent[v] = root(v) between the passes, so the heavy scan reads each
// entry's root with one load.  Pointer jumping: each thread rewrites only its
// own parent[v] (parents point at smaller ids), stepping to the parent of its
// current target, which its own thread is shortening at the same time.
__global__ void __launch_bounds__(kTPB) mst_flatten(int n, int* __restrict__ parent) {
  for (int v = blockIdx.x * kTPB + threadIdx.x; v < n; v += gridDim.x * kTPB) {
    int p = ld(&parent[v]);
    if (p == v) continue;
    int pp;
    while ((pp = ld(&parent[p])) < p) {
      st(&parent[v], pp);
      p = pp;
    }
  }
}

__global__ void mst_init(int n, int* __restrict__ parent, u64* __restrict__ minv) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    // race-free: thread-owned init, no reader in this launch
    parent[v] = v;
    minv[v] = ~0ull;
    minv[n + v] = ~0ull;
  }
}

// Threshold = the k-th smallest of kSamples sampled weights, k chosen so the
// light pass keeps about light_factor * n of the m entries (the reference
// aims at 3n, ECL-MST_10-atomic.cu:450-459; the batched engine's autotuner
// may pick another factor -- the forest does not depend on it).  No
// filtering when edges/nodes < 4.
__global__ void __launch_bounds__(kSamples) mst_threshold(int n, int m, const int* __restrict__ eweight,
                                                         MSTCtl* __restrict__ ctl, float light_factor) {
  __shared__ int s[kSamples];
  const int t = threadIdx.x;
  const bool filter = m > 0 && (m / n) >= 4;
  s[t] = filter ? __ldg(&eweight[ecl_hash((unsigned)t * 2654435761u + 12345u) % (unsigned)m]) : 0;
  __syncthreads();
  for (int k = 2; k <= kSamples; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int p = t ^ j;
      if (p > t) {
        const int a = s[t], b = s[p];
        const bool up = (t & k) == 0;
        if ((a > b) == up) {
          s[t] = b;
          s[p] = a;
        }
      }
      __syncthreads();
    }
  }
  if (t == 0) {
    ctl->filter = filter ? 1 : 0;
    if (filter) {
      const double frac = (double)light_factor * (double)n / (double)m;
      const int k = min(kSamples - 1, (int)(frac * kSamples));
      ctl->threshold = s[k];
    } else {
      ctl->threshold = 0x7fffffff;
    }
  }
}

template <bool kLight>
__device__ __forceinline__ bool mst_keep(int w, int thr) {
  return kLight ? (w <= thr) : (w > thr);
}

// Slots per warp in the shared-memory staging of worklist appends.
constexpr int kStage = 128;
// Worklists are 16 B per edge (100 MB each for R-MAT-22's light edges):
// they are written and read with evict-first hints so parent[] and the key
// arrays, which Boruvka reads at random, stay in L2.
typedef WarpStage<int4, kStage, true> Stage;

// Entries per lane whose loads are issued together in the scans.
constexpr int kScanBatch = 4;

// Emits the worklist entries for kScanBatch CSR entries of vertex v per lane
// (rv = v's root in the heavy pass): entry k of this lane is j0 + k * stride,
// present when `active` and below jend.  All index loads, then the weight
// loads of the v < u entries, then (heavy pass) their roots are in flight
// together before any is used; every lane pushes kScanBatch times.
template <bool kLight>
__device__ __forceinline__ void mst_emit_batch(int j0, int stride, int jend, bool active, int v, int rv, int n,
                                               const int* nlist, const int* eweight, int thr, const int* parent,
                                               Stage& stg, int4* wl, int* cnt, int cap, bool& overflow,
                                               Status* status) {
  int u[kScanBatch], w[kScanBatch], ru[kScanBatch];
#pragma unroll
  for (int k = 0; k < kScanBatch; k++) {
    const int j = j0 + k * stride;
    u[k] = (active && j < jend) ? __ldg(&nlist[j]) : -1;
  }
  if (kLight) {
#pragma unroll
    for (int k = 0; k < kScanBatch; k++) {
      const int j = j0 + k * stride;
      w[k] = ((unsigned)u[k] < (unsigned)n && u[k] > v) ? __ldg(&eweight[j]) : 0;
      ru[k] = -1;
    }
  } else {
    // Heavy pass: the root first (flat after mst_flatten), the weight only
    // for entries between two components.  The light pass joined the ends of
    // every light entry (and checked every weight), so those are all heavy,
    // and the ~80 % of entries inside one component cost no weight load.
#pragma unroll
    for (int k = 0; k < kScanBatch; k++)
      ru[k] = ((unsigned)u[k] < (unsigned)n && u[k] > v) ? ld(&parent[u[k]]) : -1;
#pragma unroll
    for (int k = 0; k < kScanBatch; k++) {
      const int j = j0 + k * stride;
      w[k] = (ru[k] >= 0 && ru[k] != rv) ? __ldg(&eweight[j]) : 0;
    }
  }
#pragma unroll
  for (int k = 0; k < kScanBatch; k++) {
    const int j = j0 + k * stride;
    bool keep = false;
    int4 e = make_int4(0, 0, 0, 0);
    if (active && j < jend) {
      if ((unsigned)u[k] >= (unsigned)n) {
        raise(status, ECL_ERR_BAD_GRAPH, u[k]);
      } else if (u[k] > v) {
        if (w[k] < 0) {
          raise(status, ECL_ERR_BAD_GRAPH, j);
        } else if (kLight) {
          if (mst_keep<true>(w[k], thr)) {
            keep = true;
            e = make_int4(v, u[k], w[k], j);
          }
        } else if (ru[k] != rv) {
          keep = true;
          e = make_int4(rv, ru[k], w[k], j);
        }
      }
    }
    stg.push(keep, e, wl, cnt, cap, overflow);
  }
}

// Emits the worklist entries of one warp-walked row segment [jb, je) of v.
// With `vec` (nlist and eweight 16-byte aligned) the segment is walked in
// 16-byte-aligned quads of entries, one quad a lane (128 entries a warp
// step): one 16-byte load of nlist and, when any of the quad's entries is a
// v < u entry, one of eweight.  The quads at the segment's ends are masked to
// it, and a quad reaching past the arrays' m entries is read entry by entry.
// Without `vec` the scalar mst_emit_batch walks it.  All lanes call.
template <bool kLight>
__device__ __forceinline__ void mst_emit_row(int jb, int je, int m, bool vec, int v, int rv, int n, const int* nlist,
                                             const int* eweight, int thr, const int* parent, Stage& stg, int4* wl,
                                             int* cnt, int cap, bool& overflow, Status* status) {
  const int lane = threadIdx.x & 31;
  if (!vec) {
    for (int i0 = jb; i0 < je; i0 += 32 * kScanBatch)
      mst_emit_batch<kLight>(i0 + lane, 32, je, true, v, rv, n, nlist, eweight, thr, parent, stg, wl, cnt, cap,
                             overflow, status);
    return;
  }
  for (int i0 = jb & ~3; i0 < je; i0 += 4 * 32) {
    const int q = i0 + 4 * lane;  // this lane's quad [q, q + 4)
    const bool whole = q + 4 <= m && q < je;
    bool valid[4];
    int u[4], w[4] = {0, 0, 0, 0}, ru[4];
#pragma unroll
    for (int k = 0; k < 4; k++) valid[k] = q + k >= jb && q + k < je;
    if (whole) {
      const int4 x = __ldg(reinterpret_cast<const int4*>(nlist + q));
      u[0] = x.x, u[1] = x.y, u[2] = x.z, u[3] = x.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) u[k] = valid[k] ? __ldg(&nlist[q + k]) : -1;
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (!valid[k]) u[k] = -1;
    if (u[0] > v || u[1] > v || u[2] > v || u[3] > v) {
      if (whole) {
        const int4 y = __ldg(reinterpret_cast<const int4*>(eweight + q));
        w[0] = y.x, w[1] = y.y, w[2] = y.z, w[3] = y.w;
      } else {
#pragma unroll
        for (int k = 0; k < 4; k++) w[k] = u[k] > v ? __ldg(&eweight[q + k]) : 0;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      ru[k] = (!kLight && (unsigned)u[k] < (unsigned)n && u[k] > v && mst_keep<false>(w[k], thr))
                  ? ld(&parent[u[k]])  // flat after mst_flatten
                  : -1;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int j = q + k;
      bool keep = false;
      int4 e = make_int4(0, 0, 0, 0);
      if (valid[k]) {
        if ((unsigned)u[k] >= (unsigned)n) {
          raise(status, ECL_ERR_BAD_GRAPH, u[k]);
        } else if (u[k] > v) {
          if (w[k] < 0) {
            raise(status, ECL_ERR_BAD_GRAPH, j);
          } else if (mst_keep<kLight>(w[k], thr)) {
            if (kLight) {
              keep = true;
              e = make_int4(v, u[k], w[k], j);
            } else {
              keep = ru[k] != rv;
              e = make_int4(rv, ru[k], w[k], j);
            }
          }
        }
      }
      stg.push(keep, e, wl, cnt, cap, overflow);
    }
  }
}

// More v<n entries than the worklist holds: an asymmetric graph flagged
// symmetric.
__device__ __forceinline__ void mst_overflow(bool overflow, Status* status) {
  if (__any_sync(kFull, overflow) && (threadIdx.x & 31) == 0) raise(status, ECL_ERR_BAD_GRAPH, -2);
}

template <bool kLight>
__global__ void __launch_bounds__(kTPB) mst_scan(int n, int m, const int* __restrict__ nindex,
                                                 const int* __restrict__ nlist, const int* __restrict__ eweight,
                                                 int* __restrict__ parent, int4* __restrict__ wl, int cap,
                                                 MSTCtl* __restrict__ ctl, int2* __restrict__ chunks, Bins bins,
                                                 bool vec, Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int thr = ctl->threshold;
  int* cnt = &ctl->wlcount[kLight ? 0 : 1][0];
  __shared__ int4 stage_buf[kTPB / 32][kStage];
  Stage stg{stage_buf[threadIdx.x >> 5]};
  bool overflow = false;
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
    const int deg = end - beg;
    const bool lanelvl = deg > 0 && deg <= bins.lane;
    int rv = v;
    if (!kLight && deg > 0 && v < n) rv = ld(&parent[v]);
    if (kLight)  // chunk records are built once, in the light pass
      push_chunks_warp(RowChunks{chunks, &ctl->nchunks, (int)row_chunk_capacity(m, kMinChunk)}, bins.chunk,
                       deg > bins.chunk, v, beg, end, status);
    // lane level: all lanes step through offset k together
    const int kmax = __reduce_max_sync(kFull, lanelvl ? deg : 0);
    for (int k0 = 0; k0 < kmax; k0 += kScanBatch)
      mst_emit_batch<kLight>(beg + k0, 1, end, lanelvl, v, rv, n, nlist, eweight, thr, parent, stg, wl, cnt, cap,
                             overflow, status);
    // warp level
    unsigned todo = __ballot_sync(kFull, deg > bins.lane && deg <= bins.chunk);
    while (todo) {
      const int who = __ffs(todo) - 1;
      todo &= todo - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wrv = __shfl_sync(kFull, rv, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      mst_emit_row<kLight>(wbeg, wend, m, vec, wv, wrv, n, nlist, eweight, thr, parent, stg, wl, cnt, cap, overflow,
                           status);
    }
  }
  stg.flush(wl, cnt, cap, overflow);
  mst_overflow(overflow, status);
  // chunk records (hubs): the light pass sees them only after all warps
  // passed the vertex loop, so they are handled by mst_chunks.
}

template <bool kLight>
__global__ void __launch_bounds__(kTPB) mst_chunks(int n, int m, const int* __restrict__ nindex,
                                                   const int* __restrict__ nlist,
                                                   const int* __restrict__ eweight, int* __restrict__ parent,
                                                   int4* __restrict__ wl, int cap, MSTCtl* __restrict__ ctl,
                                                   const int2* __restrict__ chunks, int chunk_cap, int chunk,
                                                   bool vec, Status* __restrict__ status) {
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int thr = ctl->threshold;
  int* cnt = &ctl->wlcount[kLight ? 0 : 1][0];
  const int total = min((unsigned)ctl->nchunks, (unsigned)chunk_cap);
  __shared__ int4 stage_buf[kTPB / 32][kStage];
  Stage stg{stage_buf[threadIdx.x >> 5]};
  bool overflow = false;
  for (int c = warp; c < total; c += nwarps) {
    const int2 rec = chunks[c];
    const int v = rec.x;
    const int end = min(rec.y + chunk, __ldg(&nindex[v + 1]));
    const int rv = kLight ? v : ld(&parent[v]);
    mst_emit_row<kLight>(rec.y, end, m, vec, v, rv, n, nlist, eweight, thr, parent, stg, wl, cnt, cap, overflow, status);
  }
  stg.flush(wl, cnt, cap, overflow);
  mst_overflow(overflow, status);
}

// Lowers mcur[root] to the smallest (weight << 32 | j) key among the lanes
// of the warp that hold `root` and keep their edge: one atomic per root per
// warp.  Late rounds give one giant component most of the edges, and an
// atomic (or load) per edge on its root would queue at one L2 slice.  All
// lanes call.
// One-entry memo of a per-thread lookup (key -> value); key -1 = empty.
struct MstMemo {
  int key = -1;
  u64 val = 0;
};

template <typename T>
using bref = cuda::atomic_ref<T, cuda::thread_scope_block>;

// A block's table of component roots (open addressing, kRootProbes probes)
// with the smallest key the block has for each.  Once a few hundred large
// components hold most of the edges (R-MAT-22's light pass has ~250 in its
// fourth round), every warp of the grid publishes to and reads the same few
// hundred key words, and their L2 slices serialise the traffic: sending every
// atomic there instead of loading first makes the pass 35 % slower.  The
// table lowers a root's key in shared memory, publishes it with one atomic
// per block, and serves phase B's reads of it from shared memory.  A root
// whose probes meet only other roots goes to global memory directly.
constexpr int kRootSlots = 1024;
constexpr int kRootProbes = 4;

struct RootTable {
  int* root;  // kRootSlots entries, -1 = empty
  u64* key;

  __device__ static int first_slot(int r) { return (int)(((unsigned)r * 2654435761u) >> 22); }

  // All threads of the block call, between block barriers.
  __device__ void reset() {
    for (int i = threadIdx.x; i < kRootSlots; i += blockDim.x) {
      root[i] = -1;  // race-free: block-owned, barrier-separated from every reader
      key[i] = ~0ull;
    }
  }
  // Slot of r, claimed if r is absent and a probed slot is free; -1 if not.
  __device__ int claim(int r) {
    int h = first_slot(r);
    for (int p = 0; p < kRootProbes; p++, h = (h + 1) & (kRootSlots - 1)) {
      int c = bref<int>(root[h]).load(cuda::memory_order_relaxed);
      if (c == -1 && bref<int>(root[h]).compare_exchange_strong(c, r, cuda::memory_order_relaxed)) return h;
      if (c == r) return h;
    }
    return -1;
  }
  // Whether r has a slot, while claims may run (phase A).
  __device__ bool has(int r) const {
    int h = first_slot(r);
    for (int p = 0; p < kRootProbes; p++, h = (h + 1) & (kRootSlots - 1)) {
      const int c = bref<int>(root[h]).load(cuda::memory_order_relaxed);
      if (c == r) return true;
      if (c == -1) return false;
    }
    return false;
  }
  // Slot of r, or -1 (read-only phase: no claims run).
  __device__ int find(int r) const {
    int h = first_slot(r);
    for (int p = 0; p < kRootProbes; p++, h = (h + 1) & (kRootSlots - 1)) {
      const int c = root[h];  // race-free: no claim runs while find() does
      if (c == r) return h;
      if (c == -1) return -1;
    }
    return -1;
  }
};

// Root of v during phase A.  Only roots are ever published, and no join runs
// in phase A, so a vertex in the block's table is a root of this round: the
// walk stops there without loading that root's word, which every find in a
// large component would otherwise end on.
__device__ __forceinline__ int mst_find_a(int v, int* parent, const RootTable& tab) {
  if (tab.has(v)) return v;
  int cur = ld(&parent[v]);
  if (cur == v || tab.has(cur)) return cur;
  int prev = v, next;
  while (cur != (next = ld(&parent[cur]))) {
    st(&parent[prev], next);
    prev = cur;
    cur = next;
    if (tab.has(cur)) break;
  }
  return cur;
}

// ... and the calling thread remembers the last root it published to with
// the smallest key it has seen there (a key word only decreases), so a giant
// root met again in the next iterations costs no load.  Roots that get a
// slot in the block's table are lowered there instead.
__device__ __forceinline__ void mst_publish(u64* mcur, int root, bool keep, int w, int j, int lane, MstMemo& memo,
                                            RootTable& tab) {
  const unsigned g = __match_any_sync(kFull, keep ? root : -1);
  const unsigned wmin = __reduce_min_sync(g, keep ? (unsigned)w : 0xffffffffu);
  const unsigned jmin = __reduce_min_sync(g, (keep && (unsigned)w == wmin) ? (unsigned)j : 0xffffffffu);
  if (keep && lane == __ffs(g) - 1) {
    const u64 key = ((u64)wmin << 32) | jmin;
    const int h = tab.claim(root);
    if (h >= 0) {
      bref<u64>(tab.key[h]).fetch_min(key, cuda::memory_order_relaxed);
      return;
    }
    if (memo.key == root && memo.val <= key) return;
    const u64 cur = ld(&mcur[root]);
    if (cur > key) fetch_min(&mcur[root], key);
    memo.key = root;
    memo.val = cur < key ? cur : key;
  }
}

// All Boruvka rounds of one pass.  wlA holds the pass's initial worklist
// (size wlcount[pass][0]); rounds alternate wlA/wlB.
__global__ void __launch_bounds__(kTPB) mst_boruvka(int n, int pass, int4* __restrict__ wlA, int4* __restrict__ wlB,
                                                    int cap, int* __restrict__ parent, u64* __restrict__ minv,
                                                    unsigned char* __restrict__ in_mst, MSTCtl* __restrict__ ctl,
                                                    Status* __restrict__ status) {
  const int tid = blockIdx.x * kTPB + threadIdx.x;
  const int nthreads = gridDim.x * kTPB;
  const int lane = threadIdx.x & 31;
  int* cnt = ctl->wlcount[pass];
  __shared__ int4 stage_buf[kTPB / 32][kStage];
  Stage stg{stage_buf[threadIdx.x >> 5]};
  __shared__ int s_root[kRootSlots];
  __shared__ u64 s_key[kRootSlots];
  RootTable tab{s_root, s_key};
  bool overflow = false;
  u64 local = 0;
  int r = 0;
  if (tid == 0) ctl->stamp[pass][0] = mst_now();
  for (; r < kMaxRounds; r++) {
    // Round 0's list comes from a scan: its entries already join two
    // distinct roots, so round 0 only publishes their keys and joins along
    // the same list (no re-rooting, no copy); round r >= 1 re-roots the list
    // round r - 1 left (wlA for r = 1) into the other buffer.
    int4* in = (r == 0 || (r & 1)) ? wlA : wlB;
    int4* out = r == 0 ? wlA : ((r & 1) ? wlB : wlA);
    u64* mcur = minv + (size_t)(r & 1) * n;
    u64* mprev = minv + (size_t)((r + 1) & 1) * n;
    // a scan that overflowed (reported as BAD_GRAPH) counted more entries
    // than the list holds
    const int sz = min(ld(&cnt[r]), cap);
    // phase A: re-root, drop intra-component edges, publish keys.  The trip
    // count is uniform across the grid so every warp step is converged for
    // the warp-aggregated append.
    // clear the keys round r-1 published: a streaming pass over all
    // vertices (a reset per edge would store to the giant component's word
    // from every warp)
    if (r > 0)
      for (int v = tid; v < n; v += nthreads) st(&mprev[v], ~0ull);
    tab.reset();  // the last phase B's reads ended at its grid barrier
    __syncthreads();
    const int iters = (sz + nthreads - 1) / nthreads;
    // per-thread memos: roots cannot change during phase A (joins happen in
    // phase B), so a remembered find is exact
    MstMemo fx, fy, px, py;
    // each step's entry is loaded one step ahead (the stream's latency then
    // overlaps the previous step's finds and publishes)
    int4 nx = tid < sz ? __ldcs(&in[tid]) : make_int4(-1, -1, 0, 0);
    for (int it = 0; it < iters; it++) {
      const int i = tid + it * nthreads;
      const bool valid = i < sz;
      const int4 e = nx;
      const long long i1 = (long long)i + nthreads;
      nx = i1 < sz ? __ldcs(&in[i1]) : make_int4(-1, -1, 0, 0);
      // each lane finds its own entry's roots (a per-lane memo, and the
      // block's table ends a find at a known root without a load): grouping
      // equal endpoints per warp first measured slower
      int ra = e.x, rb = e.y;  // round 0: the scan's entries hold roots
      if (r > 0 && valid) {
        if (fx.key != e.x) {
          fx.key = e.x;
          fx.val = (u64)mst_find_a(e.x, parent, tab);
        }
        ra = (int)fx.val;
        if (fy.key != e.y) {
          fy.key = e.y;
          fy.val = (u64)mst_find_a(e.y, parent, tab);
        }
        rb = (int)fy.val;
      }
      const bool keep = valid && ra != rb;
      if (r > 0) stg.push(keep, make_int4(ra, rb, e.z, e.w), out, &cnt[r + 1], cap, overflow);
      mst_publish(mcur, ra, keep, e.z, e.w, lane, px, tab);
      mst_publish(mcur, rb, keep, e.z, e.w, lane, py, tab);
    }
    if (r > 0)
      stg.flush(out, &cnt[r + 1], cap, overflow);
    else if (tid == 0)
      st(&cnt[1], sz);  // round 1 reads round 0's list, whole
    // publish the block's table: one load (and at most one atomic) per root
    __syncthreads();
    for (int i = threadIdx.x; i < kRootSlots; i += kTPB) {
      const int rt = s_root[i];  // race-free: claims ended at the barrier above
      if (rt >= 0 && ld(&mcur[rt]) > s_key[i]) fetch_min(&mcur[rt], s_key[i]);
    }
    if (!grid_sync(&ctl->bar, status)) return;
    if (tid == 0) ctl->stamp[pass][2 * r + 1] = mst_now();
    const int nsz = ld(&cnt[r + 1]);
    if (nsz == 0) break;
    // phase B: join along every edge that is the minimum of one of its roots
    // (each root's key is loaded once per warp, and key words do not change
    // during phase B, so a per-thread memo of the last one is exact; the
    // roots in the block's table once per block)
    for (int i = threadIdx.x; i < kRootSlots; i += kTPB) {
      const int rt = s_root[i];  // race-free: no claim runs after phase A
      if (rt >= 0) s_key[i] = ld(&mcur[rt]);  // race-free: slot i is this thread's until the barrier below
    }
    __syncthreads();
    MstMemo kxm, kym;
    int4 nxb = tid < nsz ? __ldcs(&out[tid]) : make_int4(-1, -1, 0, 0);  // one step ahead, as in phase A
    for (int i0 = tid - lane; i0 < nsz; i0 += nthreads) {
      const int i = i0 + lane;
      const bool valid = i < nsz;
      const int4 e = nxb;
      const long long i1 = (long long)i + nthreads;
      nxb = i1 < nsz ? __ldcs(&out[i1]) : make_int4(-1, -1, 0, 0);
      const unsigned gx = __match_any_sync(kFull, e.x), gy = __match_any_sync(kFull, e.y);
      const int lx = __ffs(gx) - 1, ly = __ffs(gy) - 1;
      u64 kx = 0, ky = 0;
      if (valid && lane == lx) {
        const int h = tab.find(e.x);
        if (h >= 0) {
          kx = s_key[h];  // race-free: read-only until the next round's reset
        } else {
          if (kxm.key != e.x) {
            kxm.key = e.x;
            kxm.val = ld(&mcur[e.x]);
          }
          kx = kxm.val;
        }
      }
      if (valid && lane == ly) {
        const int h = tab.find(e.y);
        if (h >= 0) {
          ky = s_key[h];  // race-free: as above
        } else {
          if (kym.key != e.y) {
            kym.key = e.y;
            kym.val = ld(&mcur[e.y]);
          }
          ky = kym.val;
        }
      }
      kx = __shfl_sync(kFull, kx, lx);
      ky = __shfl_sync(kFull, ky, ly);
      const u64 key = ((u64)(unsigned)e.z << 32) | (unsigned)e.w;
      if (valid && (key == kx || key == ky)) {
        mst_join(e.x, e.y, parent);
        in_mst[e.w] = 1;  // race-free: each entry j is joined at most once, and never read here
        local += (u64)(unsigned)e.z;
      }
    }
    if (!grid_sync(&ctl->bar, status)) return;
    if (tid == 0) ctl->stamp[pass][2 * r + 2] = mst_now();
  }
  if (r == kMaxRounds) raise(status, ECL_ERR_NO_CONVERGENCE, pass);
  // per-block sum of the joined weights
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(kFull, local, o);
  if ((threadIdx.x & 31) == 0 && local) fetch_add(&ctl->total, local);
  if (threadIdx.x == 0) fetch_max(&status->rounds, r + 1);
}

struct MSTBufs {
  MSTCtl* ctl;
  int* parent;
  u64* minv;
  int2* chunks;
  int chunk_cap;
  int4* wlA;
  int4* wlB;
  int cap;
};

void mst_layout(Carve& c, int n, int m, bool symmetric, MSTBufs* b) {
  b->ctl = c.take<MSTCtl>(1);
  b->parent = c.take<int>((size_t)n);
  b->minv = c.take<u64>((size_t)2 * n);
  b->chunks = c.take<int2>(row_chunk_capacity(m, kMinChunk));
  b->chunk_cap = (int)row_chunk_capacity(m, kMinChunk);
  // v<n entries: at most m/2 in a symmetric, self-loop-free graph, else m.
  b->cap = symmetric ? m / 2 + 1 : (m > 0 ? m : 1);
  b->wlA = c.take<int4>((size_t)b->cap);
  b->wlB = c.take<int4>((size_t)b->cap);
}

}  // namespace

size_t mst_workspace_bytes(int n, int m) {
  Carve c;
  MSTBufs b;
  mst_layout(c, n, m, false, &b);
  return c.bytes();
}

ecl_status mst_enqueue(const GraphDev& g, unsigned char* in_mst, char* ws, Status* status, const DeviceInfo& dev,
                       cudaStream_t stream, unsigned long long** total_dev, Marker mark) {
  const bool sym = (g.flags & ECL_GRAPH_SYMMETRIC) != 0;
  Carve c{ws};
  MSTBufs b;
  mst_layout(c, g.n, g.m, sym, &b);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mst_boruvka, kTPB, 0) != cudaSuccess || occ < 1)
    return ECL_ERR_CUDA;
  const int coop_grid = dev.sms * occ;
  const int grid = dev.grid_blocks(kTPB, g.n, g.m);
  const Bins bins = bins_of(dev, kMstBins);
  // 16-byte row loads need 16-byte-aligned arrays (entries j = 0 mod 4 then are)
  const bool vec =
      ((reinterpret_cast<uintptr_t>(g.nlist) | reinterpret_cast<uintptr_t>(g.eweight)) & 15) == 0 && dev.row_vec;
  if (total_dev) *total_dev = &b.ctl->total;
  ECL_CUDA_TRY(cudaMemsetAsync(b.ctl, 0, sizeof(MSTCtl), stream));
  if (g.m > 0) ECL_CUDA_TRY(cudaMemsetAsync(in_mst, 0, (size_t)g.m, stream));
  ECL_LAUNCH(mst_init, grid, kTPB, 0, stream, g.n, b.parent, b.minv);
  if (g.m > 0) {
    const float light = dev.mst_light_factor > 0.f ? dev.mst_light_factor : 0.75f;
    ECL_LAUNCH(mst_threshold, 1, kSamples, 0, stream, g.n, g.m, g.eweight, b.ctl, light);
    mark();
    for (int pass = 0; pass < 2; pass++) {
      if (pass == 0) {
        ECL_LAUNCH(mst_scan<true>, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, g.eweight, b.parent, b.wlA,
                   b.cap, b.ctl, b.chunks, bins, vec, status);
        ECL_LAUNCH(mst_chunks<true>, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, g.eweight, b.parent, b.wlA, b.cap,
                   b.ctl, b.chunks, b.chunk_cap, bins.chunk, vec, status);
      } else {
        ECL_LAUNCH(mst_flatten, grid, kTPB, 0, stream, g.n, b.parent);
        ECL_LAUNCH(mst_scan<false>, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, g.eweight, b.parent, b.wlA,
                   b.cap, b.ctl, b.chunks, bins, vec, status);
        ECL_LAUNCH(mst_chunks<false>, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, g.eweight, b.parent, b.wlA, b.cap,
                   b.ctl, b.chunks, b.chunk_cap, bins.chunk, vec, status);
      }
      mark();
      ECL_CUDA_TRY(launch_cooperative(mst_boruvka, coop_grid, kTPB, stream, g.n, pass, b.wlA, b.wlB, b.cap, b.parent,
                                      b.minv, in_mst, b.ctl, status));
      mark();
      // The heavy pass (pass 1) runs unconditionally: with no filter it finds
      // no entry above the INT_MAX threshold and ends after one round.
    }
  }
  return ECL_OK;
}

}  // namespace ecl

extern "C" ecl_status ecl_mst(const ecl_graph_view* g, uint8_t* in_mst_out, uint64_t* total_weight, ecl_opts* opts) {
  using namespace ecl;
  ecl_opts local{};
  if (!opts) opts = &local;
  if (!in_mst_out && g && g->edges > 0) return ECL_ERR_INVALID_ARG;
  Solve s(g, opts);
  GraphNeeds needs;
  needs.weights = true;
  const bool sym = g && (g->flags & ECL_GRAPH_SYMMETRIC);
  size_t wsb = 0;
  if (g && g->nodes >= 1 && g->edges >= 0) {
    Carve c;
    MSTBufs b;
    mst_layout(c, g->nodes, g->edges, sym, &b);
    wsb = c.bytes();
  }
  ecl_status st = s.begin(needs, wsb);
  if (st != ECL_OK) return s.finish(st);
  unsigned char* in_mst = s.output(in_mst_out, (size_t)(s.m > 0 ? s.m : 1));
  if (!in_mst) return s.finish(ECL_ERR_OOM);
  GraphDev gd;
  gd.n = s.n;
  gd.m = s.m;
  gd.nindex = s.nindex;
  gd.nlist = s.nlist;
  gd.eweight = s.eweight;
  gd.flags = g->flags;
  u64* total_dev = nullptr;
  u64 hostTotal = 0;
  s.start_timer();
  st = mst_enqueue(gd, in_mst, s.ws, s.status, s.dev, s.stream, &total_dev, Marker{&s});
  s.stop_timer();
  if (st == ECL_OK && total_weight && total_dev) {
    if (cudaMemcpyAsync(&hostTotal, total_dev, sizeof(u64), cudaMemcpyDeviceToHost, s.stream) != cudaSuccess)
      st = ECL_ERR_CUDA;
  }
  st = s.finish(st);
  if (total_weight) *total_weight = (st == ECL_OK) ? hostTotal : 0;
  return st;
}

extern "C" ecl_status ecl_compute_mst(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist,
                                      const int32_t* eweight, uint8_t* in_mst) {
  ecl_graph_view g{nodes, edges, nidx, nlist, eweight, ECL_HOST, 0};
  ecl_opts o{};
  return ecl_mst(&g, in_mst, nullptr, &o);
}
