// Graph colouring (ECL-GC contract).
//
// Result contract (src/racefree/egr-input/GC/ECL-GC-atomic.cu): priorities
// are (degree, hash, id) (:102); init/runLarge/runSmall (:78-303) only fix a
// colour once it is the smallest colour not taken by a decided higher-priority
// list entry and no undecided one can still take it, i.e. the result is the
// first-fit greedy colouring in descending priority order.  Self-loops are
// never higher priority (:102 compares v with itself) and are ignored.
//
// B200 design: greedy colouring pulled in priority order.
//  * gc_keys writes every vertex's priority key (the inverted (degree, hash)
//    word) and colours the isolated vertices 0; gc_init / gc_init_chunks
//    (degree-binned: lane / warp / 256-entry chunk records) compare each
//    list entry with one 8-byte key load and compact every row's
//    higher-priority entries to the front of the row's slot in nl2[];
//    hc[v] = their number.
//  * radix_sort_pairs then ranks the vertices that have entries by priority
//    (an LSD sort of their keys), which is a topological order of the
//    colouring dependencies.
//  * gc_pull is ONE cooperative persistent launch.  Ranks are dealt to the
//    warps round-robin -- one long row (> 32 entries; they form a prefix of
//    the order, priority being degree-first) or 32 short rows at a time --
//    and every warp takes its own in increasing order; each vertex waits
//    (bounded polling of exactly its own higher-priority neighbours' colour
//    words) until they are coloured and stores the smallest colour they do
//    not use.  The warp holding the lowest unfinished rank is working on it,
//    and all its dependencies have lower ranks, so the launch always makes
//    progress.  There is no push, no counter and no queue: the total work is
//    one read of every higher-priority entry, and the longest priority chain
//    (about 2700 vertices at R-MAT-22, most of it in the hub core) costs one
//    poll-and-store hop per vertex on it.
//  * A long row is scanned by a whole warp with a 2048-colour bitmap in
//    shared memory.  The first pass never blocks: colours already published
//    go into the bitmap and the undecided entries into a per-warp pending
//    list; lanes then wait on listed entries (one address per lane) and
//    re-check the rest of the list without blocking -- so a hop along the
//    chain costs one poll and a short re-check, not a rescan of the row
//    (short rows: the same with a bit mask per lane).
#include <algorithm>
#include <vector>

#include "csr_bins.cuh"
#include "radix_sort.cuh"
#include "solvers.cuh"

namespace ecl {
namespace {

using namespace dev;

constexpr int kTPB = 256;

constexpr int kWarpRow = 32;  // rows longer than this are coloured by a whole warp

struct GCCtl {
  int nchunks;
  int nbig;        // rows longer than kWarpRow: a prefix of the priority order
  int nkeys;       // vertices with at least one entry: the ones sorted and pulled
  int pad2[29];
};

// Priority hash of vertex x: the reference hashes the vertex id; in a union
// of graphs (vhash != nullptr) it is the hash of x's LOCAL id, precomputed.
__device__ __forceinline__ unsigned gc_h(const unsigned* vhash, int x) {
  return vhash ? __ldg(&vhash[x]) : ecl_hash((unsigned)x);
}

// Entries per lane whose loads are issued together in the init scans.
constexpr int kInitBatch = 4;

// Classes of kInitBatch list entries of v -- 0: ignore (self-loop or
// invalid), 1: higher priority than v, 2: lower.  A vertex's priority is its
// sort key (gc_keys: the inverted (degree, hash) word, so a SMALLER key is a
// higher priority) with ties to the larger id; kv is v's key.  The list
// entries are loaded first, then every neighbour's key (one 8-byte load each
// instead of both row bounds and a rehash), all before any is compared.
__device__ __forceinline__ void gc_class_batch(const int (&u)[kInitBatch], const bool (&valid)[kInitBatch], int v,
                                               unsigned long long kv, int n, const unsigned long long* keys,
                                               Status* status, int (&cls)[kInitBatch]) {
  unsigned long long ku[kInitBatch];
#pragma unroll
  for (int k = 0; k < kInitBatch; k++) {
    const bool ok = valid[k] && (unsigned)u[k] < (unsigned)n && u[k] != v;
    ku[k] = ok ? __ldg(&keys[n - 1 - u[k]]) : 0ull;
  }
#pragma unroll
  for (int k = 0; k < kInitBatch; k++) {
    cls[k] = 0;
    if (!valid[k]) continue;
    if ((unsigned)u[k] >= (unsigned)n) {
      raise(status, ECL_ERR_BAD_GRAPH, u[k]);
    } else if (u[k] != v) {
      cls[k] = (ku[k] < kv || (ku[k] == kv && u[k] > v)) ? 1 : 2;
    }
  }
}

// vhash[v] = hash of v's local id in a union of graphs.
__global__ void __launch_bounds__(kTPB) gc_union_hash(int n, const int* __restrict__ vbase, int ngraphs,
                                                      unsigned* __restrict__ vhash) {
  for (int v = blockIdx.x * kTPB + threadIdx.x; v < n; v += gridDim.x * kTPB) {
    int lo = 0, hi = ngraphs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(&vbase[mid]) <= v) lo = mid;
      else hi = mid - 1;
    }
    vhash[v] = ecl_hash((unsigned)(v - __ldg(&vbase[lo])));
  }
}

__global__ void __launch_bounds__(kTPB) gc_init(int n, int m, const int* __restrict__ nindex,
                                                const int* __restrict__ nlist, int* __restrict__ nl2,
                                                int* __restrict__ hc, RowChunks rc, Bins bins, bool vec,
                                                const unsigned long long* __restrict__ keys,
                                                Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    const int v = base + lane;
    int beg = 0, end = 0;
    if (v < n) csr_row(nindex, v, m, beg, end, status);
    const int dv = end - beg;
    const unsigned long long kv = (v < n) ? __ldg(&keys[n - 1 - v]) : 0ull;
    int h = 0;
    push_chunks_warp(rc, bins.chunk, dv > bins.chunk, v, beg, end, status);
    if (v < n && dv <= bins.lane) {
      for (int i0 = beg; i0 < end; i0 += kInitBatch) {
        int u[kInitBatch], cls[kInitBatch];
        bool valid[kInitBatch];
#pragma unroll
        for (int k = 0; k < kInitBatch; k++) {
          valid[k] = i0 + k < end;
          u[k] = valid[k] ? __ldg(&nlist[i0 + k]) : 0;
        }
        gc_class_batch(u, valid, v, kv, n, keys, status, cls);
#pragma unroll
        for (int k = 0; k < kInitBatch; k++)
          if (cls[k] == 1) nl2[beg + h++] = u[k];
      }
    }
    unsigned todo = __ballot_sync(kFull, dv > bins.lane && dv <= bins.chunk);
    while (todo) {
      const int who = __ffs(todo) - 1;
      todo &= todo - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      const unsigned long long wkv = __shfl_sync(kFull, kv, who);
      int wh = 0;
      warp_row(wbeg, wend, m, vec, nlist, [&](const int(&)[4], const int (&u)[4], const bool (&valid)[4]) {
        int cls[kInitBatch];
        gc_class_batch(u, valid, wv, wkv, n, keys, status, cls);
#pragma unroll
        for (int k = 0; k < kInitBatch; k++) {
          const unsigned bh = __ballot_sync(kFull, cls[k] == 1);
          if (cls[k] == 1) nl2[wbeg + wh + __popc(bh & ((1u << lane) - 1))] = u[k];
          wh += __popc(bh);
        }
      });
      if (lane == who) h = wh;
    }
    // race-free: v's own count, read only by later launches; chunked rows start at 0 (gc_init_chunks adds)
    if (v < n) hc[v] = dv > bins.chunk ? 0 : h;
  }
}

__global__ void __launch_bounds__(kTPB) gc_init_chunks(int n, int m, const int* __restrict__ nindex,
                                                       const int* __restrict__ nlist, int* __restrict__ nl2,
                                                       int* __restrict__ hc, RowChunks rc, int chunk, bool vec,
                                                       const unsigned long long* __restrict__ keys,
                                                       Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int total = chunk_total(rc);
  for (int c = warp; c < total; c += nwarps) {
    const int2 r = rc.rec[c];
    const int v = r.x;
    const int beg = __ldg(&nindex[v]), end = __ldg(&nindex[v + 1]);
    const int stop = min(r.y + chunk, end);
    const unsigned long long kv = __ldg(&keys[n - 1 - v]);
    warp_row(r.y, stop, m, vec, nlist, [&](const int(&)[4], const int (&u)[4], const bool (&valid)[4]) {
      int cls[kInitBatch];
      gc_class_batch(u, valid, v, kv, n, keys, status, cls);
      unsigned bh[kInitBatch];
      int nh = 0;
#pragma unroll
      for (int k = 0; k < kInitBatch; k++) {
        bh[k] = __ballot_sync(kFull, cls[k] == 1);
        nh += __popc(bh[k]);
      }
      int hbase = 0;
      if (lane == 0 && nh) hbase = fetch_add(&hc[v], nh);
      hbase = __shfl_sync(kFull, hbase, 0);
#pragma unroll
      for (int k = 0; k < kInitBatch; k++) {
        if (cls[k] == 1) nl2[beg + hbase + __popc(bh[k] & ((1u << lane) - 1))] = u[k];
        hbase += __popc(bh[k]);
      }
    });
  }
}

// Priority keys: keys[n - 1 - v] = ~((degree << 32) | hash) for every v, the
// array gc_init compares neighbours by; ascending order of the keys is
// descending (degree, hash), the priority (within one graph the hash is a
// bijection of the id, so no two vertices tie).  The vertices with at least
// one entry are also appended to (skeys, svals), the sort's input, counted in
// ctl->nkeys.  An isolated vertex has no neighbour to wait for or to block:
// its colour is 0, written here, and it is neither sorted nor pulled
// (R-MAT-22 has 1.8 M of them among its 4.2 M vertices).
__global__ void __launch_bounds__(kTPB) gc_keys(int n, const int* __restrict__ nindex,
                                                unsigned long long* __restrict__ keys,
                                                unsigned long long* __restrict__ skeys, int* __restrict__ svals,
                                                const unsigned* __restrict__ vhash, int* __restrict__ color,
                                                GCCtl* __restrict__ ctl) {
  // rows longer than kWarpRow are counted per block and added once per block;
  // the appends reserve their room with one atomic per block and step
  __shared__ int s_big;
  __shared__ int s_woff[kTPB / 32];
  __shared__ int s_base;
  if (threadIdx.x == 0) s_big = 0;
  __syncthreads();
  int nb = 0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int bbase = blockIdx.x * kTPB; bbase < n; bbase += gridDim.x * kTPB) {  // block-uniform trip count
    const int i = bbase + threadIdx.x;
    bool big = false, linked = false;
    unsigned long long key = 0;
    int v = 0;
    if (i < n) {
      v = n - 1 - i;
      const unsigned deg = (unsigned)(__ldg(&nindex[v + 1]) - __ldg(&nindex[v]));
      key = ~(((unsigned long long)deg << 32) | gc_h(vhash, v));
      keys[i] = key;
      big = deg > (unsigned)kWarpRow;
      linked = deg > 0;
      if (!linked) color[v] = 0;  // race-free: the output, thread-owned; nothing reads it in this launch
    }
    nb += __popc(__ballot_sync(kFull, big));
    const unsigned bal = __ballot_sync(kFull, linked);
    if (lane == 0) s_woff[wid] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
      int run = 0;
      for (int w = 0; w < kTPB / 32; w++) {
        const int c = s_woff[w];
        s_woff[w] = run;
        run += c;
      }
      s_base = run ? fetch_add(&ctl->nkeys, run) : 0;
    }
    __syncthreads();
    if (linked) {
      const int at = s_base + s_woff[wid] + __popc(bal & ((1u << lane) - 1));
      skeys[at] = key;
      svals[at] = v;
    }
    __syncthreads();  // s_woff and s_base are rewritten next step
  }
  if ((threadIdx.x & 31) == 0 && nb) atomicAdd(&s_big, nb);
  __syncthreads();
  if (threadIdx.x == 0 && s_big) fetch_add(&ctl->nbig, s_big);
}

__device__ __forceinline__ unsigned long long gc_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr unsigned long long kStallNs = 2000000000ull;  // 2 s without progress -> give up
constexpr int kMexWords = 64;                           // warp bitmap: 2048 colours per window
constexpr int kPend = 1024;                             // per-warp list of undecided entries
constexpr int kBatch = 16;                              // entries per lane whose loads are in flight together

// Colour of u once it is published (bounded wait).  Returns -1 on a stall.
__device__ __forceinline__ int gc_wait_colour(const int* color, int u, Status* status, unsigned nap_cap = 512u) {
  int c = ld(&color[u]);
  if (c >= 0) return c;
  unsigned nap = 32, spins = 0;
  const unsigned long long t0 = gc_now();
  while ((c = ld(&color[u])) < 0) {
    // the stall checks every 64th poll: status->code is one word, and every
    // polling lane of the grid reading it on every poll makes its L2 slice a
    // hot spot that slows the colour polls themselves
    if ((++spins & 63u) == 0 && (spins > (1u << 24) || gc_now() - t0 > kStallNs || ld(&status->code) != 0)) {
      raise(status, ECL_ERR_NO_CONVERGENCE, u);
      return -1;
    }
    __nanosleep(nap);
    nap = min(nap * 2, nap_cap);
  }
  return c;
}

__device__ __forceinline__ void gc_mark(unsigned* bits, int c, int off) {
  const int d = c - off;
  if (d >= 0 && d < 32 * kMexWords) atomicOr(&bits[d >> 5], 1u << (d & 31));
}

// Colour of a long row: the smallest colour no entry of nl2[wb, we) uses.
// Each window of 2048 colours starts with one non-blocking pass over the row:
// colours already published go into the bitmap, still-undecided entries into
// the per-warp list `pend`.  Then every lane waits (bounded, one address per
// lane as before) for one listed entry, and the rest of the list is
// re-checked without blocking and compacted; repeat until it is empty.  Once
// the last dependency is coloured the row is one poll and one short re-check
// from its colour -- a lane no longer walks the rest of its share of the row
// after each wait.  The pass stops while the list still has room for a whole
// step of 32 entries; the listed ones are resolved and the pass resumes where
// it stopped, so every entry is read once by the pass.  Returns -1 on a
// stall.  All lanes call.
__device__ int gc_long_row(int wb, int we, const int* nl2, const int* color, unsigned* bits, int* pend, int pend_cap,
                           unsigned nap_cap, Status* status) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1;
  for (int off = 0;; off += 32 * kMexWords) {
    bits[lane] = 0;
    bits[lane + 32] = 0;
    __syncwarp();
    int cursor = wb;
    while (cursor < we) {
      int np = 0;
      int i0 = cursor;
      // kBatch entries per lane per step: all index loads, then all colour
      // loads, are issued before any result is used (one round trip per
      // 32 * kBatch entries instead of two per 32)
      for (; i0 < we && np + 32 * kBatch <= pend_cap; i0 += 32 * kBatch) {
        int u[kBatch], c[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
          const int i = i0 + 32 * k + lane;
          u[k] = i < we ? __ldg(&nl2[i]) : -1;
        }
#pragma unroll
        for (int k = 0; k < kBatch; k++) c[k] = u[k] >= 0 ? ld(&color[u[k]]) : 0;
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
          const bool undecided = u[k] >= 0 && c[k] < 0;
          if (u[k] >= 0 && c[k] >= 0) gc_mark(bits, c[k], off);
          const unsigned ub = __ballot_sync(kFull, undecided);
          if (undecided) pend[np + __popc(ub & lt)] = u[k];
          np += __popc(ub);
        }
      }
      cursor = i0;  // the list is full or the row is done: resolve, then resume here
      int cnt = np;
      while (cnt > 0) {
        __syncwarp();
        bool stalled = false;
        if (lane < cnt) {
          const int c = gc_wait_colour(color, pend[lane], status, nap_cap);
          if (c < 0)
            stalled = true;
          else
            gc_mark(bits, c, off);
        }
        if (__any_sync(kFull, stalled)) return -1;
        int kept = 0;
        for (int j0 = 32; j0 < cnt; j0 += 32 * kBatch) {
          int u[kBatch], c[kBatch];
#pragma unroll
          for (int k = 0; k < kBatch; k++) {
            const int j = j0 + 32 * k + lane;
            u[k] = j < cnt ? pend[j] : -1;
          }
#pragma unroll
          for (int k = 0; k < kBatch; k++) c[k] = u[k] >= 0 ? ld(&color[u[k]]) : 0;
          __syncwarp();  // every lane has read its slots before any is overwritten
#pragma unroll
          for (int k = 0; k < kBatch; k++) {
            const bool still = u[k] >= 0 && c[k] < 0;
            if (u[k] >= 0 && c[k] >= 0) gc_mark(bits, c[k], off);
            const unsigned sb = __ballot_sync(kFull, still);
            if (still) pend[kept + __popc(sb & lt)] = u[k];  // index < j0: already read
            kept += __popc(sb);
          }
        }
        cnt = kept;
      }
    }
    __syncwarp();
    const unsigned w0 = bits[lane], w1 = bits[lane + 32];
    const unsigned f0 = __ballot_sync(kFull, w0 != ~0u), f1 = __ballot_sync(kFull, w1 != ~0u);
    int c = -1;
    if (f0) {
      const int wi = __ffs(f0) - 1;
      c = off + wi * 32 + __ffs(~__shfl_sync(kFull, w0, wi)) - 1;
    } else if (f1) {
      const int wi = __ffs(f1) - 1;
      c = off + (wi + 32) * 32 + __ffs(~__shfl_sync(kFull, w1, wi)) - 1;
    }
    __syncwarp();
    if (c >= 0) return c;
  }
}

// Colour of a short row (h <= 32 entries at nl2[beg]): one lane, the same
// scheme with a bit mask of the undecided entries -- wait for the first one,
// re-check the others without blocking.  -1 on a stall.
__device__ int gc_short_row(int beg, int h, const int* nl2, const int* color, Status* status) {
  // colour <= h <= 32: a neighbour's colour of 64 or more (a hub's) cannot
  // be the smallest free one and is left out of the mask
  unsigned long long used = 0;
  unsigned pendm = 0;
  for (int k0 = 0; k0 < h; k0 += kBatch) {
    int u[kBatch], c[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; k++) u[k] = k0 + k < h ? __ldg(&nl2[beg + k0 + k]) : -1;
#pragma unroll
    for (int k = 0; k < kBatch; k++) c[k] = u[k] >= 0 ? ld(&color[u[k]]) : 0;
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      if (u[k] < 0) continue;
      if (c[k] >= 0)
        used |= c[k] < 64 ? 1ull << c[k] : 0ull;
      else
        pendm |= 1u << (k0 + k);
    }
  }
  while (pendm) {
    const int k0 = __ffs(pendm) - 1;
    const int c0 = gc_wait_colour(color, __ldg(&nl2[beg + k0]), status);
    if (c0 < 0) return -1;
    used |= c0 < 64 ? 1ull << c0 : 0ull;
    pendm &= pendm - 1;
    for (unsigned mm = pendm; mm; mm &= mm - 1) {
      const int k = __ffs(mm) - 1;
      const int c = ld(&color[__ldg(&nl2[beg + k])]);
      if (c >= 0) {
        used |= c < 64 ? 1ull << c : 0ull;
        pendm &= ~(1u << k);
      }
    }
  }
  return __ffsll((long long)~used) - 1;
}

// ---- the hub core: the first ranks of the order, coloured in shared memory ----
//
// On R-MAT the longest priority chain (about 2700 vertices at scale 22)
// runs almost entirely through the long rows at the front of the order:
// about 2200 of its hops lie in the first 16k ranks and 2470 in the first 32k.
// A hop through L2 costs a store, a poll and a wake-up (about 1.5 us as the
// pull achieves it); in shared memory it costs a few hundred cycles.  So the
// first `core` ranks (core = min(long rows, cap)) are coloured by a cluster
// of CTAs of 32 warps each (two by default) with the colours in shared
// memory, indexed by rank -- a copy in every CTA, each colour stored into all
// copies through distributed shared memory: every higher-priority entry of a
// core row is itself a core vertex (it has a smaller rank), so a core row
// never waits on global memory.  Two small launches first rewrite
// the core rows' entries in nl2 from vertex ids to ranks (rank[] is the
// inverse of the order over the core) and record each core rank's row
// (start, length, vertex).
//
// The cluster's SMs stream all core rows (16.6 M entries for the first 32k
// ranks of R-MAT-22), and a warp that fetched each row with its own loads paid a
// dependent L2 round trip per 128 entries.  Instead every warp stages its
// rows through two shared-memory buffers with bulk asynchronous copies
// (cp.async.bulk, completion counted on an mbarrier): while it colours one
// segment of a row, the next segment -- of this row or of its next row -- is
// already on its way, and the scan itself reads shared memory only.  Colours
// are 16-bit words (0xffff = not yet coloured; a core colour is at most the
// row's length, below 2^15).
constexpr int kCoreThreads = 1024;
constexpr int kCoreWarps = kCoreThreads / 32;
// Default CTAs of the core's cluster.  R-MAT-22, core + pull: 1 CTA with 4096
// ranks 3.15 ms; 2 CTAs with 8192 ranks 2.86 ms; 4 CTAs 2.92 ms (a hop
// between CTAs, through distributed shared memory, costs more than one inside
// a CTA, so more CTAs than two buy nothing).
constexpr int kCoreCtas = 2;
constexpr int kCoreBatch = 4;           // entries per lane whose loads are in flight together
constexpr int kCoreDefault = 8192;      // default core size (ranks): the measured best at R-MAT-22 with 2 CTAs
constexpr int kCoreMax = 36864;         // shared memory bound
constexpr int kSegSlack = 8;            // a buffer holds a segment plus its 16-byte alignment slack
constexpr int kCorePend = 1024;         // per-warp list of undecided entries (16-bit ranks)
constexpr int kSegBufMax = 384;  // longer segments measured slower (one copy's latency per row is exposed)
constexpr unsigned kUncoloured = 0xffffu;
constexpr size_t kCoreSmemLimit = 227 * 1024;

// Dynamic shared memory of the core CTA: colours (16-bit, per rank), then per
// warp two mbarriers, two staging buffers of `segbuf` entries, a 2048-colour
// bitmap and a list of up to kCorePend undecided entries (16-bit ranks).  The
// buffers take what the colours leave, up to kSegBufMax entries.
__host__ __device__ constexpr size_t gc_core_colour_bytes(int cap) { return ((size_t)cap * 2 + 15) & ~size_t(15); }
__host__ __device__ constexpr size_t gc_core_warp_bytes(int segbuf) {
  return 2 * sizeof(unsigned long long) + (size_t)segbuf * 2 * sizeof(int) + kMexWords * sizeof(unsigned) +
         kCorePend * sizeof(unsigned short);
}
__host__ __device__ constexpr int gc_core_segbuf(int cap) {
  const size_t fixed = gc_core_colour_bytes(cap) + kCoreWarps * gc_core_warp_bytes(0);
  const size_t per = (kCoreSmemLimit - fixed) / kCoreWarps / (2 * sizeof(int));
  return (int)((per < (size_t)kSegBufMax ? per : (size_t)kSegBufMax) & ~size_t(7));
}
__host__ __device__ constexpr size_t gc_core_smem(int cap) {
  return gc_core_colour_bytes(cap) + kCoreWarps * gc_core_warp_bytes(gc_core_segbuf(cap));
}
static_assert(gc_core_segbuf(kCoreMax) >= 256 && gc_core_smem(kCoreMax) <= kCoreSmemLimit,
              "core shared memory over the per-block limit");

// Core size of this solve: the long rows (a prefix of the order), at most cap.
__device__ __forceinline__ int gc_core_size(const GCCtl* ctl, int cap) { return min(ld(&ctl->nbig), cap); }

// rank[order[r]] = r over the core.
__global__ void __launch_bounds__(kTPB) gc_core_rank(const int* __restrict__ order, int* __restrict__ rank,
                                                     const GCCtl* __restrict__ ctl, int cap) {
  const int core = gc_core_size(ctl, cap);
  for (int r = blockIdx.x * kTPB + threadIdx.x; r < core; r += gridDim.x * kTPB) rank[__ldg(&order[r])] = r;
}

// Rewrites the higher-priority entries of every core row from vertex ids to
// ranks, one warp per row, and records the row: rowinfo[r] = (first entry,
// length, vertex).  Such an entry outranks its row, so its rank is below the
// row's and inside the core.
__global__ void __launch_bounds__(kTPB) gc_core_translate(const int* __restrict__ nindex, int* __restrict__ nl2,
                                                          const int* __restrict__ hc, const int* __restrict__ order,
                                                          const int* __restrict__ rank, int4* __restrict__ rowinfo,
                                                          const GCCtl* __restrict__ ctl, int cap) {
  const int lane = threadIdx.x & 31;
  const int core = gc_core_size(ctl, cap);
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int r = warp; r < core; r += nwarps) {
    const int v = __ldg(&order[r]);
    const int b = __ldg(&nindex[v]), h = __ldg(&hc[v]);
    for (int i = b + lane; i < b + h; i += 32) nl2[i] = __ldg(&rank[nl2[i]]);
    if (lane == 0) rowinfo[r] = make_int4(b, h, v, 0);
  }
}

// ---- shared-memory and bulk-copy primitives (CTA-local, inline PTX) ----

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// 16-bit colour words: relaxed CTA-scope atomic loads and stores.
// The core's colours live in every CTA of its cluster (one copy per CTA's
// shared memory): a colour is stored into each copy (distributed shared
// memory) and read from the local one, so both sides are cluster-scope
// relaxed accesses.
__device__ __forceinline__ unsigned col_ld(const unsigned short* p) {
  unsigned short v;
  asm volatile("ld.relaxed.cluster.shared::cta.u16 %0, [%1];" : "=h"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ void col_st(unsigned short* p, unsigned v) {
  asm volatile("st.relaxed.cluster.shared::cta.u16 [%0], %1;" ::"r"(smem_u32(p)), "h"((unsigned short)v) : "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_ctas() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// Every thread of every CTA of the cluster; memory before it is visible to
// the whole cluster after it.
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
// Stores colour v of the rank at p (a local shared address) into the copy of
// every CTA of the cluster.
__device__ __forceinline__ void col_publish(unsigned short* p, unsigned v, int ctas) {
  const unsigned local = smem_u32(p);
  for (int k = 0; k < ctas; k++) {
    unsigned remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(k));
    asm volatile("st.relaxed.cluster.shared::cluster.u16 [%0], %1;" ::"r"(remote), "h"((unsigned short)v) : "memory");
  }
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Starts a bulk copy of `bytes` (a multiple of 16, both ends 16-byte aligned)
// from global src into shared dst, completing on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier generic reads of dst come first
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase `parity` of bar (2 s); false when it ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = gc_now();
  for (unsigned spins = 1;; spins++) {
    if (mbar_test(bar, parity)) return true;
    if ((spins & 255u) == 0 && gc_now() - t0 > kStallNs) return false;
  }
}

// Colour of core rank q once it is published; -1 when the wait gives up (2 s
// without the colour, or another error raised).
__device__ __forceinline__ int gc_core_wait(const unsigned short* col_s, int q, Status* status) {
  unsigned c = col_ld(&col_s[q]);
  if (c != kUncoloured) return (int)c;
  const unsigned long long t0 = gc_now();
  for (unsigned spins = 1;; spins++) {
    c = col_ld(&col_s[q]);
    if (c != kUncoloured) return (int)c;
    if ((spins & 1023u) == 0 && (gc_now() - t0 > kStallNs || ld(&status->code) != 0)) {
      raise(status, ECL_ERR_NO_CONVERGENCE, q);
      return -1;
    }
    // no nap: the core is bound by its chain, and every nap length tried
    // (32 to 512 ns) measured slower than spinning on shared memory
  }
}

// Colour of core rank r whose entries (ranks) are nl2[wb, we), for colours
// from `off0` on, read straight from global memory: the fallback for a row
// whose first 2048 colours are all taken by its neighbours.  -1 on a stall.
__device__ int gc_core_row_global(int r, int wb, int we, int off0, const int* nl2, const unsigned short* col_s,
                                  unsigned* bits, unsigned short* pend, Status* status) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1;
  for (int off = off0;; off += 32 * kMexWords) {
    bits[lane] = 0;
    bits[lane + 32] = 0;
    __syncwarp();
    for (int i0 = wb; i0 < we; i0 += 32 * kCoreBatch) {
      int np = 0;
      int q[kCoreBatch];
#pragma unroll
      for (int k = 0; k < kCoreBatch; k++) {
        const int i = i0 + 32 * k + lane;
        q[k] = i < we ? __ldg(&nl2[i]) : -1;
        if (i < we && (unsigned)q[k] >= (unsigned)r) {
          raise(status, ECL_ERR_BAD_GRAPH, r);
          q[k] = -1;
        }
      }
#pragma unroll
      for (int k = 0; k < kCoreBatch; k++) {
        const unsigned c = q[k] >= 0 ? col_ld(&col_s[q[k]]) : 0u;
        const bool undecided = q[k] >= 0 && c == kUncoloured;
        if (q[k] >= 0 && !undecided) gc_mark(bits, (int)c, off);
        const unsigned ub = __ballot_sync(kFull, undecided);
        if (undecided) pend[np + __popc(ub & lt)] = (unsigned short)q[k];
        np += __popc(ub);
      }
      __syncwarp();
      bool stalled = false;
      for (int j = lane; j < np; j += 32) {
        const int c = gc_core_wait(col_s, pend[j], status);
        if (c < 0) {
          stalled = true;
          break;
        }
        gc_mark(bits, c, off);
      }
      if (__any_sync(kFull, stalled)) return -1;
    }
    __syncwarp();
    const unsigned w0 = bits[lane], w1 = bits[lane + 32];
    const unsigned f0 = __ballot_sync(kFull, w0 != ~0u), f1 = __ballot_sync(kFull, w1 != ~0u);
    int c = -1;
    if (f0) {
      const int wi = __ffs(f0) - 1;
      c = off + wi * 32 + __ffs(~__shfl_sync(kFull, w0, wi)) - 1;
    } else if (f1) {
      const int wi = __ffs(f1) - 1;
      c = off + (wi + 32) * 32 + __ffs(~__shfl_sync(kFull, w1, wi)) - 1;
    }
    __syncwarp();
    if (c >= 0) return c;
  }
}

// Per-warp staging of row segments: two buffers, each with its mbarrier and
// the parity of its next phase.  A segment is (first entry in nl2, length <=
// segbuf - 8); the copy starts at the 16-byte boundary at or below the first entry
// and ends at the one at or above its end (nl2 holds 4 spare entries past m,
// so the rounding never leaves the array).
struct CoreStage {
  int* buf[2];
  unsigned long long* bar[2];
  unsigned parity[2] = {0u, 0u};
  int first[2] = {-1, -1};  // segment in each buffer (-1: none in flight)
  int len[2] = {0, 0};

  __device__ __forceinline__ void issue(int b, const int* nl2, int f, int l) {
    first[b] = f;
    len[b] = l;
    if ((threadIdx.x & 31) == 0) {
      const int a = f & ~3, e = (f + l + 3) & ~3;
      bulk_load(buf[b], nl2 + a, 4u * (unsigned)(e - a), bar[b]);
    }
  }
  // Waits for buffer b's copy; the segment's entries then start at
  // buf[b] + offset(b).  False when the wait ran out.
  __device__ __forceinline__ bool wait(int b) {
    const bool ok = mbar_wait(bar[b], parity[b]);
    if (ok) parity[b] ^= 1u;  // a copy that did not land stays listed for drain()
    return ok;
  }
  __device__ __forceinline__ int offset(int b) const { return first[b] & 3; }
  // Bounded wait for every copy still in flight (before leaving on an error).
  __device__ __forceinline__ void drain() {
    for (int b = 0; b < 2; b++)
      if (first[b] >= 0) {
        if (mbar_wait(bar[b], parity[b])) parity[b] ^= 1u;
        first[b] = -1;
      }
  }
};

// One CTA colours the core: rank r goes to warp r mod 32, each warp takes its
// ranks in increasing order (the warp holding the lowest uncoloured rank can
// always finish it), and every colour is published to shared memory for the
// core and to color[] for gc_pull.  A warp's rows are a stream of segments;
// while one segment is scanned from shared memory the next is being copied.
__global__ void __launch_bounds__(kCoreThreads, 1) gc_core(const int* __restrict__ nl2, const int4* __restrict__ rowinfo,
                                                           int* __restrict__ color, const GCCtl* __restrict__ ctl,
                                                           int cap, Status* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char s_core[];
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1;
  const int core = gc_core_size(ctl, cap);
  // The core runs on a cluster of `ctas` CTAs (1 without a cluster launch):
  // rank r belongs to warp r mod (32 ctas) of the cluster, so each CTA takes
  // every ctas-th block of 32 consecutive ranks (dealing longer runs of
  // consecutive ranks to one CTA measured slower; single ranks, no faster).
  const int ctas = (int)cluster_ctas();
  const int warp = (int)cluster_rank() * kCoreWarps + (threadIdx.x >> 5);
  const int cwarps = ctas * kCoreWarps;
  unsigned short* col_s = reinterpret_cast<unsigned short*>(s_core);
  const int segbuf = gc_core_segbuf(cap);
  const int kSeg = segbuf - kSegSlack;  // row entries staged at a time
  unsigned char* wbase = s_core + gc_core_colour_bytes(cap) + (size_t)(threadIdx.x >> 5) * gc_core_warp_bytes(segbuf);
  CoreStage stg;
  stg.bar[0] = reinterpret_cast<unsigned long long*>(wbase);
  stg.bar[1] = stg.bar[0] + 1;
  stg.buf[0] = reinterpret_cast<int*>(wbase + 2 * sizeof(unsigned long long));
  stg.buf[1] = stg.buf[0] + segbuf;
  unsigned* bits = reinterpret_cast<unsigned*>(stg.buf[1] + segbuf);
  unsigned short* pend = reinterpret_cast<unsigned short*>(bits + kMexWords);
  for (int r = threadIdx.x; r < core; r += kCoreThreads) col_st(&col_s[r], kUncoloured);
  if (lane == 0) {
    mbar_init(stg.bar[0]);
    mbar_init(stg.bar[1]);
    mbar_fence_init();
  }
  __syncthreads();
  if (ctas > 1) cluster_sync();  // every copy is initialised before any colour is stored into it

  // Row j of this warp is rank warp + cwarps j; lane L holds the row record
  // of row jb + L (records are fetched 32 rows at a time).
  int jb = -32;
  int4 rec = make_int4(0, 0, -1, 0);
  auto row_of = [&](int j) -> int4 {  // all lanes call
    if ((j & ~31) != jb) {
      jb = j & ~31;
      const int r = warp + cwarps * (jb + lane);
      rec = r < core ? __ldg(&rowinfo[r]) : make_int4(0, 0, -1, 0);
    }
    const int src = j & 31;
    return make_int4(__shfl_sync(kFull, rec.x, src), __shfl_sync(kFull, rec.y, src), __shfl_sync(kFull, rec.z, src),
                     0);
  };
  const int nrows = core > warp ? (core - warp + cwarps - 1) / cwarps : 0;
  int b = 0;  // buffer holding (or about to hold) the segment to scan next
  for (int j = 0; j < nrows; j++) {
    const int r = warp + cwarps * j;
    const int4 row = row_of(j);
    const int wb = row.x, h = row.y, v = row.z;
    bits[lane] = 0;
    bits[lane + 32] = 0;
    __syncwarp();
    int np = 0;
    bool stalled = false;
    for (int off = 0; off < h && !stalled; off += kSeg) {
      const int f = wb + off, l = min(kSeg, h - off);
      if (stg.first[b] >= 0 && stg.first[b] != f) {  // a prefetch of another segment: cannot happen
        raise(status, ECL_ERR_CUDA, r);
        stalled = true;
        break;
      }
      if (stg.first[b] != f) stg.issue(b, nl2, f, l);  // not prefetched
      // prefetch what comes next: this row's next segment, or the first one
      // of the warp's next row with entries (rows without any are skipped)
      __syncwarp();  // buffer b ^ 1 was scanned by every lane
      if (off + kSeg < h) {
        stg.issue(b ^ 1, nl2, f + kSeg, min(kSeg, h - off - kSeg));
      } else {
        for (int jn = j + 1; jn < nrows; jn++) {
          const int4 nx = row_of(jn);
          if (nx.y > 0) {
            stg.issue(b ^ 1, nl2, nx.x, min(kSeg, nx.y));
            break;
          }
        }
      }
      if (!__all_sync(kFull, stg.wait(b))) {  // every lane polls; the verdict is the warp's
        raise(status, ECL_ERR_NO_CONVERGENCE, r);
        stalled = true;
        break;
      }
      const int* seg = stg.buf[b] + stg.offset(b);
      stg.first[b] = -1;
      // scan the staged entries: colours already published go into the
      // bitmap, the others into the pending list
      for (int i0 = 0; i0 < l; i0 += 32 * kCoreBatch) {
        int q[kCoreBatch];
        unsigned c[kCoreBatch];
#pragma unroll
        for (int k = 0; k < kCoreBatch; k++) {
          const int i = i0 + 32 * k + lane;
          q[k] = i < l ? seg[i] : -1;
          if (i < l && (unsigned)q[k] >= (unsigned)r) {
            raise(status, ECL_ERR_BAD_GRAPH, r);
            q[k] = -1;
          }
        }
#pragma unroll
        for (int k = 0; k < kCoreBatch; k++) c[k] = q[k] >= 0 ? col_ld(&col_s[q[k]]) : 0u;
#pragma unroll
        for (int k = 0; k < kCoreBatch; k++) {
          const bool undecided = q[k] >= 0 && c[k] == kUncoloured;
          if (q[k] >= 0 && !undecided) gc_mark(bits, (int)c[k], 0);
          const unsigned ub = __ballot_sync(kFull, undecided);
          if (undecided) pend[np + __popc(ub & lt)] = (unsigned short)q[k];
          np += __popc(ub);
        }
      }
      b ^= 1;
      // resolve the pending entries once the list could not take another
      // segment, and at the end of the row
      if (np + kSeg > kCorePend || off + kSeg >= h) {  // before the list could overflow, and at the row's end
        __syncwarp();
        for (int jj = lane; jj < np && !stalled; jj += 32) {
          const int cc = gc_core_wait(col_s, pend[jj], status);
          if (cc < 0)
            stalled = true;
          else
            gc_mark(bits, cc, 0);
        }
        stalled = __any_sync(kFull, stalled);
        np = 0;
        __syncwarp();
      }
    }
    if (stalled) {
      stg.drain();
      break;
    }
    // the smallest colour of the first window the bitmap leaves free
    __syncwarp();
    const unsigned w0 = bits[lane], w1 = bits[lane + 32];
    const unsigned f0 = __ballot_sync(kFull, w0 != ~0u), f1 = __ballot_sync(kFull, w1 != ~0u);
    int c = -1;
    if (f0) {
      const int wi = __ffs(f0) - 1;
      c = wi * 32 + __ffs(~__shfl_sync(kFull, w0, wi)) - 1;
    } else if (f1) {
      const int wi = __ffs(f1) - 1;
      c = (wi + 32) * 32 + __ffs(~__shfl_sync(kFull, w1, wi)) - 1;
    }
    __syncwarp();
    if (c < 0) {  // all 2048 first colours taken: scan the row again for the next windows
      c = gc_core_row_global(r, wb, wb + h, 32 * kMexWords, nl2, col_s, bits, pend, status);
      if (c < 0) {
        stg.drain();
        break;
      }
    }
    if (lane == 0) {
      col_publish(&col_s[r], (unsigned)c, ctas);
      st(&color[v], c);
    }
    __syncwarp();
  }
  // a CTA's shared memory must outlive every store the others make into it:
  // every warp, done or given up (each wait is bounded), meets here
  if (ctas > 1) cluster_sync();
}

__global__ void __launch_bounds__(kTPB) gc_pull(int n, const int* __restrict__ nindex, const int* __restrict__ nl2,
                                                const int* __restrict__ hc, const int* __restrict__ order,
                                                int* __restrict__ color, GCCtl* __restrict__ ctl, int core_cap,
                                                unsigned long_nap, Status* __restrict__ status) {
  __shared__ unsigned s_bits[kTPB / 32][kMexWords];
  __shared__ int s_pend[kTPB / 32][kPend];
  const int lane = threadIdx.x & 31;
  unsigned* bits = s_bits[threadIdx.x >> 5];
  int* pend = s_pend[threadIdx.x >> 5];
  const int nbig = ld(&ctl->nbig);
  const int gwarp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  // Ranks are dealt to warps round-robin and each warp takes its own in
  // increasing order -- no shared claim counter (one atomic per row on a
  // single word would serialise ~10^6 claims in L2).  Still deadlock-free:
  // the warp holding the lowest unfinished rank is working on it, and all of
  // that vertex's dependencies have lower ranks.
  // Long rows, ONE per warp at a time: every long row in flight scans its
  // higher-priority list concurrently, so the dense hub core's rows all wait
  // at the same time instead of one after another.
  // ranks below the core size were coloured by gc_core
  for (int r = gc_core_size(ctl, core_cap) + gwarp; r < nbig; r += nwarps) {
    const int wv = __ldg(&order[r]);
    const int wb = __ldg(&nindex[wv]);
    const int c = gc_long_row(wb, wb + __ldg(&hc[wv]), nl2, color, bits, pend, kPend, long_nap, status);
    if (c < 0) return;
    if (lane == 0) st(&color[wv], c);
    __syncwarp();
  }
  // Short rows: 32 consecutive ranks per warp step, every lane its own vertex
  // (the order holds the nkeys vertices with entries; the isolated ones were
  // coloured by gc_keys).
  const int nk = min(ld(&ctl->nkeys), n);
  for (int base = nbig + gwarp * 32; base < nk; base += nwarps * 32) {
    const int r = base + lane;
    if (r < nk) {
      const int v = __ldg(&order[r]);
      const int c = gc_short_row(__ldg(&nindex[v]), __ldg(&hc[v]), nl2, color, status);
      if (c >= 0) st(&color[v], c);
    }
    if (__any_sync(kFull, ld(&status->code) != 0)) return;
  }
}

struct GCBufs {
  GCCtl* ctl;
  int* nl2;
  int* hc;
  unsigned long long* keys0;
  unsigned long long* keys1;
  int* vals0;
  int* vals1;
  unsigned* sort_temp;
  unsigned* vhash;
  int2* chunks;
  int4* rowinfo;
};

void gc_layout(Carve& c, int n, int m, GCBufs* b) {
  b->ctl = c.take<GCCtl>(1);
  b->nl2 = c.take<int>((size_t)m + 4);  // 4 spare entries: the core's aligned bulk copies may round up into them
  b->hc = c.take<int>((size_t)n);
  b->keys0 = c.take<unsigned long long>((size_t)n);
  b->keys1 = c.take<unsigned long long>((size_t)n);
  b->vals0 = c.take<int>((size_t)n);
  b->vals1 = c.take<int>((size_t)n);
  b->sort_temp = c.take<unsigned>(radix_temp_words((size_t)n));
  b->vhash = c.take<unsigned>((size_t)n);
  b->chunks = c.take<int2>(row_chunk_capacity(m, kMinChunk));
  b->rowinfo = c.take<int4>((size_t)std::min(n, kCoreMax));
}

}  // namespace

size_t gc_workspace_bytes(int n, int m) {
  Carve c;
  GCBufs b;
  gc_layout(c, n, m, &b);
  return c.bytes();
}

}  // namespace ecl

namespace ecl {

ecl_status gc_enqueue(const GraphDev& g, int* color, char* ws, Status* status, const DeviceInfo& dev,
                      cudaStream_t stream, const UnionInfo* uni, Marker mark) {
  Carve c{ws};
  GCBufs b;
  gc_layout(c, g.n, g.m, &b);
  // Blocks of the pull per SM: a knob, 2 by default.  Fewer warps poll
  // fewer undecided entries at a time; on R-MAT-22 two blocks per SM colour
  // faster than four (1.81 vs 2.15 ms) -- the polls of four blocks load L2
  // enough to slow the dependency chain they wait on.
  const int pull_blocks = dev.gc_pull_blocks > 0 ? dev.gc_pull_blocks : 2;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, gc_pull, kTPB, 0) != cudaSuccess || occ < 1)
    return ECL_ERR_CUDA;
  const int coop_grid = dev.sms * std::min(occ, pull_blocks);
  const int grid = dev.grid_blocks(kTPB, g.n, g.m);
  const RowChunks rc{b.chunks, &b.ctl->nchunks, (int)row_chunk_capacity(g.m, kMinChunk)};
  const Bins bins = bins_of(dev, Bins{kBinLane, kBinChunk});
  // key bits that vary: 32 hash bits + enough bits for any degree <= m
  int degbits = 1;
  while (degbits < 31 && ((long long)1 << degbits) <= (long long)g.m) degbits++;

  if (cudaMemsetAsync(b.ctl, 0, sizeof(GCCtl), stream) != cudaSuccess) return ECL_ERR_CUDA;
  if (cudaMemsetAsync(color, 0xff, sizeof(int) * (size_t)g.n, stream) != cudaSuccess) return ECL_ERR_CUDA;
  const unsigned* vhash = nullptr;
  if (uni && uni->vbase) {
    ECL_LAUNCH(gc_union_hash, grid, kTPB, 0, stream, g.n, uni->vbase, uni->ngraphs, b.vhash);
    vhash = b.vhash;
  }
  // the priority keys first: gc_init compares neighbours by them
  ECL_LAUNCH(gc_keys, grid, kTPB, 0, stream, g.n, g.nindex, b.keys0, b.keys1, b.vals1, vhash, color, b.ctl);
  const bool vec = (reinterpret_cast<uintptr_t>(g.nlist) & 15) == 0 && dev.row_vec;  // 16-byte row loads
  ECL_LAUNCH(gc_init, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, b.nl2, b.hc, rc, bins, vec, b.keys0, status);
  ECL_LAUNCH(gc_init_chunks, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, b.nl2, b.hc, rc, bins.chunk, vec, b.keys0,
             status);
  mark();
  // the nkeys appended pairs, sorted from (keys1, vals1); the per-vertex keys
  // in keys0 are dead once gc_init has run
  const bool in0 = radix_sort_pairs(b.keys1, b.vals1, b.keys0, b.vals0, g.n, 0, 32 + degbits, b.sort_temp, stream,
                                    &b.ctl->nkeys);
  const int* order = in0 ? b.vals0 : b.vals1;
  mark();
  // the hub core (the sort keys are dead now: their buffer holds the ranks)
  const int cap = std::min(std::min(dev.gc_core_ranks > 0 ? dev.gc_core_ranks : kCoreDefault, kCoreMax), g.n);
  int* rank = reinterpret_cast<int*>(b.keys0);
  ECL_LAUNCH(gc_core_rank, grid, kTPB, 0, stream, order, rank, b.ctl, cap);
  ECL_LAUNCH(gc_core_translate, grid, kTPB, 0, stream, g.nindex, b.nl2, b.hc, order, rank, b.rowinfo, b.ctl, cap);
  ECL_CUDA_TRY(cudaFuncSetAttribute(gc_core, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gc_core_smem(cap)));
  // the core's cluster: as many CTAs as asked for when such a cluster fits
  // the device, else one CTA
  const int want = dev.gc_core_ctas > 0 ? dev.gc_core_ctas : kCoreCtas;
  int ctas = 1;
  if (want > 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)want);
    cfg.blockDim = dim3((unsigned)kCoreThreads);
    cfg.dynamicSmemBytes = gc_core_smem(cap);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)want;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, gc_core, &cfg) == cudaSuccess && clusters >= 1)
      ctas = want;
    else
      cudaGetLastError();  // no such cluster here: one CTA
  }
  if (ctas > 1)
    ECL_CUDA_TRY(launch_cluster(gc_core, ctas, kCoreThreads, gc_core_smem(cap), stream, b.nl2, b.rowinfo, color,
                                b.ctl, cap, status));
  else
    ECL_LAUNCH(gc_core, 1, kCoreThreads, gc_core_smem(cap), stream, b.nl2, b.rowinfo, color, b.ctl, cap, status);
  mark();
  // the long rows' polls back off to at most gc_poll_ns, 64 ns by default
  // (they carry the dependency chain; the short rows keep 512 ns)
  const unsigned long_nap = dev.gc_poll_ns > 0 ? (unsigned)dev.gc_poll_ns : 64u;
  ECL_CUDA_TRY(launch_cooperative(gc_pull, coop_grid, kTPB, stream, g.n, g.nindex, b.nl2, b.hc, order, color, b.ctl,
                                  cap, long_nap, status));
  mark();
  return ECL_OK;
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
  GraphDev gd;
  gd.n = s.n;
  gd.m = s.m;
  gd.nindex = s.nindex;
  gd.nlist = s.nlist;
  gd.flags = g->flags;
  s.start_timer();
  st = gc_enqueue(gd, color, s.ws, s.status, s.dev, s.stream, nullptr, Marker{&s});
  s.stop_timer();
  return s.finish(st);
}

extern "C" ecl_status ecl_compute_gc(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist,
                                     int32_t* color) {
  ecl_graph_view g{nodes, edges, nidx, nlist, nullptr, ECL_HOST, 0};
  ecl_opts o{};
  return ecl_gc(&g, color, &o);
}

// ---- the colouring's critical path (a host-side diagnostic) --------------------
//
// The colour of a vertex is fixed only after every higher-priority neighbour
// has its own, so no schedule finishes faster than the longest chain of such
// dependencies.  This walks the priority order once on the host: hops[v] = 1 +
// the largest hops[u] over v's higher-priority entries u (0 with none), and a
// time model path[v] = the latest path[u] + the cost of one hop to v -- the
// shared-memory hop for a vertex the GPU colours in its core (the first
// min(long rows, core_ranks) ranks), the L2 hop for every other one.  The
// bench reports the resulting latency bound beside gc_pull's time.
extern "C" ecl_status ecl_gc_critical_path(const ecl_graph_view* g, int32_t core_ranks, double hop_core_ns,
                                           double hop_rest_ns, int32_t* hops, int32_t* hops_core, double* path_ns) {
  using namespace ecl;
  if (!g || g->location != ECL_HOST || g->nodes < 1 || g->edges < 0 || !g->nindex || (g->edges > 0 && !g->nlist))
    return ECL_ERR_INVALID_ARG;
  if (core_ranks < 0 || core_ranks > kCoreMax) return ECL_ERR_INVALID_ARG;
  const int n = g->nodes;
  const int* nindex = g->nindex;
  const int* nlist = g->nlist;
  for (int v = 0; v < n; v++)
    if (nindex[v] < 0 || nindex[v + 1] < nindex[v] || nindex[v + 1] > g->edges) return ECL_ERR_BAD_GRAPH;
  std::vector<unsigned long long> key((size_t)n);
  int nbig = 0;
  for (int v = 0; v < n; v++) {
    const unsigned deg = (unsigned)(nindex[v + 1] - nindex[v]);
    key[(size_t)v] = ((unsigned long long)deg << 32) | dev::ecl_hash((unsigned)v);
    nbig += deg > (unsigned)kWarpRow;
  }
  std::vector<int> order((size_t)n);
  for (int v = 0; v < n; v++) order[(size_t)v] = v;
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    return key[(size_t)a] != key[(size_t)b] ? key[(size_t)a] > key[(size_t)b] : a > b;
  });
  std::vector<int> rank((size_t)n);
  for (int r = 0; r < n; r++) rank[(size_t)order[(size_t)r]] = r;
  const int core = std::min(nbig, core_ranks > 0 ? core_ranks : kCoreDefault);
  std::vector<int> hop((size_t)n, 0);
  std::vector<double> path((size_t)n, 0.0);
  int best = 0, best_core = 0;
  double best_path = 0.0;
  for (int r = 0; r < n; r++) {
    const int v = order[(size_t)r];
    int h = -1;
    double t = -1.0;
    for (int i = nindex[v]; i < nindex[v + 1]; i++) {
      const int u = nlist[i];
      if (u < 0 || u >= n) return ECL_ERR_BAD_GRAPH;
      if (u == v || rank[(size_t)u] > r) continue;
      h = std::max(h, hop[(size_t)u]);
      t = std::max(t, path[(size_t)u]);
    }
    hop[(size_t)v] = h + 1;
    path[(size_t)v] = t < 0.0 ? 0.0 : t + (r < core ? hop_core_ns : hop_rest_ns);
    best = std::max(best, hop[(size_t)v]);
    if (r < core) best_core = std::max(best_core, hop[(size_t)v]);
    best_path = std::max(best_path, path[(size_t)v]);
  }
  if (hops) *hops = best;
  if (hops_core) *hops_core = best_core;
  if (path_ns) *path_ns = best_path;
  return ECL_OK;
}
