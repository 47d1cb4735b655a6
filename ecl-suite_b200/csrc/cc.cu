// Connected components (ECL-CC contract).
//
// Result contract (src/racefree/egr-input/CC/ECL-CC-atomic.cu): every vertex v
// hooks only along its list entries u = nlist[i] with u < v (:132, :174,
// :218), roots are always hooked larger -> smaller (:139-146) and flatten
// points each vertex at its root (:250-264).  Hence the label of v is the
// smallest vertex id of v's component in the graph whose edges are
// {(v, u) : u in list(v), u < v}.  That value does not depend on the schedule,
// so any union-find with the same hooking rule reproduces it bit for bit.
//
// B200 design (graphs flagged ECL_GRAPH_SYMMETRIC take the sampling path
// further down: link the first two entries of every list, find the giant
// component, then skip every list inside it):
//  * cc_init   - parent[v] = first smaller neighbour among the first
//                kInitScan entries (one free hook per vertex).
//  * cc_hook   - one pass over the vertices, 32 per warp.  Lists of <= 16
//                entries are walked by their own lane; lists of up to
//                2048 entries are walked by the whole warp (ballot loop,
//                coalesced 128-byte nlist reads); longer lists are cut into
//                2048-entry chunk records for cc_chunks (both thresholds
//                are launch knobs).
//  * cc_chunks - warp per chunk record, so a 163k-entry R-MAT hub is spread
//                over ~160 warps instead of serialising one block.
//  * cc_flatten- label[v] = root(v).
// The parent array IS the output label array (no extra n-sized buffer).
// All parent accesses are device-scope relaxed atomics; links use CAS.
#include "solvers.cuh"

#include <mutex>

namespace ecl {
namespace {

using namespace dev;

constexpr int kTPB = 256;
// Default degree bins: lists of <= 16 entries per lane, chunk records of
// 2048 entries (a launch knob may change both).
constexpr Bins kCCBins{16, 2048};
constexpr int kInitScan = 8;   // entries cc_init looks at for a first smaller neighbour

// Row [beg, end) of v, or empty when the row is malformed (cc_init reports it).
__device__ __forceinline__ void cc_row(const int* nindex, int v, int m, int& beg, int& end) {
  beg = __ldg(&nindex[v]);
  end = __ldg(&nindex[v + 1]);
  if (beg < 0 || end < beg || end > m) beg = end = 0;
}

// Entries outside [0, n) raise ECL_ERR_BAD_GRAPH and are skipped.
__device__ __forceinline__ bool cc_valid(int u, int n, Status* status) {
  if ((unsigned)u < (unsigned)n) return true;
  raise(status, ECL_ERR_BAD_GRAPH, u);
  return false;
}

struct CCCounters {
  int nchunks;
  int giant;  // root of the sampled largest component (symmetric path)
  int pad[62];
};

// Root of v with path splitting.  Parent pointers only ever point at
// smaller ids, so a vertex is a root iff parent[v] == v.
__device__ __forceinline__ int cc_root(int v, int* parent) {
  int cur = ld(&parent[v]);
  if (cur == v) return v;
  int prev = v;
  int next;
  while (cur > (next = ld(&parent[cur]))) {
    st(&parent[prev], next);
    prev = cur;
    cur = next;
  }
  return cur;
}

// Links the trees rooted (as last seen) at a and b; returns the root that
// survived the link as last seen by this thread.
__device__ __forceinline__ int cc_link(int a, int b, int* parent) {
  while (a != b) {
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int seen = cas(&parent[a], a, b);
    if (seen == a) return b;
    // Another thread already hung a under b: the two trees are one.  On a
    // mesh every vertex of a column links the same pair of roots, and all but
    // one would otherwise walk the freshly linked chain of roots.
    if (seen == b) return b;
    a = cc_root(seen, parent);
    b = cc_root(b, parent);
  }
  return a;
}

// Joins the trees of u and v without first walking to either root (the Link
// step of Sutton, Ben-Nun and Barak, IPDPS 2018): look one level above the
// larger side; if that already is the smaller side the trees are one, if it
// is a root hang it under the smaller side, otherwise climb two levels and
// retry.  Parents only point at smaller ids, so the loop ends.  A mesh links
// the same pair of roots from every vertex of a column; a full root walk
// there follows a chain of roots that grows while it is being walked.
__device__ __forceinline__ void cc_union(int u, int v, int* parent) {
  int p1 = ld(&parent[u]);
  int p2 = ld(&parent[v]);
  while (p1 != p2) {
    const int high = max(p1, p2), low = min(p1, p2);
    const int ph = ld(&parent[high]);
    if (ph == low) return;
    if (ph == high && cas(&parent[high], high, low) == high) return;
    p1 = ld(&parent[ld(&parent[high])]);
    p2 = ld(&parent[low]);
  }
}

// Also checks the CSR rows once: a malformed row (end < beg, or outside
// [0, m]) raises ECL_ERR_BAD_GRAPH and is treated as empty by every kernel.
// kHook = false: every vertex starts as its own root (the symmetric path,
// whose sampling rounds do the first links).
template <bool kHook>
__global__ void __launch_bounds__(kTPB) cc_init(int n, int m, const int* __restrict__ nindex,
                                                const int* __restrict__ nlist, int* __restrict__ parent,
                                                Status* __restrict__ status) {
  for (int v = blockIdx.x * kTPB + threadIdx.x; v < n; v += gridDim.x * kTPB) {
    int beg = __ldg(&nindex[v]), end = __ldg(&nindex[v + 1]);
    if (beg < 0 || end < beg || end > m) {
      raise(status, ECL_ERR_BAD_GRAPH, v);
      beg = end = 0;
    }
    // Only the first few entries are looked at: the hook is an optional head
    // start (the labels do not depend on it), and scanning a whole hub row
    // from one thread would serialise a 163k-entry R-MAT hub.
    int p = v;
    const int stop = kHook ? min(end, beg + kInitScan) : beg;
    for (int i = beg; i < stop; i++) {
      const int u = __ldg(&nlist[i]);
      if (u < v && u >= 0) {
        p = u;
        break;
      }
    }
    parent[v] = p;  // race-free: thread-owned init, no reader in this launch
  }
}

// Chunk records of chunk_capacity(m, chunk) cover every long row of a CSR
// whose rows do not overlap (a row of d > chunk entries needs
// ceil(d / chunk) < 2 d / chunk records).  A malformed CSR with overlapping
// rows can ask for more: the excess raises ECL_ERR_BAD_GRAPH and is not
// written.
constexpr int chunk_capacity(int m, int chunk) { return 2 * (m / chunk) + 2; }

__device__ __forceinline__ void cc_push_chunks(int v, int beg, int deg, int chunk, int2* chunks, int cap,
                                               CCCounters* ctr, Status* status) {
  const int nc = (deg + chunk - 1) / chunk;
  const int at = fetch_add(&ctr->nchunks, nc);
  for (int c = 0; c < nc; c++) {
    if ((unsigned)(at + c) < (unsigned)cap)
      chunks[at + c] = make_int2(v, beg + c * chunk);
    else
      raise(status, ECL_ERR_BAD_GRAPH, v);
  }
}

// Records the chunk kernels may read: the requested count clamped to cap.
__device__ __forceinline__ int cc_chunk_total(const CCCounters* ctr, int cap) {
  const int c = ctr->nchunks;
  return (c < 0 || c > cap) ? cap : c;
}

__global__ void __launch_bounds__(kTPB) cc_hook(int n, int m, const int* __restrict__ nindex,
                                                const int* __restrict__ nlist, int* __restrict__ parent,
                                                int2* __restrict__ chunks, int chunk_cap, Bins bins,
                                                CCCounters* __restrict__ ctr, Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    const int v = base + lane;
    int beg = 0, end = 0;
    if (v < n) cc_row(nindex, v, m, beg, end);
    const int deg = end - beg;
    if (deg > bins.chunk) {
      cc_push_chunks(v, beg, deg, bins.chunk, chunks, chunk_cap, ctr, status);
    } else if (deg > 0 && deg <= bins.lane) {
      int rv = -1;
      for (int i = beg; i < end; i++) {
        const int u = __ldg(&nlist[i]);
        if (u < v && cc_valid(u, n, status)) {
          if (rv < 0) rv = cc_root(v, parent);
          const int ru = cc_root(u, parent);
          if (ru != rv) rv = cc_link(rv, ru, parent);
        }
      }
    }
    // Medium lists: the whole warp walks one list at a time.
    unsigned mid = __ballot_sync(kFull, deg > bins.lane && deg <= bins.chunk);
    while (mid) {
      const int who = __ffs(mid) - 1;
      mid &= mid - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      int rv = -1;
      for (int i = wbeg + lane; i < wend; i += 32) {
        const int u = __ldg(&nlist[i]);
        if (u < wv && cc_valid(u, n, status)) {
          if (rv < 0) rv = cc_root(wv, parent);
          const int ru = cc_root(u, parent);
          if (ru != rv) rv = cc_link(rv, ru, parent);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kTPB) cc_chunks(int n, const int* __restrict__ nindex,
                                                  const int* __restrict__ nlist, int* __restrict__ parent,
                                                  const int2* __restrict__ chunks, int chunk_cap, int chunk,
                                                  const CCCounters* __restrict__ ctr, Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int total = cc_chunk_total(ctr, chunk_cap);
  for (int c = warp; c < total; c += nwarps) {
    const int2 rec = chunks[c];
    const int v = rec.x;
    const int end = min(rec.y + chunk, __ldg(&nindex[v + 1]));
    int rv = -1;
    for (int i = rec.y + lane; i < end; i += 32) {
      const int u = __ldg(&nlist[i]);
      if (u < v && cc_valid(u, n, status)) {
        if (rv < 0) rv = cc_root(v, parent);
        const int ru = cc_root(u, parent);
        if (ru != rv) rv = cc_link(rv, ru, parent);
      }
    }
  }
}

// parent[v] = root(v) by pointer jumping: each thread only rewrites its own
// parent[v], once per step, and steps to the parent of its current target.
// Threads on the same chain run side by side, so every step reads a target
// that has itself jumped -- a chain of depth D is flattened in about log2(D)
// dependent loads per thread instead of D (a mesh builds chains as long as a
// grid column).  parent[v] has no other writer during the launch, so the
// array ends fully flat.
__global__ void __launch_bounds__(kTPB) cc_flatten(int n, int* __restrict__ parent) {
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

// ---- symmetric graphs: sampling + giant-component skip ----------------------
//
// For a symmetric graph the components over the entries u < v are the plain
// connected components, so every entry may be used in either direction
// (Sutton, Ben-Nun and Barak, "Optimizing parallel graph connectivity
// computation via subgraph sampling", IPDPS 2018).  Links still hook the
// larger root under the smaller one, so the labels stay the minimum ids.

constexpr int kSample = 2;  // list entries linked per vertex before the skip

// Sampling round r: links v with the r-th entry of its list.  The rounds run
// as separate launches with a full compression in between, so every find of
// the next round starts one step from its root -- on a mesh, linking both
// samples at once builds chains as long as a grid column.
__global__ void __launch_bounds__(kTPB) cc_sample(int n, int m, const int* __restrict__ nindex,
                                                  const int* __restrict__ nlist, int* __restrict__ parent, int r,
                                                  Status* __restrict__ status) {
  for (int v = blockIdx.x * kTPB + threadIdx.x; v < n; v += gridDim.x * kTPB) {
    int beg, end;
    cc_row(nindex, v, m, beg, end);
    if (beg + r >= end) continue;
    const int u = __ldg(&nlist[beg + r]);
    if (u == v || !cc_valid(u, n, status)) continue;
    cc_union(v, u, parent);
  }
}

// One block: the most frequent root among 1024 sampled vertices.
__global__ void __launch_bounds__(1024) cc_giant(int n, const int* __restrict__ parent, CCCounters* __restrict__ ctr) {
  __shared__ int s[1024];
  const int t = threadIdx.x;
  s[t] = ld(&parent[ecl_hash((unsigned)t * 2654435761u + 97u) % (unsigned)n]);
  __syncthreads();
  for (int k = 2; k <= 1024; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int p = t ^ j;
      if (p > t) {
        const int a = s[t], b = s[p];
        if ((a > b) == ((t & k) == 0)) {
          s[t] = b;
          s[p] = a;
        }
      }
      __syncthreads();
    }
  }
  // Longest run of equal roots, ties to the smallest root: every run start
  // finds its end by binary search, then a block-wide max over
  // (length, ~root) keys (a serial scan by one thread cost ~15 us).
  unsigned long long key = 0;
  if (t == 0 || s[t] != s[t - 1]) {
    int lo = t + 1, hi = 1024;  // first index past the run
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (s[mid] == s[t])
        lo = mid + 1;
      else
        hi = mid;
    }
    key = ((unsigned long long)(lo - t) << 32) | (0xffffffffu - (unsigned)s[t]);
  }
  for (int o = 16; o > 0; o >>= 1) key = max(key, __shfl_xor_sync(kFull, key, o));
  __shared__ unsigned long long wbest[32];
  if ((t & 31) == 0) wbest[t >> 5] = key;
  __syncthreads();
  if (t < 32) {
    key = wbest[t];
    for (int o = 16; o > 0; o >>= 1) key = max(key, __shfl_xor_sync(kFull, key, o));
    if (t == 0) ctr->giant = (int)(0xffffffffu - (unsigned)key);
  }
}

// Frozen membership of the sampled giant component (parent is flattened).
__global__ void __launch_bounds__(kTPB) cc_mark_giant(int n, const int* __restrict__ parent,
                                                      const CCCounters* __restrict__ ctr,
                                                      unsigned char* __restrict__ ing) {
  const int gr = ctr->giant;
  for (int v = blockIdx.x * kTPB + threadIdx.x; v < n; v += gridDim.x * kTPB) ing[v] = parent[v] == gr;  // race-free: parent is not written in this launch
}

// Remaining entries of vertices outside the giant component.  An entry is
// linked when u < v (the other direction is handled from u) or when u is in
// the giant component (u skips its list entirely).
__device__ __forceinline__ bool cc_rest_wanted(int u, int v, const unsigned char* ing) {
  return u != v && (u < v || __ldg(&ing[u]));
}

__global__ void __launch_bounds__(kTPB) cc_rest(int n, int m, const int* __restrict__ nindex,
                                                const int* __restrict__ nlist, int* __restrict__ parent,
                                                const unsigned char* __restrict__ ing, int2* __restrict__ chunks,
                                                int chunk_cap, Bins bins, CCCounters* __restrict__ ctr,
                                                Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    const int v = base + lane;
    int beg = 0, end = 0;
    if (v < n && !__ldg(&ing[v])) {
      cc_row(nindex, v, m, beg, end);
      beg = min(end, beg + kSample);  // the first entries were linked by cc_sample
    }
    const int deg = end - beg;
    if (deg > bins.chunk) {
      cc_push_chunks(v, beg, deg, bins.chunk, chunks, chunk_cap, ctr, status);
    } else if (deg > 0 && deg <= bins.lane) {
      int rv = -1;
      for (int i = beg; i < end; i++) {
        const int u = __ldg(&nlist[i]);
        if (cc_valid(u, n, status) && cc_rest_wanted(u, v, ing)) {
          if (rv < 0) rv = cc_root(v, parent);
          const int ru = cc_root(u, parent);
          if (ru != rv) rv = cc_link(rv, ru, parent);
        }
      }
    }
    unsigned mid = __ballot_sync(kFull, deg > bins.lane && deg <= bins.chunk);
    while (mid) {
      const int who = __ffs(mid) - 1;
      mid &= mid - 1;
      const int wv = __shfl_sync(kFull, v, who);
      const int wbeg = __shfl_sync(kFull, beg, who);
      const int wend = __shfl_sync(kFull, end, who);
      int rv = -1;
      for (int i = wbeg + lane; i < wend; i += 32) {
        const int u = __ldg(&nlist[i]);
        if (cc_valid(u, n, status) && cc_rest_wanted(u, wv, ing)) {
          if (rv < 0) rv = cc_root(wv, parent);
          const int ru = cc_root(u, parent);
          if (ru != rv) rv = cc_link(rv, ru, parent);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kTPB) cc_rest_chunks(int n, const int* __restrict__ nindex,
                                                       const int* __restrict__ nlist, int* __restrict__ parent,
                                                       const unsigned char* __restrict__ ing,
                                                       const int2* __restrict__ chunks, int chunk_cap, int chunk,
                                                       const CCCounters* __restrict__ ctr, Status* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kTPB + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kTPB) >> 5;
  const int total = cc_chunk_total(ctr, chunk_cap);
  for (int c = warp; c < total; c += nwarps) {
    const int2 rec = chunks[c];
    const int v = rec.x;
    const int end = min(rec.y + chunk, __ldg(&nindex[v + 1]));
    int rv = -1;
    for (int i = rec.y + lane; i < end; i += 32) {
      const int u = __ldg(&nlist[i]);
      if (cc_valid(u, n, status) && cc_rest_wanted(u, v, ing)) {
        if (rv < 0) rv = cc_root(v, parent);
        const int ru = cc_root(u, parent);
        if (ru != rv) rv = cc_link(rv, ru, parent);
      }
    }
  }
}

void cc_layout(Carve& c, int n, int m, CCCounters** ctr, int2** chunks, unsigned char** ing = nullptr) {
  *ctr = c.take<CCCounters>(1);
  *chunks = c.take<int2>((size_t)chunk_capacity(m, kMinChunk));
  unsigned char* g = c.take<unsigned char>((size_t)n);
  if (ing) *ing = g;
}

}  // namespace

size_t cc_workspace_bytes(int n, int m) {
  Carve c;
  CCCounters* ctr;
  int2* chunks;
  cc_layout(c, n, m, &ctr, &chunks);
  return c.bytes();
}

}  // namespace ecl

namespace ecl {

ecl_status cc_enqueue(const GraphDev& g, int* parent, char* ws, Status* status, const DeviceInfo& dev,
                      cudaStream_t stream, Marker mark) {
  Carve c{ws};
  CCCounters* ctr;
  int2* chunks;
  unsigned char* ing;
  cc_layout(c, g.n, g.m, &ctr, &chunks, &ing);
  const int grid = dev.grid_blocks(kTPB, g.n, g.m);
  const Bins bins = bins_of(dev, kCCBins);
  const int cap = chunk_capacity(g.m, kMinChunk);  // cc_layout sized the records for the smallest chunk
  ECL_CUDA_TRY(cudaMemsetAsync(ctr, 0, sizeof(CCCounters), stream));
  if (g.flags & ECL_GRAPH_SYMMETRIC) {
    ECL_LAUNCH(cc_init<false>, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, parent, status);
    for (int r = 0; r < kSample; r++) {
      ECL_LAUNCH(cc_sample, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, parent, r, status);
      ECL_LAUNCH(cc_flatten, grid, kTPB, 0, stream, g.n, parent);
    }
    ECL_LAUNCH(cc_giant, 1, 1024, 0, stream, g.n, parent, ctr);
    ECL_LAUNCH(cc_mark_giant, grid, kTPB, 0, stream, g.n, parent, ctr, ing);
    mark();
    ECL_LAUNCH(cc_rest, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, parent, ing, chunks, cap, bins, ctr,
               status);
    mark();
    ECL_LAUNCH(cc_rest_chunks, grid, kTPB, 0, stream, g.n, g.nindex, g.nlist, parent, ing, chunks, cap, bins.chunk,
               ctr, status);
    mark();
    ECL_LAUNCH(cc_flatten, grid, kTPB, 0, stream, g.n, parent);
    mark();
    return ECL_OK;
  }
  ECL_LAUNCH(cc_init<true>, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, parent, status);
  mark();
  ECL_LAUNCH(cc_hook, grid, kTPB, 0, stream, g.n, g.m, g.nindex, g.nlist, parent, chunks, cap, bins, ctr, status);
  mark();
  ECL_LAUNCH(cc_chunks, grid, kTPB, 0, stream, g.n, g.nindex, g.nlist, parent, chunks, cap, bins.chunk, ctr, status);
  mark();
  ECL_LAUNCH(cc_flatten, grid, kTPB, 0, stream, g.n, parent);
  mark();
  return ECL_OK;
}

}  // namespace ecl

extern "C" ecl_status ecl_cc(const ecl_graph_view* g, int32_t* label, ecl_opts* opts) {
  using namespace ecl;
  ecl_opts local{};
  if (!opts) opts = &local;
  if (!label) return ECL_ERR_INVALID_ARG;
  Solve s(g, opts);
  // The sampling path of a graph flagged ECL_GRAPH_SYMMETRIC uses every entry
  // in both directions, so validation (opts->validate) checks that flag: an
  // asymmetric graph carrying it would get labels other than the reference's
  // u < v hooking gives.
  GraphNeeds needs;
  needs.symmetric = g && (g->flags & ECL_GRAPH_SYMMETRIC);
  ecl_status st = s.begin(needs, g ? cc_workspace_bytes(g->nodes, g->edges) : 0);
  if (st != ECL_OK) return s.finish(st);
  int* parent = s.output(label, (size_t)s.n);
  if (!parent) return s.finish(ECL_ERR_OOM);
  GraphDev gd;
  gd.n = s.n;
  gd.m = s.m;
  gd.nindex = s.nindex;
  gd.nlist = s.nlist;
  gd.flags = g->flags;
  s.start_timer();
  st = cc_enqueue(gd, parent, s.ws, s.status, s.dev, s.stream, Marker{&s});
  s.stop_timer();
  return s.finish(st);
}

// ---- allocation-free variant --------------------------------------------------
//
// ecl_cc_noalloc runs the same four kernels with its scratch (status block,
// counters, chunk records) in a fixed array that lives in this library's
// device memory, so the call itself allocates nothing.  Every GPU that loads
// the library holds the array until the process exits.

namespace ecl {
namespace {

constexpr size_t kNoAllocBytes = ECL_CC_NOALLOC_SCRATCH_BYTES;
// The allocation-free path always uses the default bins (no knob may enlarge
// its fixed array), so its records are sized for kCCBins.chunk.
static_assert(kStatusBytes + sizeof(CCCounters) + 256 +
                      sizeof(int2) * (size_t)chunk_capacity(ECL_CC_NOALLOC_MAX_EDGES, kCCBins.chunk) <=
                  kNoAllocBytes,
              "no-alloc scratch too small for ECL_CC_NOALLOC_MAX_EDGES");

static __device__ __align__(256) unsigned char g_cc_noalloc_scratch[kNoAllocBytes];

// cuCtxGetCurrent, reached through the runtime's driver entry point so the
// library needs no link against libcuda.
typedef int (*CtxGetCurrentFn)(void** ctx);

std::mutex g_noalloc_mu;
struct NoAllocSlot {
  void* ctx = nullptr;   // context the address belongs to
  void* addr = nullptr;  // device address of g_cc_noalloc_scratch in it
};
NoAllocSlot g_noalloc_slot[64];

// Device address of g_cc_noalloc_scratch on the current device (host code
// cannot use the symbol itself as a pointer).  It is looked up once per
// device and kept with the context it was found in: after cudaDeviceReset
// the device has a new primary context, the module is loaded again, and the
// address is looked up again instead of reusing a dead one.
ecl_status noalloc_scratch(int device, void** out) {
  if (device < 0 || device >= 64) return ECL_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  static CtxGetCurrentFn ctx_get = nullptr;
  if (!ctx_get) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      set_last_error_msg("ecl_cc_noalloc: cuCtxGetCurrent is not available");
      return ECL_ERR_CUDA;
    }
    ctx_get = reinterpret_cast<CtxGetCurrentFn>(fn);
  }
  void* ctx = nullptr;
  if (ctx_get(&ctx) != 0 || !ctx) {
    set_last_error_msg("ecl_cc_noalloc: no current CUDA context");
    return ECL_ERR_CUDA;
  }
  NoAllocSlot& slot = g_noalloc_slot[device];
  if (slot.ctx != ctx || !slot.addr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_cc_noalloc_scratch);
    if (e != cudaSuccess) {
      set_last_error("cudaGetSymbolAddress(g_cc_noalloc_scratch)", e);
      return ECL_ERR_CUDA;
    }
    slot.ctx = ctx;
    slot.addr = p;
  }
  *out = slot.addr;
  return ECL_OK;
}

}  // namespace
}  // namespace ecl

extern "C" ecl_status ecl_cc_noalloc(int32_t nodes, int32_t edges, const int32_t* nindex, const int32_t* nlist,
                                     int32_t* label, void* stream_ptr) {
  using namespace ecl;
  if (nodes < 1 || edges < 0) return ECL_ERR_BAD_GRAPH;
  if (!nindex || !label || (edges > 0 && !nlist)) return ECL_ERR_INVALID_ARG;
  if (edges > ECL_CC_NOALLOC_MAX_EDGES) {
    set_last_error_msg("ecl_cc_noalloc: graph has more CSR entries than ECL_CC_NOALLOC_MAX_EDGES; use ecl_cc");
    return ECL_ERR_UNSUPPORTED;
  }
  DeviceInfo dev;
  ecl_status st = current_device(&dev);
  if (st != ECL_OK) return st;
  void* base = nullptr;
  st = noalloc_scratch(dev.device, &base);
  if (st != ECL_OK) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  Status* status = static_cast<Status*>(base);
  Carve c{static_cast<char*>(base) + kStatusBytes};
  CCCounters* ctr;
  int2* chunks;
  cc_layout(c, nodes, edges, &ctr, &chunks);
  // The array keeps the previous call's contents: clear the status block and
  // the counters (adjacent, at the front of the array) before every solve.
  ECL_CUDA_TRY(cudaMemsetAsync(base, 0, kStatusBytes + sizeof(CCCounters), stream));
  const int grid = dev.grid_blocks(kTPB, nodes, edges);
  ECL_LAUNCH(cc_init<true>, grid, kTPB, 0, stream, nodes, edges, nindex, nlist, label, status);
  ECL_LAUNCH(cc_hook, grid, kTPB, 0, stream, nodes, edges, nindex, nlist, label, chunks,
             chunk_capacity(edges, kCCBins.chunk), kCCBins, ctr, status);
  ECL_LAUNCH(cc_chunks, grid, kTPB, 0, stream, nodes, nindex, nlist, label, chunks,
             chunk_capacity(edges, kCCBins.chunk), kCCBins.chunk, ctr, status);
  ECL_LAUNCH(cc_flatten, grid, kTPB, 0, stream, nodes, label);
  Status hs{};
  ECL_CUDA_TRY(cudaMemcpyAsync(&hs, status, sizeof(hs), cudaMemcpyDeviceToHost, stream));
  ECL_CUDA_TRY(cudaStreamSynchronize(stream));
  ECL_CUDA_TRY(cudaGetLastError());
  return static_cast<ecl_status>(hs.code);
}

extern "C" ecl_status ecl_compute_cc(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist,
                                     int32_t* nstat) {
  ecl_graph_view g{nodes, edges, nidx, nlist, nullptr, ECL_HOST, 0};
  ecl_opts o{};
  return ecl_cc(&g, nstat, &o);
}
