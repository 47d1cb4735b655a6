// Degree binning shared by the CSR scans.
//
// A row of <= bins.lane entries is walked by its own lane, all lanes of the
// warp stepping through entry offset k together (so warp-aggregated appends
// stay converged); a row of <= bins.chunk entries by the whole warp, 32
// entries per step; a longer row is cut into bins.chunk-entry chunk records
// that a second launch spreads over all warps.  R-MAT puts its heaviest rows
// at the lowest ids, i.e. in the same warp groups, so the chunk size -- not
// the lane/warp split -- bounds the work of the slowest warp.  Both
// thresholds are launch knobs (ecl_tune): each scan has its own default, and
// the results never depend on them.
#pragma once

#include "common.cuh"
#include "ecl_b200.h"

namespace ecl {
namespace dev {

constexpr int kBinLane = 32;
constexpr int kBinChunk = 256;
// Smallest chunk a knob may ask for: workspaces hold chunk records for it.
constexpr int kMinChunk = 128;
constexpr int kMaxChunk = 8192;

struct Bins {
  int lane;   // rows of at most this many entries: one lane (1..32)
  int chunk;  // rows longer than this: chunk records of this many entries (power of two)
};

// Chunk records of the long rows.  `cap` records fit: 2 * (m / chunk) + 2
// covers every row of a CSR whose rows do not overlap (each long row of d
// entries needs ceil(d / chunk) < 2 d / chunk records); a malformed CSR whose
// rows overlap can ask for more, and the excess is reported, not written.
struct RowChunks {
  int2* rec;   // (vertex, first entry of the chunk)
  int* count;  // records requested (may exceed cap on a malformed CSR)
  int cap;     // records the buffer holds
};

__host__ __device__ constexpr size_t row_chunk_capacity(int m, int chunk = kBinChunk) {
  return 2 * (size_t)(m / chunk) + 2;
}

// Records a consumer may read: the requested count clamped to the capacity.
__device__ __forceinline__ int chunk_total(const RowChunks& rc) {
  const int c = *rc.count;
  return (c < 0 || c > rc.cap) ? rc.cap : c;
}

// Row [beg, end) of v; a malformed row reports ECL_ERR_BAD_GRAPH and is empty.
__device__ __forceinline__ void csr_row(const int* nindex, int v, int m, int& beg, int& end, Status* status) {
  beg = __ldg(&nindex[v]);
  end = __ldg(&nindex[v + 1]);
  if (beg < 0 || end < beg || end > m) {
    raise(status, ECL_ERR_BAD_GRAPH, v);
    beg = end = 0;
  }
}

// Chunk records for the long rows of a warp's 32 vertices: every lane of the
// warp calls; lanes with `is_long` cut [beg, end) into `chunk`-entry records
// (vertex, first entry).  One atomic per warp reserves all of them
// (R-MAT-22 has ~50k rows over 256 entries; an atomic per row on one counter
// would serialise in L2); the records land in lane order.  Records past the
// capacity (only a CSR with overlapping rows asks for them) raise
// ECL_ERR_BAD_GRAPH and are dropped.
__device__ __forceinline__ void push_chunks_warp(const RowChunks& rc, int chunk, bool is_long, int v, int beg, int end,
                                                 Status* status) {
  const int lane = threadIdx.x & 31;
  const int nc = is_long ? (end - beg + chunk - 1) / chunk : 0;
  if (!__any_sync(kFull, nc > 0)) return;
  int incl = nc;  // inclusive prefix sum over the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  const int total = __shfl_sync(kFull, incl, 31);
  int base = 0;
  if (lane == 0) base = fetch_add(rc.count, total);
  base = __shfl_sync(kFull, base, 0) + incl - nc;
  for (int c = 0; c < nc; c++) {
    if ((unsigned)(base + c) < (unsigned)rc.cap)  // a wrapped counter stays out too
      rc.rec[base + c] = make_int2(v, beg + c * chunk);
    else
      raise(status, ECL_ERR_BAD_GRAPH, v);
  }
}

// Visits the entries [jb, je) of one row with the whole warp, four entries a
// lane per call of f(j, u, valid) -- j[k] the entry index, u[k] = nlist[j[k]],
// valid[k] whether that slot holds an entry of the row; every lane calls f the
// same number of times, so f may use warp collectives.  With `vec` (nlist
// 16-byte aligned) the row is walked in 16-byte-aligned quads of entries, one
// quad a lane and 128 entries a warp step, each read with a single 16-byte
// load; the quads at the two ends of the row are masked to it (the entries of
// the neighbouring rows they also hold are read but not used), and a quad that
// would reach past the array's m entries is read entry by entry.  Without
// `vec` every entry is a 4-byte load, 32 consecutive entries per k.
template <class F>
__device__ __forceinline__ void warp_row(int jb, int je, int m, bool vec, const int* nlist, F&& f) {
  const int lane = threadIdx.x & 31;
  int j[4], u[4];
  bool valid[4];
  if (!vec) {
    for (int i0 = jb; i0 < je; i0 += 128) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        j[k] = i0 + 32 * k + lane;
        valid[k] = j[k] < je;
        u[k] = valid[k] ? __ldg(&nlist[j[k]]) : -1;
      }
      f(j, u, valid);
    }
    return;
  }
  for (int i0 = jb & ~3; i0 < je; i0 += 128) {
    const int q = i0 + 4 * lane;  // this lane's quad [q, q + 4)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      j[k] = q + k;
      valid[k] = j[k] >= jb && j[k] < je;
    }
    if (q + 4 <= m && q < je) {
      const int4 x = __ldg(reinterpret_cast<const int4*>(nlist + q));
      u[0] = x.x, u[1] = x.y, u[2] = x.z, u[3] = x.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) u[k] = valid[k] ? __ldg(&nlist[j[k]]) : -1;
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (!valid[k]) u[k] = -1;
    f(j, u, valid);
  }
}

// Warp-aggregated slot in an append-only list; every lane of the warp calls.
__device__ __forceinline__ int warp_append(int* counter, bool pred) {
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(kFull, pred);
  if (bal == 0) return -1;
  int base = 0;
  if (lane == 0) base = fetch_add(counter, __popc(bal));
  base = __shfl_sync(kFull, base, 0);
  return pred ? base + __popc(bal & ((1u << lane) - 1)) : -1;
}

// Per-warp staging of an append-only list in shared memory.  Lanes append
// into the warp's own kCap-slot buffer (ballot + popc, no atomics); when fewer
// than 32 slots are left the warp reserves room in the global list with ONE
// atomic and writes the buffer out with coalesced stores.  A global counter
// then sees one atomic per ~kCap entries instead of one per warp step --
// appends from every warp of the grid to a single counter serialise in L2.
// All lanes call push() and flush() together; flush() once more at the end.
// kStream: write the list with evict-first stores, for a list much larger
// than L2 that must not push the per-vertex arrays out of it.
template <typename T, int kCap, bool kStream = false>
struct WarpStage {
  T* buf;         // this warp's kCap slots in shared memory
  int count = 0;  // warp-uniform

  // `overflow` is set when the global list (capacity `cap`) is full; the
  // entries that did not fit are dropped.
  __device__ __forceinline__ void push(bool pred, const T& item, T* out, int* counter, long long cap, bool& overflow) {
    const int lane = threadIdx.x & 31;
    const unsigned bal = __ballot_sync(kFull, pred);
    if (pred) buf[count + __popc(bal & ((1u << lane) - 1))] = item;
    count += __popc(bal);
    if (count > kCap - 32) flush(out, counter, cap, overflow);
  }

  __device__ __forceinline__ void flush(T* out, int* counter, long long cap, bool& overflow) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    if (count == 0) return;
    int base = 0;
    if (lane == 0) base = fetch_add(counter, count);
    base = __shfl_sync(kFull, base, 0);
    for (int i = lane; i < count; i += 32) {
      if ((long long)base + i < cap) {
        if (kStream)
          __stcs(&out[base + i], buf[i]);
        else
          out[base + i] = buf[i];
      } else
        overflow = true;
    }
    __syncwarp();
    count = 0;
  }
};

}  // namespace dev
}  // namespace ecl
