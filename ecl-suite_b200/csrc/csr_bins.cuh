// Degree binning shared by the CSR scans.
//
// A row of <= kBinLane entries is walked by its own lane, all lanes of the
// warp stepping through entry offset k together (so warp-aggregated appends
// stay converged); a row of <= kBinChunk entries by the whole warp, 32
// entries per step; a longer row is cut into kBinChunk-entry chunk records
// that a second launch spreads over all warps.  R-MAT puts its heaviest rows
// at the lowest ids, i.e. in the same warp groups, so the chunk size -- not
// the lane/warp split -- bounds the work of the slowest warp.
#pragma once

#include "common.cuh"
#include "ecl_b200.h"

namespace ecl {
namespace dev {

constexpr int kBinLane = 32;
constexpr int kBinChunk = 256;

struct RowChunks {
  int2* rec;   // (vertex, first entry of the chunk)
  int* count;  // number of records
};

inline size_t row_chunk_capacity(int m) { return 2 * (size_t)(m / kBinChunk) + 2; }

// Row [beg, end) of v; a malformed row reports ECL_ERR_BAD_GRAPH and is empty.
__device__ __forceinline__ void csr_row(const int* nindex, int v, int m, int& beg, int& end, Status* status) {
  beg = __ldg(&nindex[v]);
  end = __ldg(&nindex[v + 1]);
  if (beg < 0 || end < beg || end > m) {
    raise(status, ECL_ERR_BAD_GRAPH, v);
    beg = end = 0;
  }
}

// Called by the lane that owns a long row.
__device__ __forceinline__ void push_row_chunks(RowChunks rc, int v, int beg, int end) {
  const int nc = (end - beg + kBinChunk - 1) / kBinChunk;
  const int at = fetch_add(rc.count, nc);
  for (int c = 0; c < nc; c++) rc.rec[at + c] = make_int2(v, beg + c * kBinChunk);
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

}  // namespace dev
}  // namespace ecl
