// Stable LSD radix sort of (uint64 key, int32 value) pairs, 8-bit digits.
//
// One pass = four launches: per-tile digit histograms, a per-digit-row scan
// of the digit-major histogram table, a scan of the 256 row totals, and a
// stable scatter.  The scatter
// ranks keys inside a tile warp by warp (warp w of a tile takes the w-th
// slice of it): __match_any_sync groups the lanes holding the same digit, a
// shared-memory table gives every warp its base per digit, so equal digits
// keep their input order and the sort is stable.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ecl {

struct RadixSortTemp {
  unsigned* counts;  // 256 * tiles
  size_t tiles;
};

// Elements per tile (block of 256 threads x 16 items).
constexpr int kRadixTile = 4096;

inline size_t radix_tiles(size_t n) { return (n + kRadixTile - 1) / kRadixTile; }
inline size_t radix_temp_words(size_t n) { return 256 * radix_tiles(n) + 256; }

// Sorts keys[0..n) ascending by bits [begin_bit, end_bit) together with vals.
// Ping-pongs between (k0, v0) and (k1, v1); returns true when the result is
// in (k1, v1).  Launches are counted and stream-ordered on `stream`.  With
// n_dev, the element count is read on the device when the sort runs (at most
// n, which sizes the launches and the temp buffer), so a count produced by an
// earlier kernel needs no host round trip.
bool radix_sort_pairs(unsigned long long* k0, int* v0, unsigned long long* k1, int* v1, int n, int begin_bit,
                      int end_bit, unsigned* temp, cudaStream_t stream, const int* n_dev = nullptr);

}  // namespace ecl
