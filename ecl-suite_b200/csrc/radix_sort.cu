// Stable LSD radix sort of (uint64 key, int32 value) pairs: see radix_sort.cuh.
#include "radix_sort.cuh"
#include "runtime.cuh"

namespace ecl {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kWarpSlice = kRadixTile / kWarps;  // 512 consecutive keys per warp

__device__ __forceinline__ unsigned digit_of(unsigned long long k, int shift) { return (unsigned)(k >> shift) & 0xffu; }

// Element count of this sort: n_max, or the device-side count when one is
// given (clamped to n_max, the size the launches were made for).
__device__ __forceinline__ int sort_count(int n_max, const int* n_dev) {
  if (!n_dev) return n_max;
  const int c = *n_dev;
  return c < 0 ? 0 : (c > n_max ? n_max : c);
}

// counts[d * tiles + t] = number of keys of tile t with digit d.
__global__ void __launch_bounds__(kThreads) rs_histogram(const unsigned long long* __restrict__ keys, int n_max,
                                                         const int* __restrict__ n_dev, int shift,
                                                         unsigned* __restrict__ counts, int tiles) {
  const int n = sort_count(n_max, n_dev);
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int t = blockIdx.x;
  const int base = t * kRadixTile;
  for (int i = threadIdx.x; i < kRadixTile; i += kThreads) {
    const int idx = base + i;
    if (idx < n) atomicAdd(&h[digit_of(keys[idx], shift)], 1u);
  }
  __syncthreads();
  counts[(size_t)threadIdx.x * tiles + t] = h[threadIdx.x];
}

// Exclusive scan of each digit's row counts[d * tiles .. (d+1) * tiles) in
// place (one block per digit); rowsum[d] = the row's total.
__global__ void __launch_bounds__(1024) rs_scan_rows(unsigned* __restrict__ counts, int tiles,
                                                    unsigned* __restrict__ rowsum) {
  __shared__ unsigned part[1024];
  unsigned* row = counts + (size_t)blockIdx.x * tiles;
  const int per = (tiles + 1023) / 1024;
  const int b = threadIdx.x * per;
  const int e = min(tiles, b + per);
  unsigned s = 0;
  for (int i = b; i < e; i++) s += row[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const unsigned add = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  unsigned run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
  for (int i = b; i < e; i++) {
    const unsigned c = row[i];
    row[i] = run;
    run += c;
  }
  if (threadIdx.x == 1023) rowsum[blockIdx.x] = part[1023];
}

// Exclusive scan of the 256 row totals in place: the base of each digit.
__global__ void __launch_bounds__(256) rs_scan_digits(unsigned* __restrict__ rowsum) {
  __shared__ unsigned part[256];
  part[threadIdx.x] = rowsum[threadIdx.x];
  __syncthreads();
  for (int off = 1; off < 256; off <<= 1) {
    const unsigned add = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  rowsum[threadIdx.x] = threadIdx.x ? part[threadIdx.x - 1] : 0u;
}

__global__ void __launch_bounds__(kThreads) rs_scatter(const unsigned long long* __restrict__ kin,
                                                       const int* __restrict__ vin, unsigned long long* __restrict__ kout,
                                                       int* __restrict__ vout, int n_max, const int* __restrict__ n_dev,
                                                       int shift, const unsigned* __restrict__ offsets,
                                                       const unsigned* __restrict__ digitbase, int tiles) {
  __shared__ unsigned wcount[kWarps][256];  // per-warp digit counts, then per-warp bases
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = blockIdx.x;
  const int n = sort_count(n_max, n_dev);
  if (t * kRadixTile >= n) return;  // a tile past the device-side count: nothing to place
  const int wbase = t * kRadixTile + warp * kWarpSlice;
  for (int d = lane; d < 256; d += 32) wcount[warp][d] = 0;
  __syncwarp();
  // 1. per-warp histogram of its slice
  for (int j = 0; j < kWarpSlice; j += 32) {
    const int idx = wbase + j + lane;
    if (idx < n) atomicAdd(&wcount[warp][digit_of(kin[idx], shift)], 1u);
  }
  __syncthreads();
  // 2. base of each (warp, digit) = tile offset + counts of earlier warps
  {
    const int d = threadIdx.x;  // 256 threads, one digit each
    unsigned run = digitbase[d] + offsets[(size_t)d * tiles + t];
    for (int w = 0; w < kWarps; w++) {
      const unsigned c = wcount[w][d];
      wcount[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
  // 3. stable scatter, 32 keys at a time in input order
  for (int j = 0; j < kWarpSlice; j += 32) {
    const int idx = wbase + j + lane;
    const bool ok = idx < n;
    unsigned long long k = 0;
    int v = 0;
    unsigned d = 0x100u + lane;  // unique sentinel for idle lanes
    if (ok) {
      k = kin[idx];
      v = vin[idx];
      d = digit_of(k, shift);
    }
    const unsigned same = __match_any_sync(0xffffffffu, d);
    const int before = __popc(same & ((1u << lane) - 1));
    const int leader = __ffs(same) - 1;
    unsigned pos = 0;
    if (ok) pos = wcount[warp][d] + before;
    __syncwarp();
    if (ok && lane == leader) wcount[warp][d] += __popc(same);
    __syncwarp();
    if (ok) {
      kout[pos] = k;
      vout[pos] = v;
    }
  }
}

}  // namespace

bool radix_sort_pairs(unsigned long long* k0, int* v0, unsigned long long* k1, int* v1, int n, int begin_bit,
                      int end_bit, unsigned* temp, cudaStream_t stream, const int* n_dev) {
  const int tiles = (int)radix_tiles((size_t)n);
  bool flip = false;
  for (int shift = begin_bit; shift < end_bit; shift += 8) {
    const unsigned long long* ki = flip ? k1 : k0;
    const int* vi = flip ? v1 : v0;
    unsigned long long* ko = flip ? k0 : k1;
    int* vo = flip ? v0 : v1;
    unsigned* digitbase = temp + (size_t)256 * tiles;
    ECL_LAUNCH(rs_histogram, tiles, kThreads, 0, stream, ki, n, n_dev, shift, temp, tiles);
    ECL_LAUNCH(rs_scan_rows, 256, 1024, 0, stream, temp, tiles, digitbase);
    ECL_LAUNCH(rs_scan_digits, 1, 256, 0, stream, digitbase);
    ECL_LAUNCH(rs_scatter, tiles, kThreads, 0, stream, ki, vi, ko, vo, n, n_dev, shift, temp, digitbase, tiles);
    flip = !flip;
  }
  return flip;
}

}  // namespace ecl
