// INT32 min-plus throughput probe: the roofline denominator of the APSP
// kernels (the measured HBM copy bandwidth covers the other codes; no
// integer-pipe peak is published for B200).
//
// Every thread keeps an 8 x 8 accumulator tile like the APSP tile product and
// updates it as acc[r][c] = min(acc[r][c] + b[c], a[r]) -- each update reads
// its own previous value, so nothing folds or hoists out of the loop, and the
// 64 chains give every warp enough independent work to fill the pipe.  One
// update counts as 2 integer operations (one add, one min), the same count the
// APSP roofline uses.  Variant 0 issues the DPX __viaddmin_s32 (the
// instruction the APSP kernels use); variant 1 writes the add and the min as
// two separate operations.
#include "runtime.cuh"

namespace ecl {
namespace {

constexpr int kPeakThreads = 256;

template <int V>
__global__ void __launch_bounds__(kPeakThreads) minplus_peak_kernel(int iters, int seed, int* __restrict__ sink) {
  int a[8], b[8], acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    a[i] = (threadIdx.x * 7 + i * 131 + seed) & 0xffff;
    b[i] = ((blockIdx.x + seed) * 3 + i * 17) & 0xff;
  }
#pragma unroll
  for (int r = 0; r < 8; r++)
#pragma unroll
    for (int c = 0; c < 8; c++) acc[r][c] = a[r] ^ b[c];
#pragma unroll 1
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
      for (int c = 0; c < 8; c++) {
        if (V == 0)
          acc[r][c] = __viaddmin_s32(acc[r][c], b[c], a[r]);
        else
          acc[r][c] = min(acc[r][c] + b[c], a[r]);
      }
  }
  int x = 0;
#pragma unroll
  for (int r = 0; r < 8; r++)
#pragma unroll
    for (int c = 0; c < 8; c++) x ^= acc[r][c];
  sink[blockIdx.x * kPeakThreads + threadIdx.x] = x;
}

}  // namespace
}  // namespace ecl

using namespace ecl;

extern "C" ecl_status ecl_minplus_peak(int32_t variant, double* ops_per_s) {
  if (!ops_per_s || (variant != 0 && variant != 1)) {
    set_last_error_msg("ecl_minplus_peak: variant must be 0 or 1 and ops_per_s non-null");
    return ECL_ERR_INVALID_ARG;
  }
  *ops_per_s = 0.0;
  DeviceInfo di;
  const ecl_status st = current_device(&di);
  if (st != ECL_OK) return st;
  // One full wave: every SM holds as many blocks as its registers allow.
  int per_sm = 0;
  ECL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, variant == 0 ? minplus_peak_kernel<0> : minplus_peak_kernel<1>, kPeakThreads, 0));
  const int blocks = di.sms * (per_sm > 0 ? per_sm : 1);
  const int iters = 1 << 14;
  int* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ECL_CUDA_TRY(cudaMalloc(&sink, sizeof(int) * (size_t)blocks * kPeakThreads));
  float best_ms = 0.0f;
  cudaError_t err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  for (int rep = 0; rep < 4 && err == cudaSuccess; rep++) {  // rep 0 warms up
    cudaEventRecord(e0, 0);
    if (variant == 0)
      ECL_LAUNCH(minplus_peak_kernel<0>, blocks, kPeakThreads, 0, 0, iters, rep, sink);
    else
      ECL_LAUNCH(minplus_peak_kernel<1>, blocks, kPeakThreads, 0, 0, iters, rep, sink);
    cudaEventRecord(e1, 0);
    err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) {
    set_last_error("ecl_minplus_peak", err);
    return ECL_ERR_CUDA;
  }
  const double updates = (double)blocks * kPeakThreads * 64.0 * iters;
  *ops_per_s = 2.0 * updates / (best_ms * 1e-3);
  return ECL_OK;
}

// ---- streaming gather rate ------------------------------------------------------
//
// The roofline of the CSR scans: every scan streams the 4-byte column indices
// once and, per entry, loads one word of a per-vertex array that stays in L2
// (GC's keys, MST's roots, SCC's flags).  This probe does exactly that and
// nothing else -- each index (read once, coalesced, evict-first) selects one
// 8-byte word of an n-word table, kGatherBatch entries in flight per lane --
// so the rate it reaches on a graph's own index array bounds any scan of that
// graph.  Variant 0 loads the words through the read-only path (__ldg, as
// GC's keys are read), variant 1 with relaxed device-scope atomic loads (as
// MST's roots and SCC's flags are).
namespace ecl {
namespace {

constexpr int kGatherBatch = 4;

template <bool kCoherent>
__global__ void __launch_bounds__(kPeakThreads) gather_kernel(const int* __restrict__ idx, int m,
                                                             const unsigned long long* __restrict__ table, int n,
                                                             unsigned long long* __restrict__ sink) {
  const int tid = blockIdx.x * kPeakThreads + threadIdx.x;
  const int nthreads = gridDim.x * kPeakThreads;
  unsigned long long acc = 0;
  for (long long j0 = tid; j0 < m; j0 += (long long)nthreads * kGatherBatch) {
    int u[kGatherBatch];
#pragma unroll
    for (int k = 0; k < kGatherBatch; k++) {
      const long long j = j0 + (long long)k * nthreads;
      u[k] = j < m ? __ldcs(&idx[j]) : -1;
    }
#pragma unroll
    for (int k = 0; k < kGatherBatch; k++)
      if ((unsigned)u[k] < (unsigned)n) acc += kCoherent ? dev::ld(&table[u[k]]) : __ldg(&table[u[k]]);
  }
  sink[tid] = acc;  // thread-owned: keeps every load live
}

}  // namespace
}  // namespace ecl

extern "C" ecl_status ecl_gather_peak(const int32_t* d_index, int32_t m, int32_t n, int32_t variant,
                                      double* entries_per_s) {
  using namespace ecl;
  if (!entries_per_s || !d_index || m <= 0 || n <= 0 || (variant != 0 && variant != 1)) {
    set_last_error_msg("ecl_gather_peak: need a device index array, m > 0, n > 0, variant 0 or 1");
    return ECL_ERR_INVALID_ARG;
  }
  *entries_per_s = 0.0;
  DeviceInfo di;
  const ecl_status st = current_device(&di);
  if (st != ECL_OK) return st;
  int per_sm = 0;
  ECL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, variant == 0 ? gather_kernel<false> : gather_kernel<true>, kPeakThreads, 0));
  const int blocks = di.sms * (per_sm > 0 ? per_sm : 1);
  unsigned long long* table = nullptr;
  unsigned long long* sink = nullptr;
  char* flush = nullptr;
  const size_t flush_bytes = 256ull << 20;  // more than the 126 MB L2: every timed run starts cold
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t err = cudaMalloc(&table, sizeof(unsigned long long) * (size_t)n);
  if (err == cudaSuccess) err = cudaMalloc(&sink, sizeof(unsigned long long) * (size_t)blocks * kPeakThreads);
  if (err == cudaSuccess) err = cudaMalloc(&flush, flush_bytes);
  if (err == cudaSuccess) err = cudaMemset(table, 0x5a, sizeof(unsigned long long) * (size_t)n);
  if (err == cudaSuccess) err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  float best_ms = 0.0f;
  for (int rep = 0; rep < 4 && err == cudaSuccess; rep++) {  // rep 0 warms up
    // cold L2 for the index stream, then the table alone warmed into L2, as
    // a scan finds its per-vertex array after the kernels before it
    err = cudaMemsetAsync(flush, rep, flush_bytes, 0);
    if (err == cudaSuccess) err = cudaMemsetAsync(table, 0x5a, sizeof(unsigned long long) * (size_t)n, 0);
    if (err != cudaSuccess) break;
    cudaEventRecord(e0, 0);
    if (variant == 0)
      ECL_LAUNCH(gather_kernel<false>, blocks, kPeakThreads, 0, 0, d_index, m, table, n, sink);
    else
      ECL_LAUNCH(gather_kernel<true>, blocks, kPeakThreads, 0, 0, d_index, m, table, n, sink);
    cudaEventRecord(e1, 0);
    err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(table);
  cudaFree(sink);
  cudaFree(flush);
  if (err != cudaSuccess || best_ms <= 0.0f) {
    set_last_error("ecl_gather_peak", err);
    return ECL_ERR_CUDA;
  }
  *entries_per_s = (double)m / (best_ms * 1e-3);
  return ECL_OK;
}

// ---- dependency-hop latency ----------------------------------------------------
//
// One hop of a dependency chain: a warp stores a value another warp is
// polling for, and that warp's own next store follows.  Two warps ping-pong a
// counter `iters` times each way; one hop is the event-timed launch divided
// by the 2 * iters hops.  Variant 0: two CTAs on two SMs (one block per SM by
// their shared-memory size) through an L2 word, waiting the way GC's pull
// waits (relaxed device-scope loads, __nanosleep back-off from 32 to 512 ns).
// Variant 1: the same with a bare spin.  Variant 2: two warps of one CTA
// through a shared-memory word, waiting the way GC's core waits.  Every wait
// is bounded; a wait that runs out sets *failed and both sides stop.

namespace ecl {
namespace {

constexpr unsigned long long kHopWaitNs = 2000000000ull;  // a wait gives up after 2 s

__device__ __forceinline__ unsigned long long hop_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <int V>
__device__ __forceinline__ bool hop_wait(const unsigned* p, unsigned want, const unsigned* stop) {
  unsigned nap = 32;
  const unsigned long long t0 = hop_now();
  for (unsigned spins = 0;; spins++) {
    unsigned cur;
    if (V == 2)
      cur = cuda::atomic_ref<unsigned, cuda::thread_scope_block>(*const_cast<unsigned*>(p)).load(
          cuda::memory_order_relaxed);
    else
      cur = dev::ld(p);
    if (cur == want) return true;
    if ((spins & 255u) == 255u && (dev::ld(stop) != 0 || hop_now() - t0 > kHopWaitNs)) return false;
    if (V == 0) {
      __nanosleep(nap);
      nap = min(nap * 2, 512u);
    } else if (V == 2 && spins > 8) {
      __nanosleep(32);
    }
  }
}

template <int V>
__global__ void hop_kernel(unsigned* __restrict__ word, unsigned* __restrict__ failed, int iters) {
  __shared__ unsigned s_word;
  const int side = (V == 2) ? (int)(threadIdx.x >> 5) : (int)blockIdx.x;  // 0 or 1
  if (V == 2 && threadIdx.x == 0) s_word = 0;
  if (V == 2) __syncthreads();
  if ((threadIdx.x & 31) != 0) return;
  unsigned* p = (V == 2) ? &s_word : word;
  for (int i = 0; i < iters; i++) {
    const unsigned mine = 2u * (unsigned)i + (unsigned)side + 1u;  // side 0 writes odd, side 1 even values
    if (mine > 1 && !hop_wait<V>(p, mine - 1, failed)) {
      dev::st(failed, 1u);
      return;
    }
    if (V == 2)
      cuda::atomic_ref<unsigned, cuda::thread_scope_block>(*p).store(mine, cuda::memory_order_relaxed);
    else
      dev::st(p, mine);
  }
}

}  // namespace
}  // namespace ecl

extern "C" ecl_status ecl_hop_latency(int32_t variant, double* ns_per_hop) {
  if (!ns_per_hop || variant < 0 || variant > 2) {
    set_last_error_msg("ecl_hop_latency: variant must be 0, 1 or 2 and ns_per_hop non-null");
    return ECL_ERR_INVALID_ARG;
  }
  *ns_per_hop = 0.0;
  DeviceInfo di;
  const ecl_status st = current_device(&di);
  if (st != ECL_OK) return st;
  const int iters = 20000;
  unsigned* buf = nullptr;  // [0] the L2 word, [32] the failure flag (separate 128-byte lines)
  ECL_CUDA_TRY(cudaMalloc(&buf, 64 * sizeof(unsigned)));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  // more than half an SM's shared memory per block: the two blocks of the L2
  // variants cannot share an SM
  const size_t smem = di.smem_optin / 2 + 1024;
  if (err == cudaSuccess && variant != 2) {
    err = cudaFuncSetAttribute(variant == 0 ? hop_kernel<0> : hop_kernel<1>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  float best_ms = 0.f;
  unsigned failed = 0;
  for (int rep = 0; rep < 3 && err == cudaSuccess && !failed; rep++) {  // rep 0 warms up
    err = cudaMemset(buf, 0, 64 * sizeof(unsigned));
    if (err != cudaSuccess) break;
    cudaEventRecord(e0, 0);
    if (variant == 2) {
      ECL_LAUNCH(hop_kernel<2>, 1, 64, 0, 0, buf, buf + 32, iters);
    } else {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(2);
      cfg.blockDim = dim3(32);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeCooperative;  // both blocks resident at once
      attr[0].val.cooperative = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      err = variant == 0 ? cudaLaunchKernelEx(&cfg, hop_kernel<0>, buf, buf + 32, iters)
                         : cudaLaunchKernelEx(&cfg, hop_kernel<1>, buf, buf + 32, iters);
      count_launch();
      if (err != cudaSuccess) break;
    }
    cudaEventRecord(e1, 0);
    err = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (err == cudaSuccess) err = cudaMemcpy(&failed, buf + 32, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (rep > 0 && (best_ms == 0.f || ms < best_ms)) best_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  if (err != cudaSuccess) {
    set_last_error("ecl_hop_latency", err);
    return ECL_ERR_CUDA;
  }
  if (failed) {
    set_last_error_msg("ecl_hop_latency: a wait ran out of its bound");
    return ECL_ERR_NO_CONVERGENCE;
  }
  *ns_per_hop = best_ms * 1e6 / (2.0 * iters);
  return ECL_OK;
}
