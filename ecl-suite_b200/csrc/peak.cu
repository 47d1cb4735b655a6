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
