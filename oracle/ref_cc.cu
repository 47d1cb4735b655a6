// Reference ECL-CC (race-free) compiled from its own source -- CHECKER / BASELINE ONLY.
#include "ref_common.h"
#define main ref_cc_main
#define readECLgraph ref_cc_readECLgraph
#define writeECLgraph ref_cc_writeECLgraph
#define freeECLgraph ref_cc_freeECLgraph
#define CheckCuda ref_cc_CheckCuda
#include "src/racefree/egr-input/CC/ECL-CC-atomic.cu"
#undef main

// The timed region of computeCC (ECL-CC-atomic.cu:298-312) on device-resident
// buffers: the reference's five kernels with its launch configuration.
// Returns the elapsed milliseconds; nstat receives the labels.
extern "C" float eclref_cc_device(int nodes, const int* nidx_d, const int* nlist_d, int* nstat_d, int* wl_d) {
  cudaDeviceProp p;
  cudaGetDeviceProperties(&p, 0);
  cudaFuncSetCacheConfig(init, cudaFuncCachePreferL1);
  cudaFuncSetCacheConfig(compute1, cudaFuncCachePreferL1);
  cudaFuncSetCacheConfig(compute2, cudaFuncCachePreferL1);
  cudaFuncSetCacheConfig(compute3, cudaFuncCachePreferL1);
  cudaFuncSetCacheConfig(flatten, cudaFuncCachePreferL1);
  const int blocks = p.multiProcessorCount * p.maxThreadsPerMultiProcessor / ThreadsPerBlock;
  RefTimer t;
  init<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist_d, nstat_d);
  compute1<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist_d, nstat_d, wl_d);
  compute2<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist_d, nstat_d, wl_d);
  compute3<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist_d, nstat_d, wl_d);
  flatten<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist_d, nstat_d);
  return t.stop();
}

// The reference's own host entry (ECL-CC-atomic.cu:275): host in, host out.
extern "C" void eclref_compute_cc(int nodes, int edges, const int* nidx, const int* nlist, int* nstat) {
  computeCC(nodes, edges, nidx, nlist, nstat);
}
