// Reference ECL-MIS (race-free) compiled from its own source -- CHECKER / BASELINE ONLY.
#include "ref_common.h"
#define main ref_mis_main
#define readECLgraph ref_mis_readECLgraph
#define writeECLgraph ref_mis_writeECLgraph
#define freeECLgraph ref_mis_freeECLgraph
#define CheckCuda ref_mis_CheckCuda
#include "src/racefree/egr-input/MIS/ECL-MIS-atomic.cu"
#undef main

// The timed region of computeMIS (ECL-MIS-atomic.cu:170-176) on device
// buffers; nstat_d must hold (nodes + 3) / 4 * 4 bytes (:163).
extern "C" float eclref_mis_device(int nodes, int edges, const int* nidx_d, const int* nlist_d, unsigned char* nstat_d) {
  cudaDeviceProp p;
  cudaGetDeviceProperties(&p, 0);
  cudaFuncSetCacheConfig(init, cudaFuncCachePreferL1);
  cudaFuncSetCacheConfig(findmins, cudaFuncCachePreferL1);
  const int blocks = p.multiProcessorCount * p.maxThreadsPerMultiProcessor / ThreadsPerBlock;
  RefTimer t;
  init<<<blocks, ThreadsPerBlock>>>(nodes, edges, nidx_d, nstat_d);
  findmins<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist_d, nstat_d);
  return t.stop();
}
