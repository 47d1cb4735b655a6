// Reference ECL-GC (race-free) compiled from its own source -- CHECKER / BASELINE ONLY.
#include "ref_common.h"
#define main ref_gc_main
#define readECLgraph ref_gc_readECLgraph
#define writeECLgraph ref_gc_writeECLgraph
#define freeECLgraph ref_gc_freeECLgraph
#define CheckCuda ref_gc_CheckCuda
#include "src/racefree/egr-input/GC/ECL-GC-atomic.cu"
#undef main

// Bytes of scratch eclref_gc_device needs: nlist2[edges], posscol[nodes],
// posscol2[edges/32+1], wl[nodes] (the allocations of ECL-GC-atomic.cu:341-347).
extern "C" size_t eclref_gc_scratch_bytes(int nodes, int edges) {
  return sizeof(int) * ((size_t)edges + nodes + (edges / WS + 1) + nodes);
}

// The timed region of the GC driver in main (ECL-GC-atomic.cu:355-365): the
// reference's three kernels with its launch configuration.
extern "C" float eclref_gc_device(int nodes, int edges, const int* nidx_d, const int* nlist_d, int* color_d, int* scratch) {
  int* nlist2_d = scratch;
  int* posscol_d = nlist2_d + edges;
  int* posscol2_d = posscol_d + nodes;
  int* wl_d = posscol2_d + (edges / WS + 1);
  cudaDeviceProp p;
  cudaGetDeviceProperties(&p, 0);
  const int blocks = p.multiProcessorCount * p.maxThreadsPerMultiProcessor / ThreadsPerBlock;
  cudaFuncSetCacheConfig(init, cudaFuncCachePreferL1);
  cudaFuncSetCacheConfig(runLarge, cudaFuncCachePreferL1);
  cudaFuncSetCacheConfig(runSmall, cudaFuncCachePreferL1);
  RefTimer t;
  init<<<blocks, ThreadsPerBlock>>>(nodes, edges, nidx_d, nlist_d, nlist2_d, posscol_d, posscol2_d, color_d, wl_d);
  runLarge<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist2_d, posscol_d, posscol2_d, color_d, wl_d);
  runSmall<<<blocks, ThreadsPerBlock>>>(nodes, nidx_d, nlist_d, posscol_d, color_d);
  return t.stop();
}
