// Reference ECL-SCC (race-free) compiled from its own source -- CHECKER / BASELINE ONLY.
#include "ref_common.h"
#define main ref_scc_main
#define readECLgraph ref_scc_readECLgraph
#define writeECLgraph ref_scc_writeECLgraph
#define freeECLgraph ref_scc_freeECLgraph
#define CheckCuda ref_scc_CheckCuda
#include "src/racefree/mesh-input/ECL-SCC_10-atomic.cu"
#undef main

// Bytes of scratch: iomax[nodes], wl1[edges], wl2[edges] (ull) plus two ints
// (the allocations of ECL-SCC_10-atomic.cu:254-258).
extern "C" size_t eclref_scc_scratch_bytes(int nodes, int edges) {
  return sizeof(ull) * ((size_t)nodes + 2 * (size_t)edges) + 2 * sizeof(int) + 16;
}

// The timed region of the SCC driver inlined in main
// (ECL-SCC_10-atomic.cu:274-299): the reference's kernels, launch
// configuration and host-driven fixpoint loops, on device buffers.  label_h
// (host) receives readFirst(iomax[v]) (:318).
extern "C" float eclref_scc_device(int nodes, int edges, const int* nidx_d, const int* nlist_d, int* label_h, void* scratch) {
  ull* d_iomax = (ull*)scratch;
  ull* d_wl1 = d_iomax + nodes;
  ull* d_wl2 = d_wl1 + edges;
  int* d_wl2size = (int*)(d_wl2 + edges);
  ibool* d_goagain = d_wl2size + 1;
  ECLgraph d_g;
  d_g.nodes = nodes;
  d_g.edges = edges;
  d_g.nindex = (int*)nidx_d;
  d_g.nlist = (int*)nlist_d;
  d_g.eweight = NULL;
  cudaDeviceProp p;
  cudaGetDeviceProperties(&p, 0);
  const int blocks = p.multiProcessorCount * (p.maxThreadsPerMultiProcessor / ThreadsPerBlock);
  RefTimer t;
  int wl1size;
  globalInit<<<blocks, ThreadsPerBlock>>>(d_g, d_wl1, d_wl2size, d_iomax);
  cudaMemcpy(&wl1size, d_wl2size, sizeof(int), cudaMemcpyDeviceToHost);
  ibool goagain;
  do {
    do {
      cudaMemsetAsync(d_goagain, 0, sizeof(ibool));
      propagateMax<<<blocks, ThreadsPerBlock>>>(d_wl1, wl1size, d_iomax, d_goagain);
      cudaMemcpy(&goagain, d_goagain, sizeof(ibool), cudaMemcpyDeviceToHost);
    } while (goagain);
    cudaMemsetAsync(d_wl2size, 0, sizeof(int));
    removeEdges<<<blocks, ThreadsPerBlock>>>(d_wl1, wl1size, d_wl2, d_wl2size, d_iomax);
    std::swap(d_wl1, d_wl2);
    cudaMemcpyAsync(&wl1size, d_wl2size, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemsetAsync(d_goagain, 0, sizeof(ibool));
    localInit<<<blocks, ThreadsPerBlock>>>(nodes, d_iomax, d_goagain);
    cudaMemcpy(&goagain, d_goagain, sizeof(ibool), cudaMemcpyDeviceToHost);
  } while (goagain);
  const float ms = t.stop();
  if (label_h) {
    ull* h = new ull[nodes];
    cudaMemcpy(h, d_iomax, sizeof(ull) * nodes, cudaMemcpyDeviceToHost);
    for (int v = 0; v < nodes; v++) label_h[v] = readFirst(h[v]);
    delete[] h;
  }
  return ms;
}
