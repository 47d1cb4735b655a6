// Launch-only ("enqueue") forms of the solvers.
//
// Each X_enqueue puts the whole solve onto `stream` -- memsets and kernel
// launches only: no allocation, no host synchronisation, no host read-back --
// so a sequence of them can be captured into a CUDA graph (batched engine)
// or run concurrently on several streams (server).  The caller provides a
// workspace of X_workspace_bytes() and a zeroed-or-not Status block (each
// enqueue clears what it needs).  The public ecl_X entry points are these
// plus staging and the status read-back.
#pragma once

#include "runtime.cuh"

namespace ecl {

struct GraphDev {
  int n = 0, m = 0;
  const int* nindex = nullptr;
  const int* nlist = nullptr;
  const int* eweight = nullptr;
  int flags = 0;
};

// A disjoint union of graphs (batched engine): graph g owns vertices
// [vbase[g], vbase[g+1]); avg[g] = (float)edges_g / nodes_g, the value the
// MIS priority of that graph uses.
struct UnionInfo {
  int ngraphs = 0;
  const int* vbase = nullptr;
  const float* avg = nullptr;
};

// Optional phase marks (Solve::mark) between kernel phases.
struct Marker {
  Solve* s = nullptr;
  void operator()() const {
    if (s) s->mark();
  }
};

size_t cc_workspace_bytes(int n, int m);
size_t mis_workspace_bytes(int n, int m);
size_t gc_workspace_bytes(int n, int m);
size_t mst_workspace_bytes(int n, int m);
size_t scc_workspace_bytes(int n, int m);

ecl_status cc_enqueue(const GraphDev& g, int* label, char* ws, dev::Status* status, const DeviceInfo& dev,
                      cudaStream_t stream, Marker mark = {});
ecl_status mis_enqueue(const GraphDev& g, unsigned char* out, char* ws, dev::Status* status, const DeviceInfo& dev,
                       cudaStream_t stream, int max_sweeps, const UnionInfo* uni = nullptr, Marker mark = {});
ecl_status gc_enqueue(const GraphDev& g, int* color, char* ws, dev::Status* status, const DeviceInfo& dev,
                      cudaStream_t stream, const UnionInfo* uni = nullptr, Marker mark = {});
// *total_dev receives the device address of the forest weight (uint64).
ecl_status mst_enqueue(const GraphDev& g, unsigned char* in_mst, char* ws, dev::Status* status, const DeviceInfo& dev,
                       cudaStream_t stream, unsigned long long** total_dev, Marker mark = {});
ecl_status scc_enqueue(const GraphDev& g, int* label, char* ws, dev::Status* status, const DeviceInfo& dev,
                       cudaStream_t stream, int max_rounds, Marker mark = {});

}  // namespace ecl
