// Library-level C ABI entry points that are not tied to one solver.
#include "runtime.cuh"

namespace ecl {
size_t cc_workspace_bytes(int n, int m);
size_t mis_workspace_bytes(int n, int m);
size_t gc_workspace_bytes(int n, int m);
size_t mst_workspace_bytes(int n, int m);
size_t scc_workspace_bytes(int n, int m);
size_t apsp_workspace_bytes(int n, int m);
}  // namespace ecl

extern "C" size_t ecl_workspace_bytes(ecl_code code, int32_t nodes, int32_t edges) {
  using namespace ecl;
  if (nodes < 1 || edges < 0) return 0;
  size_t b = 0;
  switch (code) {
    case ECL_CC: b = cc_workspace_bytes(nodes, edges); break;
    case ECL_MIS: b = mis_workspace_bytes(nodes, edges); break;
    case ECL_GC: b = gc_workspace_bytes(nodes, edges); break;
    case ECL_MST: b = mst_workspace_bytes(nodes, edges); break;
    case ECL_SCC: b = scc_workspace_bytes(nodes, edges); break;
    case ECL_APSP: b = apsp_workspace_bytes(nodes, edges); break;
    default: return 0;
  }
  return b + kStatusBytes;
}
