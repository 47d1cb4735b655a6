// Solvers not yet implemented in this build step.
#include "runtime.cuh"
namespace ecl {
size_t mis_workspace_bytes(int, int) { return 0; }
size_t gc_workspace_bytes(int, int) { return 0; }
size_t mst_workspace_bytes(int, int) { return 0; }
size_t scc_workspace_bytes(int, int) { return 0; }
size_t apsp_workspace_bytes(int, int) { return 0; }
}
extern "C" {
ecl_status ecl_mis(const ecl_graph_view*, uint8_t*, ecl_opts*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_gc(const ecl_graph_view*, int32_t*, ecl_opts*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_mst(const ecl_graph_view*, uint8_t*, uint64_t*, ecl_opts*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_scc(const ecl_graph_view*, int32_t*, ecl_opts*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_apsp(const ecl_graph_view*, int32_t*, int64_t, ecl_opts*) { return ECL_ERR_UNSUPPORTED; }
}
extern "C" {
ecl_status ecl_compute_mis(int32_t, int32_t, const int32_t*, const int32_t*, uint8_t*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_compute_gc(int32_t, int32_t, const int32_t*, const int32_t*, int32_t*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_compute_mst(int32_t, int32_t, const int32_t*, const int32_t*, const int32_t*, uint8_t*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_compute_scc(int32_t, int32_t, const int32_t*, const int32_t*, int32_t*) { return ECL_ERR_UNSUPPORTED; }
ecl_status ecl_compute_apsp(int32_t, int32_t, const int32_t*, const int32_t*, const int32_t*, int32_t*) { return ECL_ERR_UNSUPPORTED; }
}
