// Drop-in for the reference's ECL-APSP executable (RF/grid-input/ECL-APSP-atomic.cu:572-624).
#include <algorithm>

#include "cli_common.h"

int main(int argc, char** argv) {
  printf("ECL-APSP (B200)\n");
  ecl_graph g = load_graph(argc, argv);
  printf("input: %s\n", argv[1]);
  printf("nodes: %d\n", g.nodes);
  printf("edges: %d\n", g.edges);
  if (!g.eweight) {
    fprintf(stderr, "ERROR: input graph has no edge weights\n\n");
    return -1;
  }
  for (int j = 0; j < g.edges; j++)  // as the reference does (:586-590)
    if (g.eweight[j] < 0) g.eweight[j] = -g.eweight[j];
  std::vector<int32_t> dist((size_t)g.nodes * g.nodes);
  ecl_graph_view v = host_view(g, true);
  ecl_opts o = {};
  o.detail = 1;
  const ecl_status st = ecl_apsp(&v, dist.data(), g.nodes, &o);
  if (st != ECL_OK) die("ecl_apsp", st);
  printf("FW_64 gpu init time: %10.6f s\n", (o.nphases > 0 ? o.phase_ms[0] : 0.f) * 1e-3);
  printf("FW_64 gpu comp time: %10.6f s\n", (o.nphases > 1 ? o.phase_ms[1] : o.elapsed_ms) * 1e-3);
  long reach = 0;
  for (size_t k = 0; k < dist.size(); k++) reach += dist[k] < ECL_APSP_INF;
  printf("reachable pairs: %ld\n", reach);
  ecl_graph_free(&g);
  return 0;
}
