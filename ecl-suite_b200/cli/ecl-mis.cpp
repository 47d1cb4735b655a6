// Drop-in for the reference's ECL-MIS executable (RF/egr-input/MIS/ECL-MIS-atomic.cu:190-236).
#include "cli_common.h"

int main(int argc, char** argv) {
  printf("ECL-MIS (B200, race-free)\n");
  ecl_graph g = load_graph(argc, argv);
  printf("configuration: %d nodes and %d edges (%s)\n", g.nodes, g.edges, argv[1]);
  printf("average degree: %.2f edges per node\n", 1.0 * g.edges / g.nodes);
  std::vector<unsigned char> st8((size_t)g.nodes);
  ecl_graph_view v = host_view(g, false);
  ecl_opts o = {};
  const ecl_status st = ecl_mis(&v, st8.data(), &o);
  if (st != ECL_OK) die("ecl_mis", st);
  const double runtime = o.elapsed_ms * 1e-3;
  printf("compute time: %.9f s\n", runtime);
  printf("throughput: %.6f Mnodes/s\n", g.nodes * 0.000001 / runtime);
  printf("throughput: %.6f Medges/s\n", g.edges * 0.000001 / runtime);
  int count = 0;
  for (int u = 0; u < g.nodes; u++) count += st8[u] == ECL_MIS_IN;
  printf("elements in set: %d (%.1f%%)\n", count, 100.0 * count / g.nodes);
  for (int u = 0; u < g.nodes; u++) {  // ECL-MIS-atomic.cu:216-231
    if (st8[u] != ECL_MIS_IN && st8[u] != ECL_MIS_OUT) {
      fprintf(stderr, "ERROR: found unprocessed node in graph\n\n");
      return -1;
    }
    bool any_in = false;
    for (int i = g.nindex[u]; i < g.nindex[u + 1]; i++) any_in |= st8[g.nlist[i]] == ECL_MIS_IN;
    if (st8[u] == ECL_MIS_IN && any_in) {
      fprintf(stderr, "ERROR: found adjacent nodes in MIS\n\n");
      return -1;
    }
    if (st8[u] == ECL_MIS_OUT && !any_in) {
      fprintf(stderr, "ERROR: set is not maximal\n\n");
      return -1;
    }
  }
  ecl_graph_free(&g);
  return 0;
}
