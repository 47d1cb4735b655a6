// Drop-in for the reference's ECL-GC executable (RF/egr-input/GC/ECL-GC-atomic.cu:316-403).
#include <algorithm>

#include "cli_common.h"

int main(int argc, char** argv) {
  printf("ECL-GC (B200, race-free)\n\n");
  ecl_graph g = load_graph(argc, argv);
  printf("input: %s\n", argv[1]);
  printf("nodes: %d\n", g.nodes);
  printf("edges: %d\n", g.edges);
  printf("avg degree: %.2f\n", 1.0 * g.edges / g.nodes);
  std::vector<int> color((size_t)g.nodes);
  ecl_graph_view v = host_view(g, false);
  ecl_opts o = {};
  const ecl_status st = ecl_gc(&v, color.data(), &o);
  if (st != ECL_OK) die("ecl_gc", st);
  const double runtime = o.elapsed_ms * 1e-3;
  printf("runtime:    %.9f s\n", runtime);
  printf("throughput: %.6f Mnodes/s\n", g.nodes * 0.000001 / runtime);
  printf("throughput: %.6f Medges/s\n", g.edges * 0.000001 / runtime);
  for (int u = 0; u < g.nodes; u++) {  // ECL-GC-atomic.cu:375-381
    if (color[u] < 0) {
      printf("ERROR: found unprocessed node in graph (node %d)\n\n", u);
      return -1;
    }
    for (int i = g.nindex[u]; i < g.nindex[u + 1]; i++)
      if (g.nlist[i] != u && color[g.nlist[i]] == color[u]) {
        printf("ERROR: found adjacent nodes with same color %d (%d %d)\n\n", color[u], u, g.nlist[i]);
        return -1;
      }
  }
  printf("result verification passed\n");
  const int vals = 16;
  int c[vals] = {0};
  int cols = -1;
  for (int u = 0; u < g.nodes; u++) {
    cols = std::max(cols, color[u]);
    if (color[u] < vals) c[color[u]]++;
  }
  cols++;
  printf("colors used: %d\n", cols);
  int sum = 0;
  for (int i = 0; i < std::min(vals, cols); i++) {
    sum += c[i];
    printf("col %2d: %10d (%5.1f%%)\n", i, c[i], 100.0 * sum / g.nodes);
  }
  ecl_graph_free(&g);
  return 0;
}
