// Drop-in for the reference's ECL-CC executable (RF/egr-input/CC/ECL-CC-atomic.cu:338-400).
#include <set>

#include "cli_common.h"

int main(int argc, char** argv) {
  printf("ECL-CC (B200, race-free)\n");
  ecl_graph g = load_graph(argc, argv);
  printf("input graph: %d nodes and %d edges (%s)\n", g.nodes, g.edges, argv[1]);
  printf("average degree: %.2f edges per node\n", 1.0 * g.edges / g.nodes);
  int mindeg, maxdeg;
  degree_stats(g, &mindeg, &maxdeg);
  printf("minimum degree: %d edges\n", mindeg);
  printf("maximum degree: %d edges\n", maxdeg);
  std::vector<int> label((size_t)g.nodes);
  ecl_graph_view v = host_view(g, false);
  ecl_opts o = {};
  const ecl_status st = ecl_cc(&v, label.data(), &o);
  if (st != ECL_OK) die("ecl_cc", st);
  const double runtime = o.elapsed_ms * 1e-3;
  printf("compute time: %.9f s\n", runtime);
  printf("throughput: %.3f Mnodes/s\n", g.nodes * 0.000001 / runtime);
  printf("throughput: %.3f Medges/s\n", g.edges * 0.000001 / runtime);
  std::set<int> ids(label.begin(), label.end());
  printf("number of connected components: %lu\n", (unsigned long)ids.size());
  // self-check as the reference's (ECL-CC-atomic.cu:373-393), iteratively
  for (int u = 0; u < g.nodes; u++) {
    if (label[u] < 0) {
      fprintf(stderr, "ERROR: found negative component number\n\n");
      return -1;
    }
    for (int i = g.nindex[u]; i < g.nindex[u + 1]; i++)
      if (label[g.nlist[i]] != label[u]) {
        fprintf(stderr, "ERROR: found adjacent nodes in different components\n\n");
        return -1;
      }
  }
  std::vector<char> seen((size_t)g.nodes, 0);
  std::vector<int> stack;
  size_t pieces = 0;
  for (int s = 0; s < g.nodes; s++) {
    if (seen[s]) continue;
    pieces++;
    seen[s] = 1;
    stack.push_back(s);
    while (!stack.empty()) {
      const int u = stack.back();
      stack.pop_back();
      if (label[u] != label[s]) {
        fprintf(stderr, "ERROR: found incorrect ID value\n\n");
        return -1;
      }
      for (int i = g.nindex[u]; i < g.nindex[u + 1]; i++)
        if (!seen[g.nlist[i]]) {
          seen[g.nlist[i]] = 1;
          stack.push_back(g.nlist[i]);
        }
    }
  }
  if (pieces != ids.size()) {
    fprintf(stderr, "ERROR: component IDs are not unique\n\n");
    return -1;
  }
  printf("verification passed\n\n");
  ecl_graph_free(&g);
  return 0;
}
