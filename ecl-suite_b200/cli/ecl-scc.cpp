// Drop-in for the reference's ECL-SCC executable (RF/mesh-input/ECL-SCC_10-atomic.cu:227-343).
#include <algorithm>
#include <functional>

#include "cli_common.h"

int main(int argc, char** argv) {
  printf("ECL-SCC (B200, race-free)\n\n");
  ecl_graph g = load_graph(argc, argv);
  printf("input: %s\n", argv[1]);
  printf("nodes: %d\n", g.nodes);
  printf("edges: %d\n", g.edges);
  printf("avg degree: %.2f\n\n", 1.0 * g.edges / g.nodes);
  std::vector<int> label((size_t)g.nodes);
  ecl_graph_view v = host_view(g, false);
  ecl_opts o = {};
  const ecl_status st = ecl_scc(&v, label.data(), &o);
  if (st != ECL_OK) die("ecl_scc", st);
  printf("compute time: %.9f s\n\n", o.elapsed_ms * 1e-3);
  // SCC sizes and frequency, as the reference prints them (:315-335)
  printf("result:\n");
  const int n = g.nodes;
  std::vector<int> count((size_t)n, 0);
  for (int u = 0; u < n; u++) count[label[u]]++;
  std::sort(count.begin(), count.end(), std::greater<int>());
  int cnt = 1, scc_cnt = 0;
  for (int u = 1; u < n; u++) {
    if (count[u] != count[u - 1]) {
      printf("%d SCCs of size %d\n", cnt, count[u - 1]);
      scc_cnt += cnt;
      cnt = 1;
    } else {
      cnt++;
    }
  }
  if (count[n - 1] > 0) {
    printf("%d SCCs of size %d\n", cnt, count[n - 1]);
    scc_cnt += cnt;
  }
  printf("number of SCCs: %d\n", scc_cnt);
  ecl_graph_free(&g);
  return 0;
}
