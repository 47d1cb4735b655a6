// Shared helpers of the command-line drop-ins: each tool takes the
// reference executable's arguments (one .egr file) and prints the reference's
// stdout key lines (e.g. "compute time: X s", ECL-CC-atomic.cu:314-316), so
// the reference's harness (scripts/analyze_results.py:61-63) parses them
// unchanged.  Times are the library's device time of the compute phase
// (opts.elapsed_ms), the region the reference times with cudaEvents.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ecl_b200.h"

inline void die(const char* what, ecl_status st) {
  fprintf(stderr, "ERROR: %s: %s %s\n\n", what, ecl_status_string(st), ecl_last_error());
  exit(-1);
}

inline ecl_graph load_graph(int argc, char** argv) {
  if (argc != 2) {
    fprintf(stderr, "USAGE: %s input_file_name\n\n", argv[0]);
    exit(-1);
  }
  ecl_graph g;
  const ecl_status st = ecl_graph_read(argv[1], &g);
  if (st != ECL_OK) die("could not read graph", st);
  return g;
}

inline ecl_graph_view host_view(const ecl_graph& g, bool weights) {
  ecl_graph_view v{g.nodes, g.edges, g.nindex, g.nlist, weights ? g.eweight : nullptr, ECL_HOST, 0};
  return v;
}

inline void degree_stats(const ecl_graph& g, int* mindeg, int* maxdeg) {
  *mindeg = g.nodes;
  *maxdeg = 0;
  for (int v = 0; v < g.nodes; v++) {
    const int d = g.nindex[v + 1] - g.nindex[v];
    if (d < *mindeg) *mindeg = d;
    if (d > *maxdeg) *maxdeg = d;
  }
}
