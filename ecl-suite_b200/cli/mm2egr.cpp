// MatrixMarket -> .egr converter (the reference's scripts/mm2ecl_real.cpp
// contract, plus an optional --symmetrise).
#include <cstring>

#include "cli_common.h"

int main(int argc, char** argv) {
  printf("MatrixMarket to ECL Graph Converter (B200 suite)\n");
  const bool sym = argc == 4 && strcmp(argv[3], "--symmetrise") == 0;
  if (argc != 3 && !sym) {
    fprintf(stderr, "USAGE: %s input_file_name output_file_name [--symmetrise]\n\n", argv[0]);
    return -1;
  }
  ecl_graph g;
  ecl_status st = ecl_graph_from_mm(argv[1], sym ? 1 : 0, &g);
  if (st != ECL_OK) die("could not convert", st);
  printf("%s\t#name\n%d\t#nodes\n%d\t#edges\n%s\t#weights\n", argv[1], g.nodes, g.edges, g.eweight ? "yes" : "no");
  st = ecl_graph_write(argv[2], &g);
  if (st != ECL_OK) die("could not write", st);
  ecl_graph_free(&g);
  return 0;
}
