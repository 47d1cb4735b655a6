// Writes the seeded synthetic inputs as .egr files:
//   egr-gen rmat SCALE EDGE_FACTOR SEED SYM WEIGHT_SEED out.egr
//   egr-gen grid ROWS COLS DELETE_FRAC SEED WEIGHT_SEED out.egr
//   egr-gen er N P SEED SYM WEIGHT_SEED out.egr
#include <cstring>

#include "cli_common.h"

int main(int argc, char** argv) {
  ecl_graph g{};
  ecl_status st = ECL_ERR_INVALID_ARG;
  const char* path = argv[argc - 1];
  if (argc == 8 && !strcmp(argv[1], "rmat")) {
    st = ecl_gen_rmat(atoi(argv[2]), atoi(argv[3]), 0.57, 0.19, 0.19, strtoull(argv[4], 0, 10), atoi(argv[5]),
                      strtoull(argv[6], 0, 10), 1 << 20, &g);
  } else if (argc == 8 && !strcmp(argv[1], "grid")) {
    st = ecl_gen_grid(atoi(argv[2]), atoi(argv[3]), atof(argv[4]), strtoull(argv[5], 0, 10), strtoull(argv[6], 0, 10),
                      1 << 20, &g);
  } else if (argc == 8 && !strcmp(argv[1], "er")) {
    st = ecl_gen_er(atoi(argv[2]), atof(argv[3]), strtoull(argv[4], 0, 10), atoi(argv[5]), strtoull(argv[6], 0, 10), 1,
                    1000, &g);
  } else {
    fprintf(stderr, "USAGE: %s rmat|grid|er ... out.egr\n", argv[0]);
    return -1;
  }
  if (st != ECL_OK) die("generator", st);
  st = ecl_graph_write(path, &g);
  if (st != ECL_OK) die("write", st);
  printf("%s: %d nodes, %d edges%s\n", path, g.nodes, g.edges, g.eweight ? ", weighted" : "");
  ecl_graph_free(&g);
  return 0;
}
