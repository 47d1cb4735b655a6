/*
 * ecl_batch.h -- batched engine: many graphs, one set of launches.
 *
 * No counterpart in the reference, whose every code solves one graph per
 * process (src/racefree/egr-input/*: main() -> one computeXX call).  Graphs
 * added to a batch are packed into "super-batches": each is the disjoint union
 * of consecutive graphs (vertex ids offset per graph, CSR concatenated, total
 * entries kept below 2^31 so the int32 kernels apply unchanged).  Every solve
 * then runs once per super-batch, not once per graph, and the whole run is
 * captured into one CUDA graph that later runs replay.  Results are per graph
 * and identical to solving each graph alone with ecl_cc / ecl_mis / ecl_mst /
 * ecl_gc / ecl_scc: none of the fixpoints crosses a graph boundary, ids keep
 * their relative order inside the union, and MIS/GC priorities use each
 * graph's own average degree and local ids.
 */
#ifndef ECL_BATCH_H
#define ECL_BATCH_H

#include "ecl_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ecl_batch ecl_batch;

/* Solver set (bit mask). */
#define ECL_BATCH_CC 0x1u
#define ECL_BATCH_MIS 0x2u
#define ECL_BATCH_GC 0x4u
#define ECL_BATCH_MST 0x8u
#define ECL_BATCH_SCC 0x10u

/* The engine's launch knobs are an ecl_tune (ecl_b200.h); ecl_batch_tune
 * chooses them for the built batch. */

ecl_status ecl_batch_create(ecl_batch** out);
void ecl_batch_destroy(ecl_batch* b);

/* Appends one host graph (copied).  Graphs keep the order they are added in. */
ecl_status ecl_batch_add(ecl_batch* b, const ecl_graph_view* g);

/* Appends `count` seeded synthetic graphs of the batched benchmark mix: vertex
 * counts log-uniform in [n_min, n_max], each drawn with equal probability from
 * Erdos-Renyi (average degree 8), a 4-neighbour grid, or R-MAT (edge factor
 * 8, a=.57 b=.19 c=.19), symmetric, weights uniform in [1, weight_max). */
ecl_status ecl_batch_add_mix(ecl_batch* b, int32_t count, int32_t n_min, int32_t n_max, uint64_t seed,
                             int32_t weight_max);

/* Packs the graphs into super-batches of at most max_entries CSR entries
 * (0 = 2^29), uploads them, and reserves outputs and workspaces for `codes`.
 * `stream` is synchronised first; the engine then works on a non-blocking
 * stream of its own (the legacy default stream cannot be captured), and
 * ecl_batch_run returns with its work finished. */
ecl_status ecl_batch_build(ecl_batch* b, uint32_t codes, int64_t max_entries, void* stream);

/* Solves every graph for every code given to ecl_batch_build.  The first run
 * captures the launch sequence into a CUDA graph; later runs replay it.
 * opts->elapsed_ms receives the device time of the run. */
ecl_status ecl_batch_run(ecl_batch* b, ecl_opts* opts);

/* The autotuner: coordinate descent over the launch knobs of ecl_tune on the
 * built batch (grid size, the per-lane / chunk row thresholds of the CSR
 * scans, the MST light-edge split and, with GC, GC's shared-memory core); each
 * setting costs one capturing run plus `trials` timed runs.  Keeps the
 * fastest, returns it in *best (may be NULL) and rebuilds the captured CUDA
 * graph.  Results never depend on the knobs. */
ecl_status ecl_batch_tune(ecl_batch* b, int32_t trials, ecl_tune* best);
ecl_status ecl_batch_set_tune(ecl_batch* b, const ecl_tune* t);
/* Number of knob settings the last ecl_batch_tune timed. */
int32_t ecl_batch_tune_points(const ecl_batch* b);

int32_t ecl_batch_graphs(const ecl_batch* b);
int32_t ecl_batch_superbatches(const ecl_batch* b);
/* Size of graph i (nodes, edges). */
ecl_status ecl_batch_graph_size(const ecl_batch* b, int32_t i, int32_t* nodes, int32_t* edges);
/* Copies graph i's CSR back to host arrays (nindex[nodes+1], nlist[edges],
 * eweight[edges] or NULL) -- for checking results against a solo solve. */
ecl_status ecl_batch_graph_csr(const ecl_batch* b, int32_t i, int32_t* nindex, int32_t* nlist, int32_t* eweight);

/* Result of graph i for one code, in that code's single-graph layout:
 * CC / SCC int32 label[nodes] (local ids), MIS uint8 status[nodes], GC int32
 * color[nodes], MST uint8 in_mst[edges] plus *total_weight. */
ecl_status ecl_batch_result(const ecl_batch* b, int32_t i, uint32_t code, void* host_out, uint64_t* total_weight);

#ifdef __cplusplus
}
#endif

#endif /* ECL_BATCH_H */
