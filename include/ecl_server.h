/*
 * ecl_server.h -- continuous-batching request server over resident graphs.
 *
 * No counterpart in the reference (one graph per process, no serving mode).
 * Graphs are registered once and stay resident in HBM.  A request names a
 * code and a registered graph and carries an arrival time; ecl_server_run
 * replays a request stream in real time:
 *  - a request that has arrived is admitted as soon as a slot (one CUDA
 *    stream each) is free AND its memory (workspace + output) fits in the HBM
 *    budget next to the resident graphs and the requests in flight -- first
 *    fit, so a small request does not wait behind a large one that does not
 *    fit yet;
 *  - admitted requests run concurrently on their slots' streams and release
 *    their memory (stream-ordered) when they finish;
 *  - latency = completion time - arrival time, measured on the host clock.
 * Every result equals the solo solve of the same request (the solvers keep no
 * state between calls and each request has its own workspace).
 */
#ifndef ECL_SERVER_H
#define ECL_SERVER_H

#include "ecl_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ecl_server ecl_server;

typedef struct ecl_server_cfg {
  int32_t slots;             /* concurrent requests (CUDA streams); 0 = 8 */
  uint64_t hbm_budget_bytes; /* resident graphs + in-flight requests; 0 = 160 GB */
} ecl_server_cfg;

typedef struct ecl_request {
  int32_t code;        /* ecl_code: ECL_CC, ECL_MIS, ECL_GC, ECL_MST or ECL_SCC */
  int32_t graph;       /* id from ecl_server_add_graph */
  double arrival_s;    /* arrival time, seconds after the start of the run */
  void* out;           /* host buffer for the result (the code's single-graph layout), or NULL.
                          It must be page-locked (cudaHostAlloc / cudaHostRegister): the result is
                          copied back asynchronously on the request's slot stream, and a pageable
                          buffer would make that copy wait for the solve, stalling the one host
                          thread that admits and completes every slot. */
  /* filled in by ecl_server_run: */
  uint64_t total_weight; /* MST only */
  double latency_s;      /* completion - arrival */
  double queue_s;        /* admission - arrival */
  int32_t status;        /* ecl_status of this request */
  int32_t slot;
} ecl_request;

typedef struct ecl_server_stats {
  int32_t completed;
  int32_t failed;
  double makespan_s;   /* first arrival to last completion */
  double graphs_per_s; /* completed / makespan */
  double p50_s, p99_s, mean_s;
  int32_t max_in_flight;
  uint64_t peak_bytes;  /* peak of resident + in-flight bytes */
} ecl_server_stats;

ecl_status ecl_server_create(const ecl_server_cfg* cfg, ecl_server** out);
void ecl_server_destroy(ecl_server* s);
/* Uploads a host graph (kept resident until destroy).  *id receives its id.
 * Fails with ECL_ERR_OOM when it does not fit in the budget. */
ecl_status ecl_server_add_graph(ecl_server* s, const ecl_graph_view* g, int32_t* id);
/* Replays the request stream (sorted or not; arrival_s decides) and returns
 * when every request has finished.  Per-request status, latency and results
 * are written into reqs[]. */
ecl_status ecl_server_run(ecl_server* s, ecl_request* reqs, int32_t count, ecl_server_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* ECL_SERVER_H */
