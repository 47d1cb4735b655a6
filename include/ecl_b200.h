/*
 * ecl_b200.h -- C ABI of the B200-native race-free graph codes.
 *
 * One shared library (libeclb200.so) exports every entry point below with
 * plain C types only: no CUDA, torch or C++ types cross this boundary, so the
 * library can be bound from ctypes, cgo, JNI or plain C.
 *
 * The reference (ECL-Suite) ships six standalone executables and no library.
 * Each entry point here replaces the internal host driver of one of them; the
 * citation beside each declaration names the reference function (path:line
 * within the ECL-Suite project) whose input/output contract it keeps.
 *
 * Conventions shared by every solver:
 *  - The graph is the ECLgraph CSR (library/ECLgraph.h:41-47): int32 nodes,
 *    int32 edges, nindex[nodes+1], nlist[edges], optional eweight[edges].
 *  - `location` says where the CSR arrays AND the output arrays live.
 *    ECL_HOST: the call copies the CSR to the device, solves, copies the
 *    result back and returns with everything finished.  ECL_DEVICE: all
 *    pointers are device pointers of the current CUDA device and nothing
 *    crosses PCIe.
 *  - Every call is stream-ordered on opts->stream (NULL = the legacy default
 *    stream) and synchronises that stream before it returns, because the
 *    device-side status word (non-convergence, bad input detected on the
 *    device) is read back to form the return code.
 *  - Errors are return codes; the library never calls exit() (the reference
 *    does, library/ECLatomic.h:57-75).
 *  - Scratch memory comes from opts->workspace when it is non-NULL and at
 *    least ecl_workspace_bytes() large; otherwise the call allocates it
 *    stream-ordered and frees it before returning.
 */
#ifndef ECL_B200_H
#define ECL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ECL_B200_ABI_VERSION 2

typedef enum ecl_status {
  ECL_OK = 0,
  ECL_ERR_INVALID_ARG = 1,    /* NULL pointer, negative size, bad option */
  ECL_ERR_BAD_GRAPH = 2,      /* CSR fails validation (nindex not monotone, id out of range, ...) */
  ECL_ERR_OOM = 3,            /* device or host allocation failed, or workspace too small */
  ECL_ERR_NO_CONVERGENCE = 4, /* a device fixpoint loop hit its round cap */
  ECL_ERR_CUDA = 5,           /* a CUDA runtime call failed */
  ECL_ERR_IO = 6,             /* file could not be opened, read or written */
  ECL_ERR_UNSUPPORTED = 7,    /* input outside the supported range (e.g. APSP n too large) */
  ECL_ERR_NO_DEVICE = 8       /* no CUDA device, or not an sm_100 device */
} ecl_status;

typedef enum ecl_location { ECL_HOST = 0, ECL_DEVICE = 1 } ecl_location;

/* Graph flags (ecl_graph_view.flags). */
#define ECL_GRAPH_SYMMETRIC 0x1 /* caller asserts that (u,v) in nlist implies (v,u) */

typedef struct ecl_graph_view {
  int32_t nodes;
  int32_t edges;
  const int32_t* nindex;  /* nodes + 1 entries, nindex[0] == 0, nindex[nodes] == edges */
  const int32_t* nlist;   /* edges entries, each in [0, nodes) */
  const int32_t* eweight; /* edges entries, or NULL when the graph has no weights */
  int32_t location;       /* ecl_location of nindex/nlist/eweight and of the outputs */
  int32_t flags;          /* ECL_GRAPH_* */
} ecl_graph_view;

typedef struct ecl_opts {
  void* stream;           /* cudaStream_t; NULL = legacy default stream */
  void* workspace;        /* device scratch, or NULL (the call allocates) */
  size_t workspace_bytes; /* size of workspace */
  int32_t validate;       /* 1: validate the CSR on the host before any launch */
  int32_t max_rounds;     /* cap on device fixpoint rounds; 0 = built-in default */
  float elapsed_ms;       /* out: device time of the compute phase (CUDA events) */
  int32_t rounds;         /* out: fixpoint rounds / sweeps the solve took */
  int32_t detail;         /* 1: also time each kernel phase (events between phases) */
  int32_t nphases;        /* out: number of phase_ms entries written */
  float phase_ms[8];      /* out: device time of each kernel phase, in launch order */
} ecl_opts;

/* Launch knobs: how the solvers schedule their work, never what they compute
 * (0 = built-in default).  The reference fixes the matching choices at compile
 * time: CC's per-thread / per-warp / per-block row thresholds
 * (ECL-CC-atomic.cu:62,120,122), GC's block size and warp rows
 * (ECL-GC-atomic.cu:60-64,93), MST's warp path and light-edge sample
 * (ECL-MST_10-atomic.cu:197,450-459). */
typedef struct ecl_tune {
  int32_t blocks_per_sm;  /* blocks of 256 threads per SM in the grid-stride kernels' grids, 1..128; 0 = 64 */
  float mst_light_factor; /* MST light-edge target, in multiples of n; 0 = 0.75 */
  int32_t gc_core_ranks;  /* GC: leading ranks coloured in shared memory (the core), 0..36864; 0 = 8192 */
  int32_t row_lane_max;   /* CSR scans: rows of at most this many entries go to one lane, 0..32; 0 = per code */
  int32_t row_chunk;      /* CSR scans: rows longer than this are cut into chunks of this many entries;
                             0 = per code, else a power of two in 128..8192 */
  int32_t scc_sweep_batch; /* SCC: edges per lane whose loads a sweep keeps in flight: 1, 2 or 4; 0 = 1 */
  int32_t gc_poll_ns;      /* GC: longest sleep between polls of a long row's dependency, 0..4096 ns; 0 = 64 */
  int32_t row_vec;         /* CSR scans: 1 = warp rows read in 16-byte quads where aligned; 0 = 4-byte loads
                              (measured faster: the quads scatter the per-entry writes that follow) */
  int32_t gc_pull_blocks;  /* GC pull: blocks of 256 threads per SM, 1..4; 0 = 2 */
  int32_t gc_core_ctas;    /* GC core: CTAs of the cluster that colours it, 1..8; 0 = 2 */
} ecl_tune;

/* Process-wide knobs of the single-graph entry points (ecl_cc ... ecl_scc);
 * the batched engine keeps its own (ecl_batch_set_tune).  Out-of-range values
 * give ECL_ERR_INVALID_ARG and change nothing. */
ecl_status ecl_set_tune(const ecl_tune* t);
ecl_status ecl_get_tune(ecl_tune* t);

/* Solver identifiers (ecl_workspace_bytes). */
typedef enum ecl_code { ECL_CC = 0, ECL_MIS = 1, ECL_GC = 2, ECL_MST = 3, ECL_SCC = 4, ECL_APSP = 5 } ecl_code;

/* MIS status bytes, as in src/racefree/egr-input/MIS/ECL-MIS-atomic.cu:67-68. */
#define ECL_MIS_IN 0xfe
#define ECL_MIS_OUT 0x00

/* APSP "infinity", as in src/racefree/grid-input/ECL-APSP-atomic.cu:69. */
#define ECL_APSP_INF (0x7fffffff / 2)

/* ---- library ------------------------------------------------------------------ */

int32_t ecl_abi_version(void);
const char* ecl_status_string(ecl_status s);
/* Text of the last CUDA/allocation failure seen by this thread ("" if none). */
const char* ecl_last_error(void);
/* Bytes of device scratch that `code` needs for a graph of this size. */
size_t ecl_workspace_bytes(ecl_code code, int32_t nodes, int32_t edges);
/* Number of this library's kernel launches since load (a process-wide counter). */
uint64_t ecl_kernel_launches(void);
/* Measured INT32 min-plus throughput of the current device, in integer
 * operations per second (one update = add + min = 2 operations): the roofline
 * denominator of ecl_apsp.  variant 0 times the DPX add-min instruction the
 * APSP kernels issue, variant 1 a separate add and min.  No counterpart in the
 * reference. */
ecl_status ecl_minplus_peak(int32_t variant, double* ops_per_s);
/* Measured time of one dependency hop on the current device, in ns: a warp
 * stores a value another warp polls for, and that warp's next store follows.
 * variant 0: between two SMs through an L2 word, polled the way GC's pull
 * polls (sleep back-off); 1: the same with a bare spin; 2: between two warps
 * of one CTA through shared memory, polled the way GC's core polls.  The
 * latency denominators of GC's roofline.  No counterpart in the reference. */
ecl_status ecl_hop_latency(int32_t variant, double* ns_per_hop);
/* Measured streaming-gather rate of the current device, in entries per second:
 * the m device indices d_index[0..m) (each in [0, n)) are read once and each
 * loads one 8-byte word of an n-word table that sits in L2 -- the work per
 * entry of every CSR scan here (GC's key, MST's root, SCC's flag), and so the
 * roofline of a scan over a graph whose column indices are d_index.  variant 0
 * loads through the read-only path, 1 with relaxed device-scope atomic loads.
 * No counterpart in the reference. */
ecl_status ecl_gather_peak(const int32_t* d_index, int32_t m, int32_t n, int32_t variant, double* entries_per_s);
/* GC's critical path, computed on the host for a host graph: *hops = the
 * longest chain of higher-priority dependencies (ECL-GC-atomic.cu:102
 * priorities), *hops_core = its part inside the first min(long rows,
 * core_ranks) ranks (0 = the default core size), and *path_ns = the longest
 * chain's time when a hop into the core costs hop_core_ns and any other hop
 * hop_rest_ns -- the latency bound of ecl_gc.  No counterpart in the reference. */
ecl_status ecl_gc_critical_path(const ecl_graph_view* g, int32_t core_ranks, double hop_core_ns, double hop_rest_ns,
                                int32_t* hops, int32_t* hops_core, double* path_ns);

/* ---- solvers ------------------------------------------------------------------ */

/* Connected components.  label[v] = smallest vertex id in v's component, where
 * the components are those of the undirected graph formed by the entries
 * nlist[i] < v of each vertex v's list -- exactly the edges the reference
 * hooks (src/racefree/egr-input/CC/ECL-CC-atomic.cu:114-153) -- so the labels
 * equal the reference's nstat for every input, symmetric or not.
 * Replaces computeCC (ECL-CC-atomic.cu:275). */
ecl_status ecl_cc(const ecl_graph_view* g, int32_t* label, ecl_opts* opts);

/* Maximal independent set.  status[v] = ECL_MIS_IN (0xfe) or ECL_MIS_OUT (0).
 * The set is the greedy MIS in descending (priority byte, vertex id) order,
 * with the reference's hash priority (ECL-MIS-atomic.cu:109-136), i.e. the
 * set the reference's findmins (ECL-MIS-atomic.cu:72-104) converges to.
 * The graph must be symmetric and free of self-loops (the reference spins
 * forever otherwise); opts->validate=1 checks this on the host.
 * Replaces computeMIS (ECL-MIS-atomic.cu:147). */
ecl_status ecl_mis(const ecl_graph_view* g, uint8_t* status, ecl_opts* opts);

/* Graph colouring.  color[v] >= 0, adjacent vertices differ.  The colouring is
 * first-fit greedy in the reference's priority order: degree, then hash, then
 * id (ECL-GC-atomic.cu:102), which is what init/runLarge/runSmall
 * (ECL-GC-atomic.cu:78-303) compute.  Graph must be symmetric, no self-loops.
 * Replaces the GC driver inlined in main (ECL-GC-atomic.cu:333-373). */
ecl_status ecl_gc(const ecl_graph_view* g, int32_t* color, ecl_opts* opts);

/* Minimum spanning forest.  in_mst[j] = 1 for the CSR entries j (the v<n copy
 * of each undirected edge, ECL-MST_10-atomic.cu:203) that form the unique
 * minimum spanning forest under the (eweight, edge index) order, else 0.
 * *total_weight (may be NULL) receives the forest weight.  Weights must be
 * non-negative; only the v<n copy of each weight is read.
 * Replaces gpuMST<filter> (ECL-MST_10-atomic.cu:285-382). */
ecl_status ecl_mst(const ecl_graph_view* g, uint8_t* in_mst, uint64_t* total_weight, ecl_opts* opts);

/* Strongly connected components of the directed graph.  label[v] = largest
 * vertex id in v's SCC, the value the reference reads out as
 * readFirst(iomax[v]) (ECL-SCC_10-atomic.cu:318).
 * Replaces the SCC driver inlined in main (ECL-SCC_10-atomic.cu:240-311). */
ecl_status ecl_scc(const ecl_graph_view* g, int32_t* label, ecl_opts* opts);

/* All-pairs shortest paths (Floyd-Warshall).  dist is nodes x ld int32,
 * row-major, ld >= nodes; dist[i*ld+j] = shortest i->j distance, ECL_APSP_INF
 * when unreachable.  The initial matrix follows init1/init2
 * (ECL-APSP-atomic.cu:63-83): 0 on the diagonal, eweight[j] at
 * (i, nlist[j]) with the LAST duplicate winning and a self-loop overwriting
 * the 0.  Weights are used as given (the reference's main negates negative
 * ones first, ECL-APSP-atomic.cu:586-590; the CLI drop-in does the same).
 * Requires eweight.  Replaces FW_gpu_64 (ECL-APSP-atomic.cu:460-531). */
ecl_status ecl_apsp(const ecl_graph_view* g, int32_t* dist, int64_t ld, ecl_opts* opts);

/* ---- allocation-free CC ------------------------------------------------------- */

/* No counterpart in the reference.
 *
 * Connected components exactly as ecl_cc computes them, for callers that must
 * not allocate device memory during a solve: code whose process hands all
 * device memory to another framework's pool (so cudaMalloc fails or fragments
 * that pool), code inside an allocator callback or a plugin whose host owns
 * every allocation, or a latency-critical section where cudaMalloc's implicit
 * device synchronisation is not acceptable.  The call allocates nothing: the
 * caller passes the graph and the label array (device pointers of the current
 * device, same meaning as ecl_cc), and the solver's scratch is a static device
 * array of ECL_CC_NOALLOC_SCRATCH_BYTES inside this library, which every GPU
 * that loads the library holds until the process exits.
 *
 *  - Graphs with more than ECL_CC_NOALLOC_MAX_EDGES CSR entries are rejected
 *    with ECL_ERR_UNSUPPORTED (use ecl_cc for those).
 *  - The first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current, and looks it up again
 *    after the device's context was replaced (cudaDeviceReset).
 *  - Do not call it while its stream is being captured into a CUDA graph
 *    (nor while a global or relaxed-mode capture is active on another
 *    stream): every call copies the status back and synchronises the stream,
 *    which a capture does not allow.
 *  - All calls share the one array and it keeps the last call's contents (the
 *    call clears what must start at zero).  Calls that overlap on the GPU --
 *    different streams, or threads calling at once -- race on it; serialise
 *    them.
 *  - Runs on `stream` (a cudaStream_t, NULL = legacy default stream) and
 *    synchronises it before returning the status. */
#define ECL_CC_NOALLOC_MAX_EDGES (1 << 27)
#define ECL_CC_NOALLOC_SCRATCH_BYTES (2u << 20)
ecl_status ecl_cc_noalloc(int32_t nodes, int32_t edges, const int32_t* nindex, const int32_t* nlist, int32_t* label,
                          void* stream);

/* ---- reference-shaped wrappers (host pointers, default stream) ---------------- */

/* computeCC(nodes, edges, nidx, nlist, nstat), ECL-CC-atomic.cu:275 */
ecl_status ecl_compute_cc(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist, int32_t* nstat);
/* computeMIS(nodes, edges, nidx, nlist, nstat), ECL-MIS-atomic.cu:147 */
ecl_status ecl_compute_mis(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist, uint8_t* nstat);
/* GC driver in main, ECL-GC-atomic.cu:333-373 */
ecl_status ecl_compute_gc(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist, int32_t* color);
/* gpuMST<filter>(g, threshold), ECL-MST_10-atomic.cu:285; the threshold is
 * a performance knob in the reference and is chosen internally here. */
ecl_status ecl_compute_mst(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist, const int32_t* eweight, uint8_t* in_mst);
/* SCC driver in main, ECL-SCC_10-atomic.cu:240-311 */
ecl_status ecl_compute_scc(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist, int32_t* label);
/* FW_gpu_64(g, AdjMat), ECL-APSP-atomic.cu:460: AdjMat is upper x upper with
 * upper = ceil(nodes/64)*64, exactly the reference's padded output layout
 * (padding rows/columns hold ECL_APSP_INF, as init1 leaves them). */
ecl_status ecl_compute_apsp(int32_t nodes, int32_t edges, const int32_t* nidx, const int32_t* nlist, const int32_t* eweight, int32_t* adjmat);

/* ---- ECLgraph files (library/ECLgraph.h:41-102) -------------------------------- */

typedef struct ecl_graph {
  int32_t nodes;
  int32_t edges;
  int32_t* nindex;
  int32_t* nlist;
  int32_t* eweight; /* NULL when the file has no weights */
} ecl_graph;

/* readECLgraph (ECLgraph.h:49-76): same byte layout and the same rejection of
 * nodes < 1 or edges < 0, but returns ECL_ERR_IO / ECL_ERR_BAD_GRAPH instead of
 * exiting.  Arrays are malloc'ed; release with ecl_graph_free. */
ecl_status ecl_graph_read(const char* path, ecl_graph* out);
/* writeECLgraph (ECLgraph.h:78-92): byte-identical output. */
ecl_status ecl_graph_write(const char* path, const ecl_graph* g);
/* freeECLgraph (ECLgraph.h:94-102). */
void ecl_graph_free(ecl_graph* g);

/* MatrixMarket "coordinate" file -> ECLgraph, with the semantics of the
 * reference's converter (scripts/mm2ecl_real.cpp:50-184): square matrices,
 * general or symmetric, pattern / integer / real; entries sorted by (row,
 * column), 1-based ids made 0-based, real weights stored as (int)(w * 100),
 * rows without entries get empty lists.  Like the reference, a "symmetric"
 * file is NOT mirrored unless symmetrise != 0; then every off-diagonal entry
 * (i, j) also yields (j, i) with the same weight. */
ecl_status ecl_graph_from_mm(const char* path, int32_t symmetrise, ecl_graph* out);

/* Host-side CSR checks.  require_symmetric / forbid_self_loops add those
 * checks (O(edges log deg)); returns ECL_OK or ECL_ERR_BAD_GRAPH. */
ecl_status ecl_graph_validate(const ecl_graph_view* g, int32_t require_symmetric, int32_t forbid_self_loops);

/* ---- seeded synthetic generators (host, deterministic for any thread count) ---- */

/* R-MAT: 2^scale vertices, edge_factor * 2^scale sampled edges with quadrant
 * probabilities (a, b, c, 1-a-b-c).  symmetrise=1 adds both directions.
 * Self-loops and duplicates are always removed; lists are sorted.
 * weight_seed != 0 attaches weights uniform in [1, weight_max), symmetric per
 * unordered pair.  The graph is malloc'ed; release with ecl_graph_free. */
ecl_status ecl_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                        int32_t symmetrise, uint64_t weight_seed, int32_t weight_max, ecl_graph* out);
/* 2D rows x cols 4-neighbour grid, undirected; each undirected edge is deleted
 * independently with probability delete_frac (seed). */
ecl_status ecl_gen_grid(int32_t rows, int32_t cols, double delete_frac, uint64_t seed, uint64_t weight_seed,
                        int32_t weight_max, ecl_graph* out);
/* Erdos-Renyi G(n, p).  symmetrise=0: each ordered pair (i != j) independently
 * (a directed graph); symmetrise=1: each unordered pair, stored both ways.
 * Weights uniform in [weight_min, weight_max] inclusive when weight_seed != 0
 * (independent per directed entry when symmetrise=0, per pair otherwise). */
ecl_status ecl_gen_er(int32_t n, double p, uint64_t seed, int32_t symmetrise, uint64_t weight_seed,
                      int32_t weight_min, int32_t weight_max, ecl_graph* out);

#ifdef __cplusplus
}
#endif

#endif /* ECL_B200_H */
