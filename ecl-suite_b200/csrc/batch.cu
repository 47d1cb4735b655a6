// Batched engine: many graphs solved by one set of launches (see ecl_batch.h).
//
// Layout per super-batch (device): the union CSR -- nindex[N+1] with every
// graph's offsets shifted by its entry base, nlist[M] with every id shifted by
// its vertex base, eweight[M] -- plus vbase[G+1], ebase[G+1], avg[G] (the
// per-graph offset tables) and the concatenated outputs.  One workspace of the
// largest solver's size is shared by the codes, which run one after another
// on the batch's stream.  The whole sequence (status clears, every code of
// every super-batch, the per-graph MST weight reduction) is captured once
// into a CUDA graph and replayed.
#include <cmath>
#include <cstring>
#include <vector>

#include <omp.h>

#include "ecl_batch.h"
#include "host_util.h"
#include "solvers.cuh"

namespace ecl {
namespace batchimpl {

struct HostGraph {
  int n = 0, m = 0;
  std::vector<int> nindex, nlist, eweight;
  bool sym = false;
};

constexpr int kCodes = 5;  // status blocks per super-batch: CC, MIS, GC, MST, SCC

struct Super {
  int first = 0, count = 0;  // graph range
  int n = 0, m = 0;
  bool sym = true, weighted = true;
  std::vector<int> h_vbase, h_ebase;
  int *nindex = nullptr, *nlist = nullptr, *eweight = nullptr;
  int *vbase = nullptr, *ebase = nullptr;
  float* avg = nullptr;
  int *cc = nullptr, *gc = nullptr, *scc = nullptr;
  unsigned char *mis = nullptr, *mst = nullptr;
  unsigned long long* totals = nullptr;  // per graph
  char* ws = nullptr;
  dev::Status* status = nullptr;  // kCodes blocks
};

}  // namespace batchimpl

namespace {

using namespace dev;
using batchimpl::HostGraph;
using batchimpl::kCodes;
using batchimpl::Super;

// Per-graph MST weight: warp per graph sums the weights of its flagged entries.
__global__ void batch_mst_totals(int ngraphs, const int* __restrict__ ebase, const unsigned char* __restrict__ in_mst,
                                 const int* __restrict__ eweight, unsigned long long* __restrict__ totals) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int g = warp; g < ngraphs; g += nwarps) {
    unsigned long long s = 0;
    for (int j = __ldg(&ebase[g]) + lane; j < __ldg(&ebase[g + 1]); j += 32)
      if (in_mst[j]) s += (unsigned)__ldg(&eweight[j]);  // race-free: in_mst is final (MST finished)
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
    if (lane == 0) totals[g] = s;
  }
}

}  // namespace
}  // namespace ecl

struct ecl_batch {
  std::vector<ecl::batchimpl::HostGraph> graphs;
  std::vector<ecl::batchimpl::Super> sup;
  uint32_t codes = 0;
  cudaStream_t stream = nullptr;  // the engine's own non-blocking stream (runs + capture)
  ecl::DeviceInfo dev;
  ecl_tune tune{};
  int32_t tune_points = 0;  // knob settings the last ecl_batch_tune timed
  std::vector<void*> allocs;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  bool built = false;
  bool capture_failed = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace ecl {
namespace {

template <class T>
T* dalloc(ecl_batch* b, size_t count, ecl_status* st) {
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
    cudaGetLastError();
    *st = ECL_ERR_OOM;
    return nullptr;
  }
  b->allocs.push_back(p);
  return static_cast<T*>(p);
}

void drop_graph_exec(ecl_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// Enqueues one full run (every code, every super-batch) on b->stream.
ecl_status enqueue_run(ecl_batch* b) {
  DeviceInfo dev = b->dev;
  apply_tune(&dev, b->tune);
  for (Super& s : b->sup) {
    ECL_CUDA_TRY(cudaMemsetAsync(s.status, 0, kStatusBytes * kCodes, b->stream));
    GraphDev g;
    g.n = s.n;
    g.m = s.m;
    g.nindex = s.nindex;
    g.nlist = s.nlist;
    g.eweight = s.eweight;
    g.flags = s.sym ? ECL_GRAPH_SYMMETRIC : 0;
    UnionInfo uni;
    uni.ngraphs = s.count;
    uni.vbase = s.vbase;
    uni.avg = s.avg;
    auto stat = [&](int k) { return reinterpret_cast<Status*>(reinterpret_cast<char*>(s.status) + k * kStatusBytes); };
    ecl_status st = ECL_OK;
    if (b->codes & ECL_BATCH_CC) st = cc_enqueue(g, s.cc, s.ws, stat(0), dev, b->stream);
    if (st == ECL_OK && (b->codes & ECL_BATCH_MIS)) st = mis_enqueue(g, s.mis, s.ws, stat(1), dev, b->stream, 1 << 22, &uni);
    if (st == ECL_OK && (b->codes & ECL_BATCH_GC)) st = gc_enqueue(g, s.gc, s.ws, stat(2), dev, b->stream, &uni);
    if (st == ECL_OK && (b->codes & ECL_BATCH_MST)) {
      st = mst_enqueue(g, s.mst, s.ws, stat(3), dev, b->stream, nullptr);
      if (st == ECL_OK) {
        ECL_LAUNCH(batch_mst_totals, dev.sms * 4, 256, 0, b->stream, s.count, s.ebase, s.mst, s.eweight, s.totals);
      }
    }
    if (st == ECL_OK && (b->codes & ECL_BATCH_SCC)) st = scc_enqueue(g, s.scc, s.ws, stat(4), dev, b->stream, 0);
    if (st != ECL_OK) return st;
  }
  return ECL_OK;
}

ecl_status check_status(ecl_batch* b) {
  std::vector<Status> hs(kCodes);
  for (Super& s : b->sup) {
    for (int k = 0; k < kCodes; k++) {
      ECL_CUDA_TRY(cudaMemcpyAsync(&hs[k], reinterpret_cast<char*>(s.status) + k * kStatusBytes, sizeof(Status),
                                   cudaMemcpyDeviceToHost, b->stream));
    }
    ECL_CUDA_TRY(cudaStreamSynchronize(b->stream));
    for (int k = 0; k < kCodes; k++)
      if (hs[k].code != 0) return static_cast<ecl_status>(hs[k].code);
  }
  return ECL_OK;
}

}  // namespace
}  // namespace ecl

extern "C" {

ecl_status ecl_batch_create(ecl_batch** out) {
  if (!out) return ECL_ERR_INVALID_ARG;
  *out = new ecl_batch();
  return ECL_OK;
}

void ecl_batch_destroy(ecl_batch* b) {
  if (!b) return;
  ecl::drop_graph_exec(b);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (void* p : b->allocs) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
}

ecl_status ecl_batch_add(ecl_batch* b, const ecl_graph_view* g) {
  if (!b || !g || b->built) return ECL_ERR_INVALID_ARG;
  if (g->location != ECL_HOST || g->nodes < 1 || g->edges < 0 || !g->nindex) return ECL_ERR_INVALID_ARG;
  ecl::batchimpl::HostGraph h;
  h.n = g->nodes;
  h.m = g->edges;
  h.nindex.assign(g->nindex, g->nindex + h.n + 1);
  if (h.nindex[0] != 0 || h.nindex[h.n] != h.m) return ECL_ERR_BAD_GRAPH;
  if (h.m) h.nlist.assign(g->nlist, g->nlist + h.m);
  if (g->eweight && h.m) h.eweight.assign(g->eweight, g->eweight + h.m);
  h.sym = (g->flags & ECL_GRAPH_SYMMETRIC) != 0;
  b->graphs.push_back(std::move(h));
  return ECL_OK;
}

ecl_status ecl_batch_add_mix(ecl_batch* b, int32_t count, int32_t n_min, int32_t n_max, uint64_t seed,
                             int32_t weight_max) {
  using ecl::host::mix64;
  using ecl::host::unit_double;
  if (!b || b->built || count < 0 || n_min < 2 || n_max < n_min || weight_max < 2) return ECL_ERR_INVALID_ARG;
  std::vector<ecl::batchimpl::HostGraph> gs((size_t)count);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int i = 0; i < count; i++) {
    const uint64_t h = mix64(seed * 0x9e3779b97f4a7c15ull + (uint64_t)i);
    const double u = unit_double(mix64(h ^ 0x1234567ull));
    const int n = (int)std::floor(std::exp(std::log((double)n_min) + u * (std::log((double)n_max) - std::log((double)n_min))));
    const int kind = (int)(mix64(h ^ 0xabcdefull) % 3);
    const uint64_t gseed = mix64(h ^ 0x5555ull) | 1, wseed = mix64(h ^ 0x7777ull) | 1;
    ecl_graph g{};
    ecl_status st;
    if (kind == 0) {
      st = ecl_gen_er(n, 8.0 / (double)(n - 1), gseed, 1, wseed, 1, weight_max - 1, &g);
    } else if (kind == 1) {
      const int rows = std::max(1, (int)std::sqrt((double)n));
      st = ecl_gen_grid(rows, std::max(1, n / rows), 0.0, gseed, wseed, weight_max, &g);
    } else {
      const int scale = std::max(1, (int)std::lround(std::log2((double)n)));
      st = ecl_gen_rmat(scale, 8, 0.57, 0.19, 0.19, gseed, 1, wseed, weight_max, &g);
    }
    if (st != ECL_OK) {
      bad |= 1;
      continue;
    }
    ecl::batchimpl::HostGraph& hg = gs[(size_t)i];
    hg.n = g.nodes;
    hg.m = g.edges;
    hg.nindex.assign(g.nindex, g.nindex + g.nodes + 1);
    hg.nlist.assign(g.nlist, g.nlist + g.edges);
    hg.eweight.assign(g.eweight, g.eweight + g.edges);
    hg.sym = true;
    ecl_graph_free(&g);
  }
  if (bad) return ECL_ERR_OOM;
  for (auto& g : gs) b->graphs.push_back(std::move(g));
  return ECL_OK;
}

ecl_status ecl_batch_build(ecl_batch* b, uint32_t codes, int64_t max_entries, void* stream) {
  using namespace ecl;
  using batchimpl::HostGraph;
  using batchimpl::Super;
  if (!b || b->built || b->graphs.empty() || codes == 0) return ECL_ERR_INVALID_ARG;
  ecl_status st = current_device(&b->dev);
  if (st != ECL_OK) return st;
  b->codes = codes;
  // Runs are captured into a CUDA graph, which the legacy default stream does
  // not allow: the engine works on its own non-blocking stream, ordered after
  // the caller's stream once here.
  ECL_CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  ECL_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  const int64_t cap = (max_entries > 0) ? std::min<int64_t>(max_entries, (int64_t)1 << 30) : ((int64_t)1 << 29);
  // pack consecutive graphs into super-batches
  size_t i = 0;
  while (i < b->graphs.size()) {
    Super s;
    s.first = (int)i;
    int64_t n = 0, m = 0;
    while (i < b->graphs.size()) {
      const HostGraph& g = b->graphs[i];
      if (s.count > 0 && (m + g.m > cap || n + g.n > ((int64_t)1 << 30))) break;
      n += g.n;
      m += g.m;
      s.count++;
      s.sym = s.sym && g.sym;
      s.weighted = s.weighted && ((int)g.eweight.size() == g.m);
      i++;
    }
    if (n > INT32_MAX - 1 || m > INT32_MAX - 1) return ECL_ERR_UNSUPPORTED;
    s.n = (int)n;
    s.m = (int)m;
    b->sup.push_back(std::move(s));
  }
  if ((codes & ECL_BATCH_MST)) {
    for (Super& s : b->sup)
      if (!s.weighted) return ECL_ERR_INVALID_ARG;
  }
  for (Super& s : b->sup) {
    // host union
    std::vector<int> nindex((size_t)s.n + 1), nlist((size_t)std::max(s.m, 1)), eweight;
    if (s.weighted) eweight.resize((size_t)std::max(s.m, 1));
    std::vector<float> avg((size_t)s.count);
    s.h_vbase.resize((size_t)s.count + 1);
    s.h_ebase.resize((size_t)s.count + 1);
    int vb = 0, eb = 0;
    for (int k = 0; k < s.count; k++) {
      const HostGraph& g = b->graphs[(size_t)s.first + k];
      s.h_vbase[k] = vb;
      s.h_ebase[k] = eb;
      avg[k] = (float)g.m / (float)g.n;  // as ECL-MIS-atomic.cu:123
      vb += g.n;
      eb += g.m;
    }
    s.h_vbase[s.count] = vb;
    s.h_ebase[s.count] = eb;
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < s.count; k++) {
      const HostGraph& g = b->graphs[(size_t)s.first + k];
      const int v0 = s.h_vbase[k], e0 = s.h_ebase[k];
      for (int v = 0; v < g.n; v++) nindex[(size_t)v0 + v] = e0 + g.nindex[v];
      for (int j = 0; j < g.m; j++) nlist[(size_t)e0 + j] = v0 + g.nlist[j];
      if (s.weighted && g.m) memcpy(&eweight[(size_t)e0], g.eweight.data(), sizeof(int) * (size_t)g.m);
    }
    nindex[s.n] = s.m;
    // device buffers
    s.nindex = dalloc<int>(b, (size_t)s.n + 1, &st);
    s.nlist = dalloc<int>(b, (size_t)std::max(s.m, 1), &st);
    if (s.weighted) s.eweight = dalloc<int>(b, (size_t)std::max(s.m, 1), &st);
    s.vbase = dalloc<int>(b, (size_t)s.count + 1, &st);
    s.ebase = dalloc<int>(b, (size_t)s.count + 1, &st);
    s.avg = dalloc<float>(b, (size_t)s.count, &st);
    if (codes & ECL_BATCH_CC) s.cc = dalloc<int>(b, (size_t)s.n, &st);
    if (codes & ECL_BATCH_MIS) s.mis = dalloc<unsigned char>(b, (size_t)s.n, &st);
    if (codes & ECL_BATCH_GC) s.gc = dalloc<int>(b, (size_t)s.n, &st);
    if (codes & ECL_BATCH_SCC) s.scc = dalloc<int>(b, (size_t)s.n, &st);
    if (codes & ECL_BATCH_MST) {
      s.mst = dalloc<unsigned char>(b, (size_t)std::max(s.m, 1), &st);
      s.totals = dalloc<unsigned long long>(b, (size_t)s.count, &st);
    }
    size_t wsb = 0;
    if (codes & ECL_BATCH_CC) wsb = std::max(wsb, cc_workspace_bytes(s.n, s.m));
    if (codes & ECL_BATCH_MIS) wsb = std::max(wsb, mis_workspace_bytes(s.n, s.m));
    if (codes & ECL_BATCH_GC) wsb = std::max(wsb, gc_workspace_bytes(s.n, s.m));
    if (codes & ECL_BATCH_MST) wsb = std::max(wsb, mst_workspace_bytes(s.n, s.m));
    if (codes & ECL_BATCH_SCC) wsb = std::max(wsb, scc_workspace_bytes(s.n, s.m));
    s.ws = dalloc<char>(b, wsb, &st);
    s.status = reinterpret_cast<Status*>(dalloc<char>(b, kStatusBytes * kCodes, &st));
    if (st != ECL_OK) return st;
    ECL_CUDA_TRY(cudaMemcpyAsync(s.nindex, nindex.data(), sizeof(int) * ((size_t)s.n + 1), cudaMemcpyHostToDevice, b->stream));
    if (s.m) ECL_CUDA_TRY(cudaMemcpyAsync(s.nlist, nlist.data(), sizeof(int) * (size_t)s.m, cudaMemcpyHostToDevice, b->stream));
    if (s.weighted && s.m)
      ECL_CUDA_TRY(cudaMemcpyAsync(s.eweight, eweight.data(), sizeof(int) * (size_t)s.m, cudaMemcpyHostToDevice, b->stream));
    ECL_CUDA_TRY(cudaMemcpyAsync(s.vbase, s.h_vbase.data(), sizeof(int) * ((size_t)s.count + 1), cudaMemcpyHostToDevice, b->stream));
    ECL_CUDA_TRY(cudaMemcpyAsync(s.ebase, s.h_ebase.data(), sizeof(int) * ((size_t)s.count + 1), cudaMemcpyHostToDevice, b->stream));
    ECL_CUDA_TRY(cudaMemcpyAsync(s.avg, avg.data(), sizeof(float) * (size_t)s.count, cudaMemcpyHostToDevice, b->stream));
    ECL_CUDA_TRY(cudaStreamSynchronize(b->stream));  // host union buffers go out of scope
  }
  ECL_CUDA_TRY(cudaEventCreate(&b->ev0));
  ECL_CUDA_TRY(cudaEventCreate(&b->ev1));
  b->built = true;
  return ECL_OK;
}

ecl_status ecl_batch_run(ecl_batch* b, ecl_opts* opts) {
  using namespace ecl;
  if (!b || !b->built) return ECL_ERR_INVALID_ARG;
  if (!b->exec && !b->capture_failed) {
    // Capture the whole run once; fall back to direct launches if the
    // capture is refused.
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
      const ecl_status st = enqueue_run(b);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      cudaError_t ie = cudaErrorUnknown;
      if (st == ECL_OK && e == cudaSuccess && g) ie = cudaGraphInstantiate(&b->exec, g, 0);
      if (ie == cudaSuccess) {
        b->graph = g;
      } else {
        set_last_error(st != ECL_OK ? "batch capture: enqueue" : (e != cudaSuccess ? "batch capture: end" : "batch capture: instantiate"),
                       st != ECL_OK ? cudaGetLastError() : (e != cudaSuccess ? e : ie));
        if (g) cudaGraphDestroy(g);
        b->exec = nullptr;
        b->capture_failed = true;
      }
    } else {
      set_last_error("batch capture: begin", cudaGetLastError());
      b->capture_failed = true;
    }
    cudaGetLastError();
  }
  ECL_CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
  if (b->exec) {
    ECL_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    count_launch();
  } else {
    const ecl_status st = enqueue_run(b);
    if (st != ECL_OK) return st;
  }
  ECL_CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
  ECL_CUDA_TRY(cudaEventSynchronize(b->ev1));
  if (opts) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    opts->elapsed_ms = ms;
    opts->rounds = b->exec ? 1 : 0;  // 1 when the run was a CUDA-graph replay
  }
  return check_status(b);
}

ecl_status ecl_batch_set_tune(ecl_batch* b, const ecl_tune* t) {
  if (!b || !t || !ecl::tune_valid(*t)) return ECL_ERR_INVALID_ARG;
  b->tune = *t;
  ecl::drop_graph_exec(b);
  b->capture_failed = false;
  return ECL_OK;
}

// The autotuner: coordinate descent over the launch knobs on the built batch.
// Starting from the defaults, each knob in turn takes every candidate value
// (the others held at the best point so far) and keeps the fastest; a point
// costs one capturing run plus `trials` timed replays.  The knobs are the
// ones the reference fixes at compile time -- grid size, the per-lane / per-
// warp / chunk row thresholds (ECL-CC-atomic.cu:62,120,122; ECL-MST_10-
// atomic.cu:197), the MST light/heavy split (ECL-MST_10-atomic.cu:450-459)
// and, with GC in the batch, the size of GC's shared-memory core.
ecl_status ecl_batch_tune(ecl_batch* b, int32_t trials, ecl_tune* best) {
  using namespace ecl;
  if (!b || !b->built || trials < 1) return ECL_ERR_INVALID_ARG;
  auto time_point = [&](const ecl_tune& t, float* ms) -> ecl_status {
    ecl_status st = ecl_batch_set_tune(b, &t);
    if (st != ECL_OK) return st;
    float tot = 0.f;
    for (int r = 0; r < trials + 1; r++) {  // the first run captures
      ecl_opts o{};
      st = ecl_batch_run(b, &o);
      if (st != ECL_OK) return st;
      if (r > 0) tot += o.elapsed_ms;
    }
    *ms = tot;
    return ECL_OK;
  };
  struct Knob {
    bool active;
    std::vector<float> values;
    void (*set)(ecl_tune&, float);
  };
  const std::vector<Knob> knobs = {
      {true, {64.f, 32.f, 16.f, 8.f}, [](ecl_tune& t, float v) { t.blocks_per_sm = (int32_t)v; }},
      {(b->codes & ECL_BATCH_MST) != 0, {0.75f, 1.5f, 3.f, 0.4f}, [](ecl_tune& t, float v) { t.mst_light_factor = v; }},
      {true, {32.f, 16.f, 8.f}, [](ecl_tune& t, float v) { t.row_lane_max = (int32_t)v; }},
      {true, {256.f, 128.f, 512.f, 2048.f}, [](ecl_tune& t, float v) { t.row_chunk = (int32_t)v; }},
      {(b->codes & ECL_BATCH_GC) != 0, {8192.f, 4096.f, 16384.f}, [](ecl_tune& t, float v) { t.gc_core_ranks = (int32_t)v; }},
      {(b->codes & ECL_BATCH_GC) != 0, {2.f, 1.f, 4.f}, [](ecl_tune& t, float v) { t.gc_core_ctas = (int32_t)v; }},
      {(b->codes & ECL_BATCH_GC) != 0, {2.f, 4.f, 1.f}, [](ecl_tune& t, float v) { t.gc_pull_blocks = (int32_t)v; }},
      {(b->codes & ECL_BATCH_SCC) != 0, {1.f, 2.f, 4.f}, [](ecl_tune& t, float v) { t.scc_sweep_batch = (int32_t)v; }},
  };
  ecl_tune winner{};
  for (const Knob& k : knobs)
    if (k.active) k.set(winner, k.values[0]);
  float best_ms = 0.f;
  ecl_status st = time_point(winner, &best_ms);
  if (st != ECL_OK) return st;
  b->tune_points = 1;
  for (const Knob& k : knobs) {
    if (!k.active) continue;
    for (size_t i = 1; i < k.values.size(); i++) {
      ecl_tune t = winner;
      k.set(t, k.values[i]);
      float ms = 0.f;
      st = time_point(t, &ms);
      if (st != ECL_OK) return st;
      b->tune_points++;
      if (ms < best_ms) {
        best_ms = ms;
        winner = t;
      }
    }
  }
  if (best) *best = winner;
  return ecl_batch_set_tune(b, &winner);
}

int32_t ecl_batch_tune_points(const ecl_batch* b) { return b ? b->tune_points : 0; }

int32_t ecl_batch_graphs(const ecl_batch* b) { return b ? (int32_t)b->graphs.size() : 0; }
int32_t ecl_batch_superbatches(const ecl_batch* b) { return b ? (int32_t)b->sup.size() : 0; }

ecl_status ecl_batch_graph_size(const ecl_batch* b, int32_t i, int32_t* nodes, int32_t* edges) {
  if (!b || i < 0 || i >= (int32_t)b->graphs.size()) return ECL_ERR_INVALID_ARG;
  if (nodes) *nodes = b->graphs[(size_t)i].n;
  if (edges) *edges = b->graphs[(size_t)i].m;
  return ECL_OK;
}

ecl_status ecl_batch_graph_csr(const ecl_batch* b, int32_t i, int32_t* nindex, int32_t* nlist, int32_t* eweight) {
  if (!b || i < 0 || i >= (int32_t)b->graphs.size()) return ECL_ERR_INVALID_ARG;
  const ecl::batchimpl::HostGraph& g = b->graphs[(size_t)i];
  if (nindex) memcpy(nindex, g.nindex.data(), sizeof(int) * ((size_t)g.n + 1));
  if (nlist && g.m) memcpy(nlist, g.nlist.data(), sizeof(int) * (size_t)g.m);
  if (eweight && g.m && !g.eweight.empty()) memcpy(eweight, g.eweight.data(), sizeof(int) * (size_t)g.m);
  return ECL_OK;
}

ecl_status ecl_batch_result(const ecl_batch* b, int32_t i, uint32_t code, void* host_out, uint64_t* total_weight) {
  using namespace ecl;
  using batchimpl::Super;
  if (!b || !b->built || i < 0 || i >= (int32_t)b->graphs.size() || !host_out) return ECL_ERR_INVALID_ARG;
  if (!(b->codes & code)) return ECL_ERR_INVALID_ARG;
  size_t si = 0;
  while (si + 1 < b->sup.size() && b->sup[si + 1].first <= i) si++;
  const Super& s = b->sup[si];
  const int k = i - s.first;
  const int v0 = s.h_vbase[k], n = s.h_vbase[k + 1] - v0;
  const int e0 = s.h_ebase[k], m = s.h_ebase[k + 1] - e0;
  switch (code) {
    case ECL_BATCH_CC:
    case ECL_BATCH_SCC: {
      int32_t* out = static_cast<int32_t*>(host_out);
      ECL_CUDA_TRY(cudaMemcpy(out, (code == ECL_BATCH_CC ? s.cc : s.scc) + v0, sizeof(int) * (size_t)n,
                              cudaMemcpyDeviceToHost));
      for (int v = 0; v < n; v++) out[v] -= v0;  // union ids -> local ids
      return ECL_OK;
    }
    case ECL_BATCH_MIS:
      ECL_CUDA_TRY(cudaMemcpy(host_out, s.mis + v0, (size_t)n, cudaMemcpyDeviceToHost));
      return ECL_OK;
    case ECL_BATCH_GC:
      ECL_CUDA_TRY(cudaMemcpy(host_out, s.gc + v0, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
      return ECL_OK;
    case ECL_BATCH_MST:
      if (m) ECL_CUDA_TRY(cudaMemcpy(host_out, s.mst + e0, (size_t)m, cudaMemcpyDeviceToHost));
      if (total_weight) ECL_CUDA_TRY(cudaMemcpy(total_weight, s.totals + k, sizeof(uint64_t), cudaMemcpyDeviceToHost));
      return ECL_OK;
  }
  return ECL_ERR_INVALID_ARG;
}

}  // extern "C"
