// Continuous-batching request server (see ecl_server.h).
//
// One host thread drives the loop: move arrived requests to the ready list,
// retire finished slots (event query, status block read from pinned host
// memory, stream-ordered free), then admit ready requests first-fit into free
// slots while their bytes fit in the budget.  Each admitted request gets a
// workspace + output from cudaMallocAsync on its slot's stream (the pool makes
// this cheap and returns memory to later requests), its solver's launch-only
// enqueue form, a D2H copy of the result into the caller's buffer and of its
// status block into pinned memory, and a completion event.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "ecl_server.h"
#include "solvers.cuh"

namespace ecl {
namespace serverimpl {

struct ResidentGraph {
  GraphDev g;
  size_t bytes = 0;
  void* nindex = nullptr;
  void* nlist = nullptr;
  void* eweight = nullptr;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  dev::Status* hstatus = nullptr;  // pinned host mirror of the request's status block
  unsigned long long* htotal = nullptr;
  int req = -1;
  void* mem = nullptr;
  size_t bytes = 0;
};

using Clock = std::chrono::steady_clock;

}  // namespace serverimpl
}  // namespace ecl

struct ecl_server {
  ecl_server_cfg cfg{};
  ecl::DeviceInfo dev;
  std::vector<ecl::serverimpl::ResidentGraph> graphs;
  std::vector<ecl::serverimpl::Slot> slots;
  uint64_t resident = 0;
};

namespace ecl {
namespace {

using namespace serverimpl;

size_t out_bytes(int code, const GraphDev& g) {
  switch (code) {
    case ECL_CC:
    case ECL_GC:
    case ECL_SCC: return sizeof(int) * (size_t)g.n;
    case ECL_MIS: return (size_t)g.n;
    case ECL_MST: return (size_t)(g.m > 0 ? g.m : 1);
  }
  return 0;
}

size_t ws_bytes(int code, const GraphDev& g) {
  switch (code) {
    case ECL_CC: return cc_workspace_bytes(g.n, g.m);
    case ECL_MIS: return mis_workspace_bytes(g.n, g.m);
    case ECL_GC: return gc_workspace_bytes(g.n, g.m);
    case ECL_MST: return mst_workspace_bytes(g.n, g.m);
    case ECL_SCC: return scc_workspace_bytes(g.n, g.m);
  }
  return 0;
}

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t request_bytes(int code, const GraphDev& g) {
  return align256(kStatusBytes) + align256(ws_bytes(code, g)) + align256(out_bytes(code, g));
}

// Everything request r puts on slot s's stream after its memory is allocated.
ecl_status enqueue_request(ecl_server* sv, Slot& s, ecl_request& r) {
  const GraphDev& g = sv->graphs[(size_t)r.graph].g;
  char* base = static_cast<char*>(s.mem);
  dev::Status* status = reinterpret_cast<dev::Status*>(base);
  char* ws = base + align256(kStatusBytes);
  char* out = ws + align256(ws_bytes(r.code, g));
  ECL_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(dev::Status), s.stream));
  ecl_status st = ECL_OK;
  unsigned long long* total_dev = nullptr;
  switch (r.code) {
    case ECL_CC: st = cc_enqueue(g, reinterpret_cast<int*>(out), ws, status, sv->dev, s.stream); break;
    case ECL_MIS: st = mis_enqueue(g, reinterpret_cast<unsigned char*>(out), ws, status, sv->dev, s.stream, 1 << 22); break;
    case ECL_GC: st = gc_enqueue(g, reinterpret_cast<int*>(out), ws, status, sv->dev, s.stream); break;
    case ECL_MST:
      st = mst_enqueue(g, reinterpret_cast<unsigned char*>(out), ws, status, sv->dev, s.stream, &total_dev);
      break;
    case ECL_SCC: st = scc_enqueue(g, reinterpret_cast<int*>(out), ws, status, sv->dev, s.stream, 0); break;
    default: st = ECL_ERR_INVALID_ARG;
  }
  if (st != ECL_OK) return st;
  if (r.out) ECL_CUDA_TRY(cudaMemcpyAsync(r.out, out, out_bytes(r.code, g), cudaMemcpyDeviceToHost, s.stream));
  if (total_dev) ECL_CUDA_TRY(cudaMemcpyAsync(s.htotal, total_dev, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s.stream));
  ECL_CUDA_TRY(cudaMemcpyAsync(s.hstatus, status, sizeof(dev::Status), cudaMemcpyDeviceToHost, s.stream));
  return ECL_OK;
}

// Launches request r on slot s.  Memory layout: status | workspace | output.
// The request's memory goes back to the pool on the slot's stream whether or
// not every step was enqueued, so a failed launch leaks nothing.
ecl_status launch(ecl_server* sv, Slot& s, ecl_request& r) {
  const GraphDev& g = sv->graphs[(size_t)r.graph].g;
  const size_t need = request_bytes(r.code, g);
  ECL_CUDA_TRY(cudaMallocAsync(&s.mem, need, s.stream));
  s.bytes = need;
  const ecl_status st = enqueue_request(sv, s, r);
  const cudaError_t fe = cudaFreeAsync(s.mem, s.stream);
  s.mem = nullptr;
  if (st != ECL_OK) return st;
  if (fe != cudaSuccess) {
    set_last_error("cudaFreeAsync", fe);
    return ECL_ERR_CUDA;
  }
  ECL_CUDA_TRY(cudaEventRecord(s.done, s.stream));
  return ECL_OK;
}

}  // namespace
}  // namespace ecl

extern "C" {

ecl_status ecl_server_create(const ecl_server_cfg* cfg, ecl_server** out) {
  using namespace ecl;
  if (!out) return ECL_ERR_INVALID_ARG;
  ecl_server* sv = new ecl_server();
  if (cfg) sv->cfg = *cfg;
  if (sv->cfg.slots <= 0) sv->cfg.slots = 8;
  if (sv->cfg.hbm_budget_bytes == 0) sv->cfg.hbm_budget_bytes = 160ull * 1000 * 1000 * 1000;
  ecl_status st = current_device(&sv->dev);
  if (st != ECL_OK) {
    delete sv;
    return st;
  }
  sv->slots.resize((size_t)sv->cfg.slots);
  for (auto& s : sv->slots) {
    if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&s.hstatus, sizeof(dev::Status)) != cudaSuccess ||
        cudaMallocHost(&s.htotal, sizeof(unsigned long long)) != cudaSuccess) {
      ecl_server_destroy(sv);
      return ECL_ERR_CUDA;
    }
  }
  *out = sv;
  return ECL_OK;
}

void ecl_server_destroy(ecl_server* sv) {
  if (!sv) return;
  for (auto& s : sv->slots) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.stream) cudaStreamDestroy(s.stream);
    if (s.done) cudaEventDestroy(s.done);
    if (s.hstatus) cudaFreeHost(s.hstatus);
    if (s.htotal) cudaFreeHost(s.htotal);
  }
  for (auto& g : sv->graphs) {
    cudaFree(g.nindex);
    cudaFree(g.nlist);
    cudaFree(g.eweight);
  }
  delete sv;
}

ecl_status ecl_server_add_graph(ecl_server* sv, const ecl_graph_view* g, int32_t* id) {
  using namespace ecl;
  using serverimpl::ResidentGraph;
  if (!sv || !g || !id || g->location != ECL_HOST || g->nodes < 1 || g->edges < 0 || !g->nindex) return ECL_ERR_INVALID_ARG;
  ResidentGraph r;
  const size_t nb = sizeof(int) * ((size_t)g->nodes + 1), mb = sizeof(int) * (size_t)(g->edges > 0 ? g->edges : 1);
  r.bytes = nb + mb + (g->eweight ? mb : 0);
  if (sv->resident + r.bytes > sv->cfg.hbm_budget_bytes) return ECL_ERR_OOM;
  if (cudaMalloc(&r.nindex, nb) != cudaSuccess || cudaMalloc(&r.nlist, mb) != cudaSuccess ||
      (g->eweight && cudaMalloc(&r.eweight, mb) != cudaSuccess)) {
    cudaGetLastError();
    cudaFree(r.nindex);
    cudaFree(r.nlist);
    cudaFree(r.eweight);
    return ECL_ERR_OOM;
  }
  ECL_CUDA_TRY(cudaMemcpy(r.nindex, g->nindex, nb, cudaMemcpyHostToDevice));
  if (g->edges) ECL_CUDA_TRY(cudaMemcpy(r.nlist, g->nlist, sizeof(int) * (size_t)g->edges, cudaMemcpyHostToDevice));
  if (g->eweight && g->edges) ECL_CUDA_TRY(cudaMemcpy(r.eweight, g->eweight, sizeof(int) * (size_t)g->edges, cudaMemcpyHostToDevice));
  r.g.n = g->nodes;
  r.g.m = g->edges;
  r.g.nindex = static_cast<int*>(r.nindex);
  r.g.nlist = static_cast<int*>(r.nlist);
  r.g.eweight = static_cast<int*>(r.eweight);
  r.g.flags = g->flags;
  sv->resident += r.bytes;
  *id = (int32_t)sv->graphs.size();
  sv->graphs.push_back(r);
  return ECL_OK;
}

ecl_status ecl_server_run(ecl_server* sv, ecl_request* reqs, int32_t count, ecl_server_stats* stats) {
  using namespace ecl;
  using namespace ecl::serverimpl;
  if (!sv || (count > 0 && !reqs)) return ECL_ERR_INVALID_ARG;
  std::vector<int> order((size_t)count);
  for (int i = 0; i < count; i++) {
    order[(size_t)i] = i;
    ecl_request& r = reqs[i];
    r.status = ECL_OK;
    r.latency_s = r.queue_s = -1.0;
    r.slot = -1;
    r.total_weight = 0;
    if (r.graph < 0 || r.graph >= (int32_t)sv->graphs.size() || r.code < ECL_CC || r.code > ECL_SCC) {
      r.status = ECL_ERR_INVALID_ARG;
    } else if (r.code == ECL_MST && !sv->graphs[(size_t)r.graph].g.eweight) {
      r.status = ECL_ERR_INVALID_ARG;
    } else if (sv->resident + request_bytes(r.code, sv->graphs[(size_t)r.graph].g) > sv->cfg.hbm_budget_bytes) {
      r.status = ECL_ERR_OOM;  // can never fit, even alone
    }
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
  std::vector<int> ready;
  std::vector<double> done_at((size_t)count, -1.0);
  size_t next = 0;
  int finished = 0, failed = 0, in_flight = 0, max_in_flight = 0;
  uint64_t inflight_bytes = 0, peak = sv->resident;
  for (int i = 0; i < count; i++)
    if (reqs[i].status != ECL_OK) {
      finished++;
      failed++;
    }
  const auto t0 = Clock::now();
  auto now_s = [&] { return std::chrono::duration<double>(Clock::now() - t0).count(); };
  double first_arrival = count ? 1e300 : 0.0, last_done = 0.0;
  ecl_status result = ECL_OK;
  while (finished < count) {
    bool progress = false;
    const double now = now_s();
    while (next < order.size() && reqs[order[next]].arrival_s <= now) {
      const int i = order[next++];
      first_arrival = std::min(first_arrival, reqs[i].arrival_s);
      if (reqs[i].status == ECL_OK) ready.push_back(i);
      progress = true;
    }
    // retire finished slots
    for (size_t k = 0; k < sv->slots.size(); k++) {
      Slot& s = sv->slots[k];
      if (s.req < 0) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) continue;
      ecl_request& r = reqs[s.req];
      const double t = now_s();
      r.latency_s = t - r.arrival_s;
      last_done = std::max(last_done, t);
      if (q != cudaSuccess) {
        set_last_error("server request", q);
        r.status = ECL_ERR_CUDA;
        result = ECL_ERR_CUDA;
      } else {
        r.status = s.hstatus->code;
        if (r.code == ECL_MST) r.total_weight = *s.htotal;
      }
      if (r.status != ECL_OK) failed++;
      inflight_bytes -= s.bytes;
      in_flight--;
      finished++;
      s.req = -1;
      progress = true;
    }
    // admit ready requests first-fit into free slots
    for (size_t k = 0; k < sv->slots.size() && !ready.empty(); k++) {
      Slot& s = sv->slots[k];
      if (s.req >= 0) continue;
      auto it = std::find_if(ready.begin(), ready.end(), [&](int i) {
        return sv->resident + inflight_bytes + request_bytes(reqs[i].code, sv->graphs[(size_t)reqs[i].graph].g) <=
               sv->cfg.hbm_budget_bytes;
      });
      if (it == ready.end()) break;
      const int i = *it;
      ready.erase(it);
      ecl_request& r = reqs[i];
      r.queue_s = now_s() - r.arrival_s;
      r.slot = (int32_t)k;
      s.req = i;
      const ecl_status st = launch(sv, s, r);
      if (st != ECL_OK) {
        cudaStreamSynchronize(s.stream);
        cudaGetLastError();
        r.status = st;
        r.latency_s = now_s() - r.arrival_s;
        failed++;
        finished++;
        s.req = -1;
        result = st;
      } else {
        inflight_bytes += s.bytes;
        in_flight++;
        max_in_flight = std::max(max_in_flight, in_flight);
        peak = std::max<uint64_t>(peak, sv->resident + inflight_bytes);
      }
      progress = true;
    }
    if (!progress) {
      // idle: nothing arrived, finished or fit -- wait a little (until the
      // next arrival at most)
      double wait = 20e-6;
      if (in_flight == 0 && ready.empty() && next < order.size()) wait = std::max(0.0, reqs[order[next]].arrival_s - now_s());
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
    }
  }
  if (stats) {
    std::vector<double> lat;
    double sum = 0;
    for (int i = 0; i < count; i++)
      if (reqs[i].status == ECL_OK) {
        lat.push_back(reqs[i].latency_s);
        sum += reqs[i].latency_s;
      }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) { return lat.empty() ? 0.0 : lat[std::min(lat.size() - 1, (size_t)(p * (double)lat.size()))]; };
    stats->completed = count - failed;
    stats->failed = failed;
    stats->makespan_s = (count && last_done > first_arrival) ? last_done - first_arrival : 0.0;
    stats->graphs_per_s = stats->makespan_s > 0 ? (double)stats->completed / stats->makespan_s : 0.0;
    stats->p50_s = pct(0.50);
    stats->p99_s = pct(0.99);
    stats->mean_s = lat.empty() ? 0.0 : sum / (double)lat.size();
    stats->max_in_flight = max_in_flight;
    stats->peak_bytes = peak;
  }
  return result;
}

}  // extern "C"
