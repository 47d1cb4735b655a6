// Host runtime: see runtime.cuh.
#include "runtime.cuh"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

namespace ecl {

std::atomic<uint64_t> g_launches{0};

namespace {
thread_local std::string t_last_error;
std::mutex g_dev_mu;
DeviceInfo g_dev_cache[64];
ecl_tune g_tune{};  // process-wide knobs of the single-graph entry points (under g_dev_mu)
}  // namespace

bool tune_valid(const ecl_tune& t) {
  const bool chunk_ok = t.row_chunk == 0 || (t.row_chunk >= dev::kMinChunk && t.row_chunk <= dev::kMaxChunk &&
                                              (t.row_chunk & (t.row_chunk - 1)) == 0);
  return t.blocks_per_sm >= 0 && t.blocks_per_sm <= 128 && t.mst_light_factor >= 0.f && t.mst_light_factor <= 64.f &&
         t.gc_core_ranks >= 0 && t.gc_core_ranks <= 36864 && t.row_lane_max >= 0 && t.row_lane_max <= 32 && chunk_ok &&
         (t.scc_sweep_batch == 0 || t.scc_sweep_batch == 1 || t.scc_sweep_batch == 2 || t.scc_sweep_batch == 4) &&
         t.gc_poll_ns >= 0 && t.gc_poll_ns <= 4096 && (t.row_vec == 0 || t.row_vec == 1) &&
         (t.gc_pull_blocks >= 0 && t.gc_pull_blocks <= 4) && t.gc_core_ctas >= 0 && t.gc_core_ctas <= 8;
}

void apply_tune(DeviceInfo* d, const ecl_tune& t) {
  d->blocks_per_sm = t.blocks_per_sm;
  d->mst_light_factor = t.mst_light_factor;
  d->gc_core_ranks = t.gc_core_ranks;
  d->row_lane_max = t.row_lane_max;
  d->row_chunk = t.row_chunk;
  d->scc_sweep_batch = t.scc_sweep_batch;
  d->gc_poll_ns = t.gc_poll_ns;
  d->row_vec = t.row_vec;
  d->gc_pull_blocks = t.gc_pull_blocks;
  d->gc_core_ctas = t.gc_core_ctas;
}

void set_last_error(const char* where, cudaError_t e) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s (%d)", where, cudaGetErrorString(e), (int)e);
  t_last_error = buf;
}
void set_last_error_msg(const char* msg) { t_last_error = msg; }

ecl_status current_device(DeviceInfo* info) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_last_error_msg("no CUDA device");
    return ECL_ERR_NO_DEVICE;
  }
  int d = 0;
  ECL_CUDA_TRY(cudaGetDevice(&d));
  if (d < 0 || d >= 64) return ECL_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DeviceInfo& c = g_dev_cache[d];
  if (c.device != d) {
    cudaDeviceProp p;
    ECL_CUDA_TRY(cudaGetDeviceProperties(&p, d));
    c.sms = p.multiProcessorCount;
    c.max_threads_per_sm = p.maxThreadsPerMultiProcessor;
    c.major = p.major;
    c.minor = p.minor;
    c.smem_optin = p.sharedMemPerBlockOptin;
    c.device = d;
    // Workspaces come from the device's default memory pool (cudaMallocAsync).
    // Its default release threshold (0) hands freed memory back to the driver
    // at every synchronisation, so the next large workspace is mapped again;
    // keep freed memory in the pool instead.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, d) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  if (c.major != 10) {
    set_last_error_msg("this library is built for sm_100a (B200) only");
    return ECL_ERR_NO_DEVICE;
  }
  *info = c;
  apply_tune(info, g_tune);
  return ECL_OK;
}

Solve::~Solve() {
  if (!finished_) finish(ECL_ERR_CUDA);
}

ecl_status Solve::begin(const GraphNeeds& needs, size_t ws_bytes) {
  if (!g_ || !opts_) return ECL_ERR_INVALID_ARG;
  if (g_->nodes < 1 || g_->edges < 0) return ECL_ERR_BAD_GRAPH;
  if (!g_->nindex || (g_->edges > 0 && !g_->nlist)) return ECL_ERR_INVALID_ARG;
  if (needs.weights && g_->edges > 0 && !g_->eweight) return ECL_ERR_INVALID_ARG;
  if (g_->location != ECL_HOST && g_->location != ECL_DEVICE) return ECL_ERR_INVALID_ARG;
  n = g_->nodes;
  m = g_->edges;
  stream = static_cast<cudaStream_t>(opts_->stream);

  ecl_status st = current_device(&dev);
  if (st != ECL_OK) return st;

  if (opts_->validate) {
    if (g_->location == ECL_HOST) {
      st = ecl_graph_validate(g_, needs.symmetric, needs.no_self_loops);
    } else {
      std::vector<int32_t> hidx((size_t)n + 1), hl((size_t)m);
      ECL_CUDA_TRY(cudaMemcpyAsync(hidx.data(), g_->nindex, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, stream));
      if (m) ECL_CUDA_TRY(cudaMemcpyAsync(hl.data(), g_->nlist, sizeof(int32_t) * (size_t)m, cudaMemcpyDeviceToHost, stream));
      ECL_CUDA_TRY(cudaStreamSynchronize(stream));
      ecl_graph_view hv = *g_;
      hv.nindex = hidx.data();
      hv.nlist = hl.data();
      hv.location = ECL_HOST;
      st = ecl_graph_validate(&hv, needs.symmetric, needs.no_self_loops);
    }
    if (st != ECL_OK) return st;
  }

  if (g_->location == ECL_HOST) {
    int* d_idx = static_cast<int*>(temp(sizeof(int) * ((size_t)n + 1)));
    int* d_list = static_cast<int*>(temp(sizeof(int) * (size_t)(m > 0 ? m : 1)));
    int* d_w = nullptr;
    if (needs.weights && g_->eweight) d_w = static_cast<int*>(temp(sizeof(int) * (size_t)(m > 0 ? m : 1)));
    if (alloc_failed) return ECL_ERR_OOM;
    ECL_CUDA_TRY(cudaMemcpyAsync(d_idx, g_->nindex, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, stream));
    if (m) ECL_CUDA_TRY(cudaMemcpyAsync(d_list, g_->nlist, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice, stream));
    if (d_w && m) ECL_CUDA_TRY(cudaMemcpyAsync(d_w, g_->eweight, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice, stream));
    nindex = d_idx;
    nlist = d_list;
    eweight = d_w;
  } else {
    nindex = g_->nindex;
    nlist = g_->nlist;
    eweight = needs.weights ? g_->eweight : nullptr;
  }

  const size_t need = ws_bytes + kStatusBytes;
  if (opts_->workspace && opts_->workspace_bytes >= need) {
    ws = static_cast<char*>(opts_->workspace);
  } else {
    ws = static_cast<char*>(temp(need));
    if (alloc_failed) return ECL_ERR_OOM;
  }
  ws_size = need;
  status = reinterpret_cast<dev::Status*>(ws);
  ws += kStatusBytes;
  ECL_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(dev::Status), stream));
  return ECL_OK;
}

void* Solve::temp(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocAsync(&p, bytes ? bytes : 1, stream) != cudaSuccess) {
    cudaGetLastError();
    alloc_failed = true;
    set_last_error_msg("device allocation failed");
    return nullptr;
  }
  temps_.push_back(p);
  return p;
}

void* Solve::output_bytes(void* user, size_t bytes) {
  if (g_->location == ECL_DEVICE) return user;
  void* d = temp(bytes);
  if (d) outs_.push_back(Copy{user, d, bytes});
  return d;
}

void Solve::start_timer() {
  if (!ev0_) {
    cudaEventCreate(&ev0_);
    cudaEventCreate(&ev1_);
  }
  cudaEventRecord(ev0_, stream);
}

void Solve::mark() {
  if (!opts_ || !opts_->detail || marks_.size() >= 8) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, stream);
  marks_.push_back(e);
}

void Solve::stop_timer() {
  cudaEventRecord(ev1_, stream);
  timed_ = true;
}

ecl_status Solve::finish(ecl_status st) {
  finished_ = true;
  dev::Status hs{};
  if (st == ECL_OK && status) {
    for (const Copy& c : outs_) {
      if (c.bytes && cudaMemcpyAsync(c.host, c.dev, c.bytes, cudaMemcpyDeviceToHost, stream) != cudaSuccess) {
        set_last_error("cudaMemcpyAsync(D2H)", cudaGetLastError());
        st = ECL_ERR_CUDA;
      }
    }
    if (cudaMemcpyAsync(&hs, status, sizeof(hs), cudaMemcpyDeviceToHost, stream) != cudaSuccess) st = ECL_ERR_CUDA;
  }
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess && st == ECL_OK) {
    set_last_error("solve", e);
    st = ECL_ERR_CUDA;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess && st == ECL_OK) {
    set_last_error("kernel launch", e);
    st = ECL_ERR_CUDA;
  }
  if (st == ECL_OK && hs.code != 0) st = static_cast<ecl_status>(hs.code);
  if (opts_) {
    opts_->rounds = hs.rounds;
    opts_->elapsed_ms = 0.f;
    opts_->nphases = 0;
    if (timed_ && e == cudaSuccess) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess) opts_->elapsed_ms = ms;
      cudaEvent_t prev = ev0_;
      for (size_t i = 0; i < marks_.size(); i++) {
        float pm = 0.f;
        cudaEventElapsedTime(&pm, prev, marks_[i]);
        opts_->phase_ms[i] = pm;
        prev = marks_[i];
      }
      opts_->nphases = (int32_t)marks_.size();
    }
  }
  for (cudaEvent_t m : marks_) cudaEventDestroy(m);
  marks_.clear();
  for (void* p : temps_) cudaFreeAsync(p, stream);
  temps_.clear();
  outs_.clear();
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  ev0_ = ev1_ = nullptr;
  cudaGetLastError();
  return st;
}

}  // namespace ecl

extern "C" {

int32_t ecl_abi_version(void) { return ECL_B200_ABI_VERSION; }

ecl_status ecl_set_tune(const ecl_tune* t) {
  if (!t || !ecl::tune_valid(*t)) return ECL_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ecl::g_dev_mu);
  ecl::g_tune = *t;
  return ECL_OK;
}

ecl_status ecl_get_tune(ecl_tune* t) {
  if (!t) return ECL_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(ecl::g_dev_mu);
  *t = ecl::g_tune;
  return ECL_OK;
}

const char* ecl_status_string(ecl_status s) {
  switch (s) {
    case ECL_OK: return "ok";
    case ECL_ERR_INVALID_ARG: return "invalid argument";
    case ECL_ERR_BAD_GRAPH: return "bad graph";
    case ECL_ERR_OOM: return "out of memory";
    case ECL_ERR_NO_CONVERGENCE: return "no convergence";
    case ECL_ERR_CUDA: return "CUDA error";
    case ECL_ERR_IO: return "I/O error";
    case ECL_ERR_UNSUPPORTED: return "unsupported input";
    case ECL_ERR_NO_DEVICE: return "no sm_100 device";
  }
  return "unknown status";
}

const char* ecl_last_error(void) { return ecl::t_last_error.c_str(); }

uint64_t ecl_kernel_launches(void) { return ecl::g_launches.load(std::memory_order_relaxed); }

}  // extern "C"
