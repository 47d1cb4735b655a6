// Host runtime shared by the solver entry points: argument checks, staging of
// host-resident CSR arrays, workspace carving, launch accounting, timing and
// the read-back of the device status word.
#pragma once

#include <algorithm>

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "common.cuh"
#include "csr_bins.cuh"
#include "ecl_b200.h"

namespace ecl {

// Process-wide count of kernel launches made by this library.
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// Records a CUDA failure message for ecl_last_error().
void set_last_error(const char* where, cudaError_t e);
void set_last_error_msg(const char* msg);

#define ECL_CUDA_TRY(call)                          \
  do {                                              \
    cudaError_t ecl_e_ = (call);                    \
    if (ecl_e_ != cudaSuccess) {                    \
      ::ecl::set_last_error(#call, ecl_e_);         \
      return ECL_ERR_CUDA;                          \
    }                                               \
  } while (0)

// Launch + accounting.  Kernel launch errors surface at the next CUDA call.
#define ECL_LAUNCH(kernel, grid, block, smem, stream, ...)        \
  do {                                                            \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);   \
    ::ecl::count_launch();                                        \
  } while (0)

// One thread-block cluster of `ctas` CTAs (its CTAs share distributed shared
// memory), through cudaLaunchKernelEx and the cluster-dimension attribute.
template <typename... KArgs, typename... Args>
cudaError_t launch_cluster(void (*kernel)(KArgs...), int ctas, int block, size_t smem, cudaStream_t stream,
                           Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ctas);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
  count_launch();
  return e;
}

// Cooperative (all blocks co-resident) launch through cudaLaunchKernelEx and
// the cooperative launch attribute, which stream capture turns into a
// cooperative CUDA-graph kernel node.
template <typename... KArgs, typename... Args>
cudaError_t launch_cooperative(void (*kernel)(KArgs...), int grid, int block, cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
  count_launch();
  return e;
}

constexpr int kGridBlocksPerSm = 64;

struct DeviceInfo {
  int device = -1;
  int sms = 0;
  int max_threads_per_sm = 0;
  int major = 0, minor = 0;
  size_t smem_optin = 0;
  // Tunable launch knobs (0 = default), set by the batched engine's autotuner.
  int blocks_per_sm = 0;
  float mst_light_factor = 0.f;
  int gc_core_ranks = 0;  // GC: ranks coloured in one CTA's shared memory (0 = default)
  int row_lane_max = 0;   // degree bins of the CSR scans (0 = each scan's default)
  int row_chunk = 0;
  int scc_sweep_batch = 0;  // SCC: edges per lane in flight in a sweep (0 = default)
  int gc_poll_ns = 0;       // GC pull: longest back-off of a long row's polls, ns (0 = default)
  int row_vec = 0;          // CSR scans: 1 = warp rows read in 16-byte quads where aligned
  int gc_pull_blocks = 0;   // GC pull: blocks per SM, 1..4 (0 = 2)
  int gc_core_ctas = 0;     // GC core: CTAs of its cluster, 1..8 (0 = 2)
  // Grid of a grid-stride kernel with `tpb` threads per block: by default
  // every SM filled to its thread limit.
  // Grid of the grid-stride kernels: blocks_per_sm blocks of 256 threads per
  // SM (scaled for other block sizes), 64 by default -- eight times what fits
  // at once.  A power-law graph's long rows sit in a few vertex groups, and
  // with more, smaller blocks the groups are dealt finer and the SMs that
  // finish early take new blocks: at R-MAT-22 the CSR scans ran 15-27 %
  // faster with 64 blocks per SM than with 8 (the suite 11.4 -> 10.6 ms).
  // A small graph gets no more blocks than it has work for -- a thread per
  // vertex, or per 8 CSR entries -- so concurrent solves of small graphs (the
  // request server) do not queue behind thousands of empty blocks.
  int grid_blocks(int tpb, long long n, long long m) const {
    const int per = blocks_per_sm > 0 ? blocks_per_sm : kGridBlocksPerSm;
    const long long full = (long long)sms * (per * 256 / tpb > 0 ? per * 256 / tpb : 1);
    const long long work = (std::max(n, m / 8) + tpb - 1) / tpb;
    return (int)std::max(1LL, std::min(full, work));
  }
};
// Properties of the current device (cached per device id), with the
// process-wide knobs of ecl_set_tune applied.
ecl_status current_device(DeviceInfo* info);
// Range check of a knob set, and its application to a DeviceInfo.
bool tune_valid(const ecl_tune& t);
void apply_tune(DeviceInfo* d, const ecl_tune& t);

// Degree bins of a scan: the knobs of `d` where set, else the scan's default.
inline dev::Bins bins_of(const DeviceInfo& d, dev::Bins dflt) {
  return dev::Bins{d.row_lane_max > 0 ? d.row_lane_max : dflt.lane, d.row_chunk > 0 ? d.row_chunk : dflt.chunk};
}

// Workspace carving: the same sequence of take() calls sizes a workspace
// (base == nullptr) and then hands out 256-byte-aligned sub-buffers.
struct Carve {
  char* base = nullptr;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
  size_t bytes() const { return (off + 255) & ~size_t(255); }
};

// Requirements a solver places on its input graph.
struct GraphNeeds {
  bool weights = false;      // eweight must be non-NULL
  bool symmetric = false;    // checked only when opts->validate
  bool no_self_loops = false;  // checked only when opts->validate
};

// One solve: stages inputs/outputs and owns temporaries until finish().
class Solve {
 public:
  Solve(const ecl_graph_view* g, ecl_opts* opts) : g_(g), opts_(opts) {}
  ~Solve();

  // Checks arguments, validates (if asked), stages the CSR on the device and
  // provides `ws_bytes` of workspace.  The device Status block is placed at
  // the start of the workspace and zeroed.
  ecl_status begin(const GraphNeeds& needs, size_t ws_bytes);

  // Device pointer through which the solver writes an output of `count`
  // elements: the caller's pointer for device-resident graphs, else a
  // temporary that finish() copies back to `user`.
  template <class T>
  T* output(T* user, size_t count) {
    return static_cast<T*>(output_bytes(user, count * sizeof(T)));
  }
  void* output_bytes(void* user, size_t bytes);
  // Device scratch outside the workspace (freed by finish()).
  void* temp(size_t bytes);

  void start_timer();
  // Ends a kernel phase (only recorded when opts->detail is set).
  void mark();
  void stop_timer();
  // Copies outputs back, synchronises, folds the device status into the
  // return code and releases temporaries.
  ecl_status finish(ecl_status st = ECL_OK);

  int n = 0, m = 0;
  const int* nindex = nullptr;
  const int* nlist = nullptr;
  const int* eweight = nullptr;
  cudaStream_t stream = nullptr;
  char* ws = nullptr;            // workspace base (Status block first)
  size_t ws_size = 0;
  dev::Status* status = nullptr;
  DeviceInfo dev;
  bool alloc_failed = false;

 private:
  const ecl_graph_view* g_;
  ecl_opts* opts_;
  struct Copy {
    void* host;
    void* dev;
    size_t bytes;
  };
  std::vector<Copy> outs_;
  std::vector<void*> temps_;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  std::vector<cudaEvent_t> marks_;
  bool timed_ = false;
  bool finished_ = false;
};

// Offset of the first usable byte of a workspace after the Status block.
constexpr size_t kStatusBytes = 256;

}  // namespace ecl
