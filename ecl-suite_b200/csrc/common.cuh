// Device-side building blocks shared by every solver.
//
// Race-freedom.  The reference removes data races by routing every access to
// state that another thread may write concurrently through relaxed
// cuda::atomic<T> loads/stores (library/ECLatomic.h:45-55), which are
// system-scope.  Here the same rule is kept with cuda::atomic_ref at DEVICE
// scope (no host or peer-GPU thread ever touches solver state while a kernel
// runs), with explicit memory orders: relaxed for the monotone fixpoint state,
// acquire/release where a flag or counter publishes data.  Read-only inputs
// (nindex, nlist, eweight) are never written during a solve and use plain
// read-only loads.
#pragma once

#include <cuda/atomic>
#include <cuda_runtime.h>

#include <cstdint>

namespace ecl {
namespace dev {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

template <typename T>
using aref = cuda::atomic_ref<T, cuda::thread_scope_device>;

template <typename T>
__device__ __forceinline__ T ld(const T* p) {
  return aref<T>(*const_cast<T*>(p)).load(cuda::memory_order_relaxed);
}
template <typename T>
__device__ __forceinline__ T ld_acquire(const T* p) {
  return aref<T>(*const_cast<T*>(p)).load(cuda::memory_order_acquire);
}
template <typename T>
__device__ __forceinline__ void st(T* p, T v) {
  aref<T>(*p).store(v, cuda::memory_order_relaxed);
}
template <typename T>
__device__ __forceinline__ void st_release(T* p, T v) {
  aref<T>(*p).store(v, cuda::memory_order_release);
}
// Compare-and-swap; returns the value found (== expected on success).
template <typename T>
__device__ __forceinline__ T cas(T* p, T expected, T desired) {
  aref<T>(*p).compare_exchange_strong(expected, desired, cuda::memory_order_relaxed);
  return expected;
}
template <typename T>
__device__ __forceinline__ T fetch_add(T* p, T v) {
  return aref<T>(*p).fetch_add(v, cuda::memory_order_relaxed);
}
template <typename T>
__device__ __forceinline__ T fetch_min(T* p, T v) {
  return aref<T>(*p).fetch_min(v, cuda::memory_order_relaxed);
}
template <typename T>
__device__ __forceinline__ T fetch_max(T* p, T v) {
  return aref<T>(*p).fetch_max(v, cuda::memory_order_relaxed);
}
template <typename T>
__device__ __forceinline__ T fetch_or(T* p, T v) {
  return aref<T>(*p).fetch_or(v, cuda::memory_order_relaxed);
}
template <typename T>
__device__ __forceinline__ T fetch_and(T* p, T v) {
  return aref<T>(*p).fetch_and(v, cuda::memory_order_relaxed);
}

// Read-only input loads (never written during a solve).
__device__ __forceinline__ int ldg(const int* p) { return __ldg(p); }

// Device status block, one per solve, in the workspace.  Kernels report
// failures here instead of trapping; the host reads it after the solve.
struct Status {
  int code;      // ecl_status value, 0 = OK
  int detail;    // solver-specific detail (e.g. the vertex that stalled)
  int rounds;    // fixpoint rounds used
  int pad;
};

__device__ __forceinline__ void raise(Status* s, int code, int detail) {
  if (cas(&s->code, 0, code) == 0) st(&s->detail, detail);
}

// The reference's integer hash (ECL-MIS-atomic.cu:109-114 and
// ECL-GC-atomic.cu:70-75; the published 0x45d9f3b multiply-xorshift hash).
__host__ __device__ __forceinline__ unsigned int ecl_hash(unsigned int val) {
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  return (val >> 16) ^ val;
}

}  // namespace dev
}  // namespace ecl
