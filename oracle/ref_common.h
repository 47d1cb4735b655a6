// Shared glue for the ref_*.cu harnesses -- TEST/BASELINE INFRASTRUCTURE ONLY.
//
// Each ref_<code>.cu includes one race-free reference source file unchanged,
// where it lies under the reference checkout (-I points there), and exports C
// entry points that run the reference's own kernels or CPU routines.  The
// reference headers define non-static, non-inline functions (ECLgraph.h:49-102,
// ECLatomic.h:57-75) and every file has its own main(); these symbols
// get per-file names through #defines placed before the #include, so the
// six files link into one library.
#pragma once
#include <cuda_runtime.h>

struct RefTimer {
  cudaEvent_t a, b;
  RefTimer() { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, 0); }
  float stop() { cudaEventRecord(b, 0); cudaEventSynchronize(b); float ms = 0; cudaEventElapsedTime(&ms, a, b); cudaEventDestroy(a); cudaEventDestroy(b); return ms; }
};
