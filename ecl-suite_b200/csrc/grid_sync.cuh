// Grid-wide barrier for cooperative (co-resident) launches, with a bounded
// wait: a barrier that does not complete within the spin budget records
// ECL_ERR_NO_CONVERGENCE in the status block and every block returns, so a
// wait can never hang the GPU.
#pragma once

#include "common.cuh"
#include "ecl_b200.h"

namespace ecl {
namespace dev {

struct GridBarrier {
  unsigned count;
  unsigned gen;
  unsigned pad[62];
};

// Returns false when the barrier timed out or an error was raised; callers
// then leave the kernel.
__device__ __forceinline__ bool grid_sync(GridBarrier* b, Status* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = ld_acquire(&b->gen);
    __threadfence();
    if (aref<unsigned>(b->count).fetch_add(1u, cuda::memory_order_acq_rel) == gridDim.x - 1) {
      st(&b->count, 0u);
      st_release(&b->gen, g + 1);
    } else {
      unsigned spins = 0;
      while (ld_acquire(&b->gen) == g) {
        if (++spins > (1u << 26)) {  // ~seconds with the back-off below
          raise(status, ECL_ERR_NO_CONVERGENCE, -1);
          ok = 0;
          break;
        }
        // an error anywhere ends the wait; read every 64th spin, as every
        // waiting block polling one more word would crowd its L2 slice
        if ((spins & 63u) == 0 && ld(&status->code) != 0) {
          ok = 0;
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    if (ld(&status->code) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

}  // namespace dev
}  // namespace ecl
