// Launchers of the packed wide descents (k = 2, 3; n > 32767).
#include <cuda_runtime.h>

#include "ccb_descent_wide_packed.cuh"
#include "ccb_plans.h"

namespace ccb {

cudaError_t LaunchDescentWidePacked(const DescentArgs<int32_t>& a, int grid, bool sparse, cudaStream_t st) {
  if (a.k == 2 && sparse) {
    const int words = (a.gr.n + 31) / 32;
    const int per_thread = (words + 1023) / 1024;  // row words per thread
    if (per_thread <= 1) {
      k_descent_wide2_sparse<1024, 1><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 2) {
      k_descent_wide2_sparse<1024, 2><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 4) {
      k_descent_wide2_sparse<1024, 4><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 8) {
      k_descent_wide2_sparse<1024, 8><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 16) {
      k_descent_wide2_sparse<1024, 16><<<grid, 1024, 0, st>>>(a);
    } else {
      k_descent_wide2_sparse<1024, 32><<<grid, 1024, 0, st>>>(a);
    }
  } else if (a.k == 3 && sparse) {
    const int words = (a.gr.n + 31) / 32;
    const int per_thread = (words + 1023) / 1024;
    if (per_thread <= 1) {
      k_descent_wide3_sparse<1024, 1><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 2) {
      k_descent_wide3_sparse<1024, 2><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 4) {
      k_descent_wide3_sparse<1024, 4><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 8) {
      k_descent_wide3_sparse<1024, 8><<<grid, 1024, 0, st>>>(a);
    } else if (per_thread <= 16) {
      k_descent_wide3_sparse<1024, 16><<<grid, 1024, 0, st>>>(a);
    } else {
      k_descent_wide3_sparse<1024, 32><<<grid, 1024, 0, st>>>(a);
    }
  } else if (a.k == 2) {
    k_descent_wide_packed<2, 1024><<<grid, 1024, 0, st>>>(a);
  } else if (a.k == 3) {
    k_descent_wide_packed<3, 1024><<<grid, 1024, 0, st>>>(a);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace ccb
