// Launchers of the packed wide descents (k = 2, 3; n > 32767).
#include <cuda_runtime.h>

#include "ccb_descent_wide_packed.cuh"
#include "ccb_plans.h"

namespace ccb {

cudaError_t LaunchDescentWidePacked(const DescentArgs<int32_t>& a, int grid, cudaStream_t st) {
  if (a.k == 2) {
    k_descent_wide_packed<2, 1024><<<grid, 1024, 0, st>>>(a);
  } else if (a.k == 3) {
    k_descent_wide_packed<3, 1024><<<grid, 1024, 0, st>>>(a);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace ccb
