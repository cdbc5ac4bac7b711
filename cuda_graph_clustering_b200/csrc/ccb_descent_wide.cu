// Launchers of the packed wide descents (k = 2, 3; n > 32767).
#include <cuda_runtime.h>

#include "ccb_descent_wide_packed.cuh"
#include "ccb_plans.h"

namespace ccb {

namespace {

template <int W, bool kSmem16>
cudaError_t GoWide2Sparse(const DescentArgs<int32_t>& a, int grid, cudaStream_t st) {
  auto kernel = k_descent_wide2_sparse<1024, W, kSmem16>;
  size_t smem = 0;
  if (kSmem16) {
    smem = Wide2Smem16Bytes(a.gr.n);
    const cudaError_t e = RaiseDynamicSmem(kernel, smem);
    if (e != cudaSuccess) return e;
  }
  if (grid > 0) kernel<<<grid, 1024, smem, st>>>(a);
  return cudaGetLastError();
}

template <bool kSmem16>
cudaError_t Wide2Sparse(const DescentArgs<int32_t>& a, int grid, cudaStream_t st) {
  const int words = (a.gr.n + 31) / 32;
  const int per_thread = (words + 1023) / 1024;  // row words per thread
  if (per_thread <= 1) return GoWide2Sparse<1, kSmem16>(a, grid, st);
  if (per_thread <= 2) return GoWide2Sparse<2, kSmem16>(a, grid, st);
  if (per_thread <= 4) return GoWide2Sparse<4, kSmem16>(a, grid, st);
  if constexpr (!kSmem16) {
    if (per_thread <= 8) return GoWide2Sparse<8, false>(a, grid, st);
    if (per_thread <= 16) return GoWide2Sparse<16, false>(a, grid, st);
    return GoWide2Sparse<32, false>(a, grid, st);
  }
  return cudaErrorInvalidValue;  // a shared-memory state this large does not fit
}

template <int W, bool kSmem26>
cudaError_t GoWide3Sparse(const DescentArgs<int32_t>& a, int grid, cudaStream_t st) {
  auto kernel = k_descent_wide3_sparse<1024, W, kSmem26>;
  size_t smem = 0;
  if (kSmem26) {
    smem = Wide3Smem26Bytes(a.gr.n);
    const cudaError_t e = RaiseDynamicSmem(kernel, smem);
    if (e != cudaSuccess) return e;
  }
  if (grid > 0) kernel<<<grid, 1024, smem, st>>>(a);
  return cudaGetLastError();
}

template <bool kSmem26>
cudaError_t Wide3Sparse(const DescentArgs<int32_t>& a, int grid, cudaStream_t st) {
  const int words = (a.gr.n + 31) / 32;
  const int per_thread = (words + 1023) / 1024;
  if (per_thread <= 1) return GoWide3Sparse<1, kSmem26>(a, grid, st);
  if (per_thread <= 2) return GoWide3Sparse<2, kSmem26>(a, grid, st);
  if (per_thread <= 4) return GoWide3Sparse<4, kSmem26>(a, grid, st);
  if constexpr (!kSmem26) {
    if (per_thread <= 8) return GoWide3Sparse<8, false>(a, grid, st);
    if (per_thread <= 16) return GoWide3Sparse<16, false>(a, grid, st);
    return GoWide3Sparse<32, false>(a, grid, st);
  }
  return cudaErrorInvalidValue;  // a shared-memory state this large does not fit
}

}  // namespace

size_t Wide2Smem16Bytes(int n) { return ((size_t)n * 2 + 15) / 16 * 16; }
size_t Wide3Smem26Bytes(int n) { return (size_t)((n + 31) / 32) * 104 + 16; }  // 26 words per row word

cudaError_t LaunchDescentWidePacked(const DescentArgs<int32_t>& a, int grid, bool sparse, bool smem16,
                                    cudaStream_t st) {
  if (a.k == 2 && sparse) {
    return smem16 ? Wide2Sparse<true>(a, grid, st) : Wide2Sparse<false>(a, grid, st);
  } else if (a.k == 3 && sparse) {
    return smem16 ? Wide3Sparse<true>(a, grid, st) : Wide3Sparse<false>(a, grid, st);
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
