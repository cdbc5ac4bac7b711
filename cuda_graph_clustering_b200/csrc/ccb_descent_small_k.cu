// Instances and launcher of the K <= 8 descent (ccb_descent_small_k.cuh), in a translation unit of their own
// so that the many template instances compile in parallel with the rest of the library.
#include <cuda_runtime.h>

#include "ccb_descent_cluster.cuh"
#include "ccb_descent_incremental.cuh"
#include "ccb_descent_registers.cuh"
#include "ccb_descent_stream.cuh"
#include "ccb_plans.h"

namespace ccb {
namespace {

template <int K, int T, bool S, bool H = false>
cudaError_t GoStream(const DescentArgs<int16_t>& a, int grid, size_t smem, cudaStream_t st, bool configure) {
  auto kernel = k_descent_stream<K, T, S, H>;
  if (configure) return RaiseDynamicSmem(kernel, smem);
  kernel<<<grid, T, smem, st>>>(a);
  return cudaGetLastError();
}

template <int K, int C>
cudaError_t GoCluster(const DescentArgs<int16_t>& a, int slots, size_t smem, cudaStream_t st, bool configure) {
  auto kernel = k_descent_cluster<K, 1024, C>;
  if (configure) return RaiseDynamicSmem(kernel, smem);
  if (slots <= 0) return cudaSuccess;
  kernel<<<slots * C, 1024, smem, st>>>(a);
  return cudaGetLastError();
}

template <int K, int T, int V, bool R>
cudaError_t GoRegisters(const DescentArgs<int16_t>& a, int grid, size_t smem, cudaStream_t st, bool configure) {
  auto kernel = k_descent_registers<K, T, V, R>;
  if (configure) return RaiseDynamicSmem(kernel, smem);
  kernel<<<grid, T, smem, st>>>(a);
  return cudaGetLastError();
}

template <int K, bool R>
cudaError_t RegistersByShape(int threads, int vpt, const DescentArgs<int16_t>& a, int grid, size_t smem,
                             cudaStream_t st, bool cfg) {
  if (vpt == 16) return GoRegisters<K, 64, 16, R>(a, grid, smem, st, cfg);
  if (vpt == 8) {
    switch (threads) {
      case 128: return GoRegisters<K, 128, 8, R>(a, grid, smem, st, cfg);
      case 256: return GoRegisters<K, 256, 8, R>(a, grid, smem, st, cfg);
      default: return GoRegisters<K, 512, 8, R>(a, grid, smem, st, cfg);
    }
  }
  switch (threads) {
    case 128: return GoRegisters<K, 128, 4, R>(a, grid, smem, st, cfg);
    case 256: return GoRegisters<K, 256, 4, R>(a, grid, smem, st, cfg);
    case 512: return GoRegisters<K, 512, 4, R>(a, grid, smem, st, cfg);
    default: return GoRegisters<K, 1024, 4, R>(a, grid, smem, st, cfg);
  }
}

template <int K>
cudaError_t ByPlacement(const SmallKPlan& p, const DescentArgs<int16_t>& a, int grid, cudaStream_t st, bool cfg) {
  if (p.registers) {
    return p.smem_rows ? RegistersByShape<K, true>(p.threads, p.vpt, a, grid, p.smem_bytes, st, cfg)
                       : RegistersByShape<K, false>(p.threads, p.vpt, a, grid, p.smem_bytes, st, cfg);
  }
  if (p.cluster > 0) {
    switch (p.cluster) {
      case 2: return GoCluster<K, 2>(a, grid, p.smem_bytes, st, cfg);
      case 4: return GoCluster<K, 4>(a, grid, p.smem_bytes, st, cfg);
      default: return GoCluster<K, 8>(a, grid, p.smem_bytes, st, cfg);
    }
  }
  if (p.threads == 512) {
    if (p.smem_state) return GoStream<K, 512, true>(a, grid, p.smem_bytes, st, cfg);
    return p.l2_hints ? GoStream<K, 512, false, true>(a, grid, p.smem_bytes, st, cfg)
                      : GoStream<K, 512, false>(a, grid, p.smem_bytes, st, cfg);
  }
  if (p.smem_state) return GoStream<K, 1024, true>(a, grid, p.smem_bytes, st, cfg);
  return p.l2_hints ? GoStream<K, 1024, false, true>(a, grid, p.smem_bytes, st, cfg)
                    : GoStream<K, 1024, false>(a, grid, p.smem_bytes, st, cfg);
}

template <int T, bool S>
cudaError_t GoIncremental(const DescentArgs<int16_t>& a, int grid, size_t smem, cudaStream_t st, bool configure) {
  auto kernel = k_descent_incremental<T, S>;
  if (configure) return RaiseDynamicSmem(kernel, smem);
  kernel<<<grid, T, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

size_t IncrementalBytes(int k, int ld) { return IncState::Bytes(k, ld); }

template <int T, int V, bool S>
cudaError_t GoIncrementalRegs(const DescentArgs<int16_t>& a, int grid, size_t smem, cudaStream_t st, bool configure) {
  auto kernel = k_descent_incremental_regs<T, V, S, (V >= 16)>;
  if (configure) return RaiseDynamicSmem(kernel, smem);
  kernel<<<grid, T, smem, st>>>(a);
  return cudaGetLastError();
}

size_t IncrementalRegsSmem(int k, int ld, int threads, int vpt, bool counters_in_smem) {
  return (vpt >= 16 ? (size_t)vpt * threads * 12 : 0) + (counters_in_smem ? (size_t)k * ld * 2 : 0);
}

void IncrementalRegsShape(int n, int* threads, int* vpt) {
  if (n <= 1024) {
    *threads = 256, *vpt = 4;
  } else if (n <= 2048) {
    *threads = 512, *vpt = 4;
  } else if (n <= 4096) {
    *threads = 512, *vpt = 8;
  } else if (n <= 8192) {
    *threads = 512, *vpt = 16;
  } else {
    *threads = 512, *vpt = 32;
  }
}

cudaError_t LaunchDescentIncremental(const SmallKPlan& p, const DescentArgs<int16_t>& a, int grid, cudaStream_t st,
                                     bool configure) {
  if (p.registers) {
#define CCB_INC(T, V)                                                                                     \
  if (p.threads == T && p.vpt == V)                                                                       \
    return p.smem_state ? GoIncrementalRegs<T, V, true>(a, grid, p.smem_bytes, st, configure)             \
                        : GoIncrementalRegs<T, V, false>(a, grid, p.smem_bytes, st, configure);
    CCB_INC(256, 4) CCB_INC(512, 4) CCB_INC(512, 8) CCB_INC(512, 16) CCB_INC(512, 32)
#undef CCB_INC
    return cudaErrorInvalidValue;
  }
  switch (p.threads) {
    case 256:
      return p.smem_state ? GoIncremental<256, true>(a, grid, p.smem_bytes, st, configure)
                          : GoIncremental<256, false>(a, grid, p.smem_bytes, st, configure);
    case 512:
      return p.smem_state ? GoIncremental<512, true>(a, grid, p.smem_bytes, st, configure)
                          : GoIncremental<512, false>(a, grid, p.smem_bytes, st, configure);
    default:
      return p.smem_state ? GoIncremental<1024, true>(a, grid, p.smem_bytes, st, configure)
                          : GoIncremental<1024, false>(a, grid, p.smem_bytes, st, configure);
  }
}

cudaError_t LaunchDescentIncrementalWide(const DescentArgs<int32_t>& a, int grid, cudaStream_t st) {
  k_descent_incremental_wide<1024><<<grid, 1024, 0, st>>>(a);
  return cudaGetLastError();
}

size_t SmallKSmem(int k, int n, int pitch, int ld, int threads, bool smem_state, bool smem_rows) {
  (void)pitch;
  (void)threads;
  (void)smem_rows;
  return smem_state ? (size_t)ld * PackedLanes(k) * 2 : 0;
}

int SmallKLanes(int k) { return PackedLanes(k); }

int StreamCluster(int k, int n, size_t limit, size_t* bytes_per_cta) {
  for (int c = 2; c <= 8; c *= 2) {
    const size_t bytes = (size_t)ClusterSpan(n, c) * PackedLanes(k) * 2;
    if (bytes <= limit) {
      *bytes_per_cta = bytes;
      return c;
    }
  }
  return 0;
}

size_t RegistersSmem(int n, int pitch, bool smem_rows) {
  return smem_rows ? ((size_t)n * pitch * 4 + 15) / 16 * 16 : 0;
}

bool RegistersShapeBuilt(int threads, int vpt) {
  return (vpt == 16 && threads == 64) || (vpt == 8 && (threads == 128 || threads == 256 || threads == 512)) ||
         (vpt == 4 && (threads == 128 || threads == 256 || threads == 512 || threads == 1024));
}

cudaError_t LaunchDescentSmallK(const SmallKPlan& p, const DescentArgs<int16_t>& a, int grid, cudaStream_t st,
                                bool configure) {
  switch (p.k) {
    case 2: return ByPlacement<2>(p, a, grid, st, configure);
    case 3: return ByPlacement<3>(p, a, grid, st, configure);
    case 4: return ByPlacement<4>(p, a, grid, st, configure);
    case 5: return ByPlacement<5>(p, a, grid, st, configure);
    case 6: return ByPlacement<6>(p, a, grid, st, configure);
    case 7: return ByPlacement<7>(p, a, grid, st, configure);
    case 8: return ByPlacement<8>(p, a, grid, st, configure);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ccb
