// Launch plans shared between the solver and the separately compiled descent instances.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "ccb_device.cuh"

namespace ccb {

// Descent specialised for 2 <= k <= 8 on the narrow path (ccb_descent_small_k.cuh).
struct SmallKPlan {
  int k = 0;
  int threads = 256;
  bool registers = false;   // whole state in registers (ccb_descent_registers.cuh), n <= vpt * threads
  int vpt = 4;              // vertices per thread of the register form (4 or 8)
  bool smem_state = false;  // packed G + labels in shared memory (else the slot's rows of `next`)
  bool smem_rows = false;   // whole bitset in shared memory
  size_t smem_bytes = 0;
  int cluster = 0;          // streamed form whose state does not fit one CTA: CTAs of the cluster holding it
  bool l2_hints = false;    // streamed form from global memory: state loads/stores evict_last, rows evict_first
};
// The smallest cluster (2, 4 or 8 CTAs) whose shares of the packed state fit `limit` bytes of shared memory per
// CTA, with its bytes per CTA; 0 if none.
int StreamCluster(int k, int n, size_t limit, size_t* bytes_per_cta);

size_t SmallKSmem(int k, int n, int pitch, int ld, int threads, bool smem_state, bool smem_rows);
int SmallKLanes(int k);
size_t RegistersSmem(int n, int pitch, bool smem_rows);
bool RegistersShapeBuilt(int threads, int vpt);
// Incremental descent for 9 <= k <= 64 (ccb_descent_incremental.cuh): SmallKPlan fields threads,
// smem_state and smem_bytes apply; k is the runtime cluster count.
size_t IncrementalBytes(int k, int ld);
// Threads and vertices per thread of the register-cached incremental form (n <= 16384).
void IncrementalRegsShape(int n, int* threads, int* vpt);
// Its dynamic shared memory: the cached keys (vpt >= 16) and, optionally, the counters.
size_t IncrementalRegsSmem(int k, int ld, int threads, int vpt, bool counters_in_smem);
cudaError_t LaunchDescentIncremental(const SmallKPlan& plan, const DescentArgs<int16_t>& args, int grid,
                                     cudaStream_t stream, bool configure);
// Incremental descent on the wide population (int32 G, 32767 < n <= 65536, 2 <= k <= 64): 1024 threads,
// state in global memory (IncrementalBytes per slot), no dynamic shared memory.
cudaError_t LaunchDescentIncrementalWide(const DescentArgs<int32_t>& args, int grid, cudaStream_t stream);
// Packed wide descent (k = 2 or 3, int32 population G, n > 32767): 1024 threads, one 4- or 8-byte word per
// vertex in the slot's rows of `next`, no dynamic shared memory.
// With `sparse`: the degree-proportional forms (per-thread best vertex of each cluster, k = 2, or of each
// (cluster, target) class, k = 3).
// With `smem16` the sparse forms keep the slot's words in shared memory: k = 2 as int16 (Wide2Smem16Bytes(n)
// bytes, every degree below 16384), k = 3 as 26-bit records (Wide3Smem26Bytes(n) bytes, every degree below 2048).
cudaError_t LaunchDescentWidePacked(const DescentArgs<int32_t>& args, int grid, bool sparse, bool smem16,
                                    cudaStream_t stream);
size_t Wide2Smem16Bytes(int n);
size_t Wide3Smem26Bytes(int n);
cudaError_t LaunchDescentSmallK(const SmallKPlan& plan, const DescentArgs<int16_t>& args, int grid,
                                cudaStream_t stream, bool configure);

}  // namespace ccb
