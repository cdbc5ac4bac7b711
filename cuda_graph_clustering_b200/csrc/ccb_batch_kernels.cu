// Persistent kernels of the batched engine.  A bucket's grid is sized to what stays resident; every block
// claims (instance, slot) items from the bucket's queue and runs the same descent / rebuild body as the
// one-slot-per-block kernels of the plain path, until the queue is empty.  Claims never wait on anything,
// so every block finishes after at most `total` claims.
#include <cuda_runtime.h>

#include "ccb_batch.h"
#include "ccb_descent_incremental.cuh"
#include "ccb_descent_registers.cuh"
#include "ccb_descent_stream.cuh"

namespace ccb {
namespace {

// Next item of the queue for the whole block: instance entry and slot, or false once the queue is empty.
__device__ __forceinline__ bool ClaimItem(const BatchQueue& q, int* s_item, int& entry, int& slot) {
  if (threadIdx.x == 0) *s_item = atomicAdd(q.head, 1);
  __syncthreads();
  const int item = *s_item;
  __syncthreads();
  if (item >= q.total) return false;
  int lo = 0, hi = q.count;  // largest lo with prefix[lo] <= item
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (q.prefix[mid] <= item) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  entry = q.instances[lo];
  slot = item - q.prefix[lo];
  return true;
}

__device__ __forceinline__ DescentArgs<int16_t> CurrentDescent(const BatchEntry& e) {
  DescentArgs<int16_t> a = e.descent;
  a.iteration = a.ctl->iter;
  return a;
}

template <int K, int T, int V, bool R>
__global__ void __launch_bounds__(T, 1) kb_descent_registers(const BatchEntry* __restrict__ entries, BatchQueue q) {
  __shared__ int s_item;
  int entry, slot;
  while (ClaimItem(q, &s_item, entry, slot)) {
    DescentRegisters<K, T, V, R>(CurrentDescent(entries[entry]), slot);
    __syncthreads();
  }
}

template <int K, int T, bool S>
__global__ void __launch_bounds__(T, 1) kb_descent_stream(const BatchEntry* __restrict__ entries, BatchQueue q) {
  __shared__ int s_item;
  int entry, slot;
  while (ClaimItem(q, &s_item, entry, slot)) {
    DescentStream<K, T, S>(CurrentDescent(entries[entry]), slot);
    __syncthreads();
  }
}

// 1024 / T resident blocks per SM fit the register file (the body needs no more than 64 registers).
template <int T, bool S>
__global__ void __launch_bounds__(T, 1024 / T) kb_descent_incremental(const BatchEntry* __restrict__ entries,
                                                                      BatchQueue q) {
  __shared__ int s_item;
  int entry, slot;
  while (ClaimItem(q, &s_item, entry, slot)) {
    DescentIncremental<T, S>(CurrentDescent(entries[entry]), slot);
    __syncthreads();
  }
}

template <int T, int V, bool S>
__global__ void __launch_bounds__(T, 1) kb_descent_incremental_regs(const BatchEntry* __restrict__ entries,
                                                                     BatchQueue q) {
  __shared__ int s_item;
  int entry, slot;
  while (ClaimItem(q, &s_item, entry, slot)) {
    DescentIncrementalRegs<T, V, S, (V >= 16)>(CurrentDescent(entries[entry]), slot);
    __syncthreads();
  }
}

constexpr int kBatchRebuildThreads = 512;

__global__ void __launch_bounds__(kBatchRebuildThreads) kb_rebuild(const BatchEntry* __restrict__ entries,
                                                                    BatchQueue q) {
  __shared__ int s_item;
  int entry, slot;
  while (ClaimItem(q, &s_item, entry, slot)) {
    RebuildArgs<int16_t> a = entries[entry].rebuild;
    a.iteration = a.ctl->iter;
    RebuildBody<int16_t, kBatchRebuildThreads>(a, slot);
    __syncthreads();
  }
}

constexpr int kBatchRecordThreads = 1024;

__global__ void __launch_bounds__(kBatchRecordThreads) kb_record(const BatchEntry* __restrict__ entries) {
  RecordArgs a = entries[blockIdx.x].record;
  a.iteration = a.ctl->iter;
  RecordBody<kBatchRecordThreads>(a);
}

__global__ void kb_advance(const BatchEntry* __restrict__ entries, int count, int32_t* active, int32_t* stops) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  Control* c = entries[i].descent.ctl;
  if (!c->stop) {
    c->iter += 1;
    if (c->iter >= entries[i].iterations) {
      c->stop = 1;
    } else {
      atomicAdd(active, 1);
    }
  }
  if (stops != nullptr) stops[i] = c->stop;
}

template <typename Kernel>
cudaError_t Run(Kernel kernel, const BatchShape& s, const BatchEntry* e, const BatchQueue& q, cudaStream_t st,
                bool configure) {
  if (configure) return RaiseDynamicSmem(kernel, s.smem_bytes);
  if (q.total == 0 || s.grid <= 0) return cudaSuccess;
  kernel<<<s.grid, s.threads, s.smem_bytes, st>>>(e, q);
  return cudaGetLastError();
}

template <typename Kernel>
int Occupancy(Kernel kernel, const BatchShape& s) {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, s.threads, s.smem_bytes) != cudaSuccess) return 1;
  return blocks > 0 ? blocks : 1;
}

// Visits the kernel instance of a shape.
template <typename F>
cudaError_t WithKernel(const BatchShape& s, F&& f) {
#define CCB_REG(K, T, V)                                                                              \
  if (s.kind == kBatchRegisters && s.k == K && s.threads == T && s.vpt == V)                         \
    return s.smem ? f(kb_descent_registers<K, T, V, true>) : f(kb_descent_registers<K, T, V, false>);
#define CCB_REG_K(K) CCB_REG(K, 128, 4) CCB_REG(K, 256, 4) CCB_REG(K, 512, 4) CCB_REG(K, 1024, 4)
  CCB_REG_K(2) CCB_REG_K(3) CCB_REG_K(4) CCB_REG_K(5) CCB_REG_K(6) CCB_REG_K(7) CCB_REG_K(8)
#undef CCB_REG_K
#undef CCB_REG
#define CCB_STREAM(K) \
  if (s.kind == kBatchStream && s.k == K) return s.smem ? f(kb_descent_stream<K, 1024, true>) : f(kb_descent_stream<K, 1024, false>);
  CCB_STREAM(2) CCB_STREAM(3) CCB_STREAM(4) CCB_STREAM(5) CCB_STREAM(6) CCB_STREAM(7) CCB_STREAM(8)
#undef CCB_STREAM
  if (s.kind == kBatchIncrementalRegs) {
#define CCB_INC(T, V) \
  if (s.threads == T && s.vpt == V) \
    return s.smem ? f(kb_descent_incremental_regs<T, V, true>) : f(kb_descent_incremental_regs<T, V, false>);
    CCB_INC(256, 4) CCB_INC(512, 4) CCB_INC(512, 8) CCB_INC(512, 16) CCB_INC(512, 32)
#undef CCB_INC
    return cudaErrorInvalidValue;
  }
  if (s.kind == kBatchIncremental) {
    switch (s.threads) {
      case 256: return s.smem ? f(kb_descent_incremental<256, true>) : f(kb_descent_incremental<256, false>);
      case 512: return s.smem ? f(kb_descent_incremental<512, true>) : f(kb_descent_incremental<512, false>);
      default: return s.smem ? f(kb_descent_incremental<1024, true>) : f(kb_descent_incremental<1024, false>);
    }
  }
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t LaunchBatchDescent(const BatchShape& shape, const BatchEntry* entries, const BatchQueue& queue,
                               cudaStream_t stream, bool configure) {
  return WithKernel(shape, [&](auto kernel) { return Run(kernel, shape, entries, queue, stream, configure); });
}

int BatchDescentBlocksPerSm(const BatchShape& shape) {
  int blocks = 1;
  WithKernel(shape, [&](auto kernel) {
    RaiseDynamicSmem(kernel, shape.smem_bytes);
    blocks = Occupancy(kernel, shape);
    return cudaSuccess;
  });
  return blocks;
}

cudaError_t LaunchBatchRebuild(const BatchEntry* entries, const BatchQueue& queue, int grid, cudaStream_t stream) {
  if (queue.total == 0) return cudaSuccess;
  kb_rebuild<<<grid, kBatchRebuildThreads, 0, stream>>>(entries, queue);
  return cudaGetLastError();
}

cudaError_t LaunchBatchRecord(const BatchEntry* entries, int count, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  kb_record<<<count, kBatchRecordThreads, 0, stream>>>(entries);
  return cudaGetLastError();
}

cudaError_t LaunchBatchAdvance(const BatchEntry* entries, int count, int32_t* active, int32_t* stops,
                               cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  kb_advance<<<(count + 255) / 256, 256, 0, stream>>>(entries, count, active, stops);
  return cudaGetLastError();
}

}  // namespace ccb
