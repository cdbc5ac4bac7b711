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

// ---- flow engine ---------------------------------------------------------------------------------------
constexpr uint32_t kFlowNone = 0x80000000u;  // slot field of an epoch with nothing to claim (finished, withheld)

__device__ __forceinline__ int32_t LoadAcquire(const int32_t* p) {
  int32_t v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long LoadAcquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// The claim / finish protocol.  A slot's results are written by its block; thread 0 then fences (release,
// cumulative over the block's writes ordered by the barrier) and counts the slot done.  The block that counts
// the last slot fences (acquire) before reading the other slots' results, writes the epoch's conclusion, resets
// the done count, fences and publishes the next epoch with one atomic exchange of the claim word.  A claimer's
// atomic add returns the word it incremented: a slot field below the population is a valid claim of that epoch
// (the epoch may be newer than the one it read first), anything else is not; after the add thread 0 fences
// (acquire) and the block barrier extends that to every thread.  An epoch is concluded only after all of its
// slots were claimed and completed, so a late add to a concluded epoch finds its slot field at or above the
// population.  Nothing here waits on anything but the bucket's own running blocks.
template <int T, typename Descent>
__device__ __forceinline__ void FlowLoop(const BatchEntry* __restrict__ entries, FlowState* flow, const FlowBucket& b,
                                         Descent&& descent) {
  __shared__ int s_entry, s_slot, s_flag;
  __shared__ unsigned long long s_epoch;
  unsigned long long idle_since = 0;
  if (threadIdx.x == 0) atomicAdd(b.remaining + 2, 1);
  for (;;) {
    if (threadIdx.x == 0) {
      s_entry = -1;
      s_flag = 0;
      for (int i = 0; i < b.count; ++i) {
        const int e = b.members[i];
        FlowState* f = flow + e;
        const uint32_t pop = static_cast<uint32_t>(entries[e].descent.population);
        if (LoadAcquire(&f->finished)) continue;
        const unsigned long long w = LoadAcquire(&f->claim);
        if (static_cast<uint32_t>(w) >= pop) continue;
        const unsigned long long old = atomicAdd(&f->claim, 1ull);
        if (static_cast<uint32_t>(old) < pop) {
          s_entry = e;
          s_slot = static_cast<int>(static_cast<uint32_t>(old));
          s_epoch = old >> 32;
          break;
        }
      }
      if (s_entry >= 0) {
        __threadfence();
        idle_since = 0;
      } else if (LoadAcquire(b.remaining) <= 0 || LoadAcquire(b.error) != 0) {
        s_flag = 1;  // the bucket is done (or gave up): leave
      } else {
        // more blocks run than the unfinished instances have slots: a surplus block is never needed again and
        // leaves, freeing its SM for the other buckets.  The decision is taken on the count after this block's
        // own decrement, so blocks that look at the same time cannot all leave: as many stay as there are slots
        if (LoadAcquire(b.remaining + 2) > LoadAcquire(b.remaining + 1)) {
          if (atomicSub(b.remaining + 2, 1) - 1 >= LoadAcquire(b.remaining + 1)) {
            s_flag = 2;  // left (already counted out)
          } else {
            atomicAdd(b.remaining + 2, 1);  // still needed: stay
          }
        }
      }
      if (s_entry < 0 && s_flag == 0) {
        const unsigned long long now = GlobalTimerNs();
        if (idle_since == 0) {
          idle_since = now;
        } else if (now - idle_since > b.idle_limit_ns) {
          atomicExch(b.error, kErrorWaitTimeout);
          s_flag = 1;
        }
        if (!s_flag) __nanosleep(2000);
      }
    }
    __syncthreads();
    if (s_entry < 0) {
      if (s_flag) {
        if (threadIdx.x == 0 && s_flag == 1) atomicSub(b.remaining + 2, 1);
        break;
      }
      continue;
    }
    const int e = s_entry, slot = s_slot;
    const unsigned long long epoch = s_epoch;
    const int iteration = static_cast<int>(epoch >> 1);
    const BatchEntry& E = entries[e];
    if ((epoch & 1) == 0) {
      DescentArgs<int16_t> a = E.descent;
      a.iteration = iteration;
      descent(a, slot);
    } else {
      RebuildArgs<int16_t> a = E.rebuild;
      a.iteration = iteration;
      RebuildBody<int16_t, T>(a, slot);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      s_flag = atomicAdd(&flow[e].done, 1) == E.descent.population - 1;
      if (s_flag) __threadfence();
    }
    __syncthreads();
    if (!s_flag) continue;
    Control* c = E.descent.ctl;
    if ((epoch & 1) == 0) {
      RecordArgs r = E.record;
      r.iteration = iteration;
      RecordBody<T>(r);  // sets c->stop on the stall or time rule
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      bool stop = c->stop != 0;
      if ((epoch & 1) == 1) {
        c->iter = iteration + 1;
        if (iteration + 1 >= E.iterations) {
          c->stop = 1;
          stop = true;
        }
      }
      flow[e].done = 0;
      if (stop) {
        flow[e].t_done_ns = GlobalTimerNs();
        flow[e].finished = 1;
        __threadfence();
        atomicExch(&flow[e].claim, ((epoch + 1) << 32) | kFlowNone);
        atomicSub(b.remaining + 1, E.descent.population);
        atomicSub(b.remaining, 1);
      } else {
        __threadfence();
        atomicExch(&flow[e].claim, (epoch + 1) << 32);
      }
    }
    __syncthreads();
  }
}

template <int K, int T, int V, bool R>
__global__ void __launch_bounds__(T, 1) kf_registers(const BatchEntry* __restrict__ entries, FlowState* flow,
                                                     FlowBucket b) {
  FlowLoop<T>(entries, flow, b, [](const DescentArgs<int16_t>& a, int slot) { DescentRegisters<K, T, V, R>(a, slot); });
}

template <int K, int T, bool S>
__global__ void __launch_bounds__(T, 1) kf_stream(const BatchEntry* __restrict__ entries, FlowState* flow,
                                                  FlowBucket b) {
  FlowLoop<T>(entries, flow, b, [](const DescentArgs<int16_t>& a, int slot) { DescentStream<K, T, S>(a, slot); });
}

template <int T, bool S>
__global__ void __launch_bounds__(T, 1024 / T) kf_incremental(const BatchEntry* __restrict__ entries, FlowState* flow,
                                                              FlowBucket b) {
  FlowLoop<T>(entries, flow, b, [](const DescentArgs<int16_t>& a, int slot) { DescentIncremental<T, S>(a, slot); });
}

template <int T, int V, bool S>
__global__ void __launch_bounds__(T, 1) kf_incremental_regs(const BatchEntry* __restrict__ entries, FlowState* flow,
                                                            FlowBucket b) {
  FlowLoop<T>(entries, flow, b, [](const DescentArgs<int16_t>& a, int slot) {
    DescentIncrementalRegs<T, V, S, (V >= 16)>(a, slot);
  });
}

__global__ void kb_flow_init(const BatchEntry* __restrict__ entries, FlowState* flow, FlowBucket b,
                             const int32_t* withheld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.count) return;
  const int e = b.members[i];
  FlowState& f = flow[e];
  const bool stopped = entries[e].descent.ctl->stop != 0;
  f.done = 0;
  f.t_done_ns = 0;
  f.finished = stopped ? 1 : 0;
  f.claim = (stopped || (withheld != nullptr && withheld[e])) ? kFlowNone : 0ull;
  if (!stopped) {
    atomicAdd(b.remaining, 1);
    atomicAdd(b.remaining + 1, entries[e].descent.population);
  }
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

// Visits the kernel instance of a shape: the lock-step queue kernel (kb_*) or, with kFlow, the flow kernel (kf_*).
template <bool kFlow, typename F>
cudaError_t WithKernel(const BatchShape& s, F&& f) {
#define CCB_PICK(KB, KF) \
  if constexpr (kFlow) { return f(KF); } else { return f(KB); }
#define CCB_REG(K, T, V)                                                                                \
  if (s.kind == kBatchRegisters && s.k == K && s.threads == T && s.vpt == V) {                         \
    if (s.smem) { CCB_PICK((kb_descent_registers<K, T, V, true>), (kf_registers<K, T, V, true>)) }     \
    CCB_PICK((kb_descent_registers<K, T, V, false>), (kf_registers<K, T, V, false>))                   \
  }
#define CCB_REG_K(K) CCB_REG(K, 128, 4) CCB_REG(K, 256, 4) CCB_REG(K, 512, 4) CCB_REG(K, 1024, 4)
  CCB_REG_K(2) CCB_REG_K(3) CCB_REG_K(4) CCB_REG_K(5) CCB_REG_K(6) CCB_REG_K(7) CCB_REG_K(8)
#undef CCB_REG_K
#undef CCB_REG
#define CCB_STREAM(K)                                                                                   \
  if (s.kind == kBatchStream && s.k == K) {                                                             \
    if (s.smem) { CCB_PICK((kb_descent_stream<K, 1024, true>), (kf_stream<K, 1024, true>)) }            \
    CCB_PICK((kb_descent_stream<K, 1024, false>), (kf_stream<K, 1024, false>))                          \
  }
  CCB_STREAM(2) CCB_STREAM(3) CCB_STREAM(4) CCB_STREAM(5) CCB_STREAM(6) CCB_STREAM(7) CCB_STREAM(8)
#undef CCB_STREAM
  if (s.kind == kBatchIncrementalRegs) {
#define CCB_INC(T, V)                                                                                   \
  if (s.threads == T && s.vpt == V) {                                                                   \
    if (s.smem) { CCB_PICK((kb_descent_incremental_regs<T, V, true>), (kf_incremental_regs<T, V, true>)) } \
    CCB_PICK((kb_descent_incremental_regs<T, V, false>), (kf_incremental_regs<T, V, false>))            \
  }
    CCB_INC(256, 4) CCB_INC(512, 4) CCB_INC(512, 8) CCB_INC(512, 16) CCB_INC(512, 32)
#undef CCB_INC
    return cudaErrorInvalidValue;
  }
  if (s.kind == kBatchIncremental) {
#define CCB_INCG(T)                                                                                     \
  if (s.threads == T || T == 1024) {                                                                    \
    if (s.smem) { CCB_PICK((kb_descent_incremental<T, true>), (kf_incremental<T, true>)) }              \
    CCB_PICK((kb_descent_incremental<T, false>), (kf_incremental<T, false>))                            \
  }
    CCB_INCG(256) CCB_INCG(512) CCB_INCG(1024)
#undef CCB_INCG
  }
#undef CCB_PICK
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t LaunchBatchDescent(const BatchShape& shape, const BatchEntry* entries, const BatchQueue& queue,
                               cudaStream_t stream, bool configure) {
  return WithKernel<false>(shape, [&](auto kernel) { return Run(kernel, shape, entries, queue, stream, configure); });
}

int BatchDescentBlocksPerSm(const BatchShape& shape) {
  int blocks = 1;
  WithKernel<false>(shape, [&](auto kernel) {
    RaiseDynamicSmem(kernel, shape.smem_bytes);
    blocks = Occupancy(kernel, shape);
    return cudaSuccess;
  });
  return blocks;
}

cudaError_t LaunchFlowInit(const BatchEntry* entries, FlowState* flow, const FlowBucket& bucket,
                           const int32_t* withheld, cudaStream_t stream) {
  if (bucket.count == 0) return cudaSuccess;
  kb_flow_init<<<(bucket.count + 255) / 256, 256, 0, stream>>>(entries, flow, bucket, withheld);
  return cudaGetLastError();
}

cudaError_t LaunchBatchFlow(const BatchShape& shape, const BatchEntry* entries, FlowState* flow,
                            const FlowBucket& bucket, cudaStream_t stream, bool configure) {
  return WithKernel<true>(shape, [&](auto kernel) -> cudaError_t {
    if (configure) return RaiseDynamicSmem(kernel, shape.smem_bytes);
    if (bucket.count == 0 || shape.grid <= 0) return cudaSuccess;
    kernel<<<shape.grid, shape.threads, shape.smem_bytes, stream>>>(entries, flow, bucket);
    return cudaGetLastError();
  });
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
