// Device-side data views, control block and warp/block primitives of the PBILS pipeline.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "ccb_streams.cuh"

namespace ccb {

constexpr int kWarp = 32;
constexpr unsigned kAllLanes = 0xffffffffu;
constexpr int kMaxK = 64;  // largest cluster bound (cc_gpu.hpp:10)

// Per-solve control block in device memory.  Every kernel of an iteration reads `stop` first and
// returns at once when it is set, so an early stop needs no host round trip.
struct Control {
  int32_t stop;             // set by the record kernel when the stall or time limit is reached
  int32_t iterations_done;  // Progress::Next count (cc_pbils.hpp:69-78)
  int32_t stall;            // iterations since the record last improved
  int32_t have_record;      // a record exists (the first offer always takes)
  int64_t record_f;         // best objective so far
  unsigned long long moves; // accepted local-search moves, summed over all descents
  unsigned long long t0_ns; // %globaltimer at solve start, for the device-side time limit
  int32_t record_slot;      // slot the record last came from
  int32_t error;            // kErrorMoveBound or kErrorWaitTimeout (0: none)
  int32_t iter;             // current iteration of a batched instance (the plain path passes it as argument)
  int32_t pad;
};

// Values of Control::error.
constexpr int32_t kErrorMoveBound = 1;    // a descent exceeded its move bound (inconsistent state)
constexpr int32_t kErrorWaitTimeout = 2;  // a bounded wait on a kernel's own pipeline barriers gave up

// One line of the --verbose progress log, written by the record kernel.
struct TraceEntry {
  int64_t record;
  int32_t stall;
  int32_t pad;
  unsigned long long t_ns;
};

// Adjacency bitset: row v is `pitch` uint32 words (pitch a multiple of 4, so rows start 16-byte
// aligned); bit u of row v is set iff {u, v} is an edge; pad bits are zero.
struct GraphView {
  const uint32_t* bits;
  const int32_t* degrees;
  int n;
  int words;  // meaningful words per row, ceil(n / 32)
  int pitch;  // words per row in memory
  int64_t edges;
};

// A population: labels (1 byte each) and G (cluster-major) share the leading dimension ld, a
// multiple of 32 entries; sizes have kpad entries per slot.
template <typename GainT>
struct PopView {
  uint8_t* labels;  // [slot][ld]
  GainT* g;         // [slot][k][ld]
  int32_t* sizes;   // [slot][kpad]
  int64_t* f;       // [slot]
};

__device__ __forceinline__ unsigned long long GlobalTimerNs() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t WarpMin(uint32_t key) { return __reduce_min_sync(kAllLanes, key); }

// 64-bit minimum in two 32-bit hardware reductions: high halves first, then the low halves of the
// lanes that hold the smallest high half.
__device__ __forceinline__ unsigned long long WarpMin(unsigned long long key) {
  const uint32_t hi = __reduce_min_sync(kAllLanes, static_cast<uint32_t>(key >> 32));
  const uint32_t lo =
      __reduce_min_sync(kAllLanes, static_cast<uint32_t>(key >> 32) == hi ? static_cast<uint32_t>(key) : ~0u);
  return (static_cast<unsigned long long>(hi) << 32) | lo;
}

template <typename Key>
struct KeyTraits;
template <>
struct KeyTraits<uint32_t> {
  static constexpr uint32_t kNone = ~0u;
};
template <>
struct KeyTraits<unsigned long long> {
  static constexpr unsigned long long kNone = ~0ull;
};

// A candidate move as a sortable key: the gain (offset to be positive) above the vertex.  Smaller key
// = smaller gain, then smaller vertex, which is the reference's scan order (cc_pbils_cpu.cpp:99-118);
// the target cluster rides along as payload because each vertex offers only its own best target.
template <typename Key>
__device__ __forceinline__ Key PackMove(int delta, int vertex, int bits) {
  return (static_cast<Key>(static_cast<uint32_t>(delta + (1 << bits))) << bits) | static_cast<Key>(vertex);
}
template <typename Key>
__device__ __forceinline__ int MoveVertex(Key key, int bits) {
  return static_cast<int>(key & ((static_cast<Key>(1) << bits) - 1));
}
template <typename Key>
__device__ __forceinline__ int MoveDelta(Key key, int bits) {
  return static_cast<int>(key >> bits) - (1 << bits);
}

template <typename Key>
struct MoveRecord {
  Key key;
  uint32_t payload;  // from | to << 8
};

// Minimum key over the block with its payload, one barrier.  Warps reduce their keys in hardware; the
// lane holding the warp minimum publishes (key, payload) into this move's half of a double buffer;
// after the barrier every warp folds the published records itself.  A warp can run at most one move
// ahead of another (the next barrier stops it), so two halves suffice.
template <typename Key, int kWarps>
__device__ __forceinline__ MoveRecord<Key> BlockArgMin(Key key, uint32_t payload, MoveRecord<Key>* half) {
  const int lane = threadIdx.x % kWarp;
  const Key m = WarpMin(key);
  if (key == m && (m != KeyTraits<Key>::kNone || lane == 0)) half[threadIdx.x / kWarp] = MoveRecord<Key>{m, payload};
  __syncthreads();
  MoveRecord<Key> r{KeyTraits<Key>::kNone, 0u};
  if (lane < kWarps) r = half[lane];
  const Key best = WarpMin(r.key);
  const unsigned owners = __ballot_sync(kAllLanes, r.key == best);
  const uint32_t pay = __shfl_sync(kAllLanes, r.payload, __ffs(owners) - 1);
  return MoveRecord<Key>{best, pay};
}

// Sum over the block, valid in every thread; `scratch` holds kWarps entries and is reused after the
// trailing barrier.
template <int kWarps>
__device__ __forceinline__ long long BlockSum(long long v, long long* scratch) {
  for (int o = kWarp / 2; o > 0; o /= 2) v += __shfl_xor_sync(kAllLanes, v, o);
  if (threadIdx.x % kWarp == 0) scratch[threadIdx.x / kWarp] = v;
  __syncthreads();
  long long s = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) s += scratch[w];
  __syncthreads();
  return s;
}

// Raises a kernel's dynamic shared-memory limit to at least `bytes`, never lowers it: several solvers (and
// batches) share one kernel instance, each with its own need, so the limit must cover the largest.
template <typename Kernel>
inline cudaError_t RaiseDynamicSmem(Kernel kernel, size_t bytes) {
  cudaFuncAttributes attr;
  cudaError_t e = cudaFuncGetAttributes(&attr, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)attr.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

__device__ __forceinline__ int Bit(const uint32_t* row, int u) { return (row[u >> 5] >> (u & 31)) & 1; }

// Arguments of the descent kernel (passed by value).
template <typename GainT>
struct DescentArgs {
  GraphView gr;
  PopView<GainT> cur;   // population the tournament draws from (read only)
  PopView<GainT> next;  // labels and f written here; g used as scratch by the global-state form
  Control* ctl;
  int k;
  int kpad;
  int ld;
  int key_bits;         // bit width of n: the vertex field of a move key
  int population;       // slots in cur (tournament range)
  int tournament;       // 0: slot s descends from cur[s] (Neighborhood), else tournament size
  int iteration;
  uint64_t select_stream;
};


}  // namespace ccb
