// Batched execution of many independent PBILS instances: device-side instance table, work queues and the
// persistent kernels that drain them (ccb_batch_kernels.cu), driven by the host engine in ccb_solver.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "ccb_kernels.cuh"

namespace ccb {

// Launch state of one instance, resident in device memory.  The iteration fields of the argument structs
// are ignored: every batched kernel reads the instance's current iteration from its control block.
struct BatchEntry {
  DescentArgs<int16_t> descent;
  RebuildArgs<int16_t> rebuild;  // perturb (or copy) mode of the instance
  RecordArgs record;             // iteration mode of the instance
  int32_t iterations;            // iteration limit of the instance
  int32_t pad;
};

// One work list: the (instance, slot) items of a set of instances, drained through an atomic counter.
struct BatchQueue {
  const int32_t* instances;  // entry index of each listed instance, in queue order
  const int32_t* prefix;     // first item of each listed instance; count + 1 entries
  int32_t count;
  int32_t total;             // prefix[count]
  int32_t* head;             // next unclaimed item (reset to 0 before every phase)
};

enum BatchKind : int { kBatchRegisters = 0, kBatchStream = 1, kBatchIncremental = 2, kBatchIncrementalRegs = 3 };

// Kernel instance of one descent bucket and its persistent grid.
struct BatchShape {
  int kind = kBatchRegisters;
  int k = 0;            // compile-time K of the register and streamed forms
  int threads = 256;
  int vpt = 4;          // register form
  bool smem = false;    // register form: bitset in shared memory; streamed / incremental: state in shared memory
  size_t smem_bytes = 0;
  int blocks_per_sm = 0;  // tuned resident slots per SM (0: the occupancy limit)
  int max_slots = 0;      // tuned cap on slots running at once (0: none)
  int grid = 0;
};

cudaError_t LaunchBatchDescent(const BatchShape& shape, const BatchEntry* entries, const BatchQueue& queue,
                               cudaStream_t stream, bool configure);
// Occupancy of the bucket's kernel (blocks per SM at its shared memory), for sizing the persistent grid.
int BatchDescentBlocksPerSm(const BatchShape& shape);
cudaError_t LaunchBatchRebuild(const BatchEntry* entries, const BatchQueue& queue, int grid, cudaStream_t stream);
cudaError_t LaunchBatchRecord(const BatchEntry* entries, int count, cudaStream_t stream);
// Advances every running instance to its next iteration, stops those at their limit, counts the rest, and
// (stops non-null) writes every instance's stop flag.
cudaError_t LaunchBatchAdvance(const BatchEntry* entries, int count, int32_t* active, int32_t* stops,
                               cudaStream_t stream);

}  // namespace ccb
