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

// ---- flow engine: per-instance progress ----------------------------------------------------------------
// One persistent kernel per bucket runs every iteration of the bucket's instances.  Each instance moves
// through epochs e = 2 * iteration + phase (phase 0: descents, phase 1: perturbation + rebuild); a block claims
// the next slot of the heaviest instance that has one, runs it, and the block that completes an epoch's last
// slot finishes the epoch for the instance: after the descents the record (and stop rule), after the rebuilds
// the iteration count, then publishes the next epoch.  No instance waits for another.
struct FlowState {
  unsigned long long claim;  // (epoch << 32) | next slot of the epoch; slot field >= population: none left
  int32_t done;              // slots of the epoch completed
  int32_t finished;          // the instance stopped: its record is final
  unsigned long long t_done_ns;  // %globaltimer when it stopped
};

struct FlowBucket {
  const int32_t* members;    // entry indices, heaviest first
  int32_t count;
  int32_t* remaining;        // [0] unfinished members (the kernel ends at 0), [1] their slots, [2] running blocks
  int32_t* error;            // kErrorWaitTimeout when a block found no work for idle_limit_ns
  unsigned long long idle_limit_ns;
};

// Flow states of a bucket's members from their control blocks; `withheld` (may be null) marks instances whose
// work is never published (a host-side fault injection for the bounded idle wait).
cudaError_t LaunchFlowInit(const BatchEntry* entries, FlowState* flow, const FlowBucket& bucket,
                           const int32_t* withheld, cudaStream_t stream);
cudaError_t LaunchBatchFlow(const BatchShape& shape, const BatchEntry* entries, FlowState* flow,
                            const FlowBucket& bucket, cudaStream_t stream, bool configure);
// Occupancy of the bucket's kernel (blocks per SM at its shared memory), for sizing the persistent grid.
int BatchDescentBlocksPerSm(const BatchShape& shape);
cudaError_t LaunchBatchRebuild(const BatchEntry* entries, const BatchQueue& queue, int grid, cudaStream_t stream);
cudaError_t LaunchBatchRecord(const BatchEntry* entries, int count, cudaStream_t stream);
// Advances every running instance to its next iteration, stops those at their limit, counts the rest, and
// (stops non-null) writes every instance's stop flag.
cudaError_t LaunchBatchAdvance(const BatchEntry* entries, int count, int32_t* active, int32_t* stops,
                               cudaStream_t stream);

}  // namespace ccb
