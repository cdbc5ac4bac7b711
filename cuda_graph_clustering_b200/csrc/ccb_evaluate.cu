// Device recount of labelings: objective f, cluster sizes and G = A*Z for a batch of labelings of one graph.
// This is the GPU form of the reference's post-solve recount ObjectiveBitwise (src/cc_pbils_cpu.cpp:25-53,
// run by the CLI at include/cc_cli.hpp:337-343) and of State::Rebuild (src/cc_pbils_cpu.cpp:74-95).
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "ccb.h"
#include "ccb_device.cuh"
#include "ccb_error.h"

namespace ccb {
namespace {

constexpr int kEvalThreads = 512;
constexpr int kEvalChunk = 8;

// One block per labeling.  Phase 1 packs a bit mask per cluster with warp ballots into `masks`
// ([labeling][k][words], scratch) and counts cluster sizes; every mask word is written before it is
// read, so the scratch needs no clearing.  Phase 2 gives each warp whole rows: lanes stride over the
// row's words and count the bits shared with each cluster's mask, reduced across the warp in hardware.
// A label outside [0, k) marks the labeling invalid: its f is written as -1.
__global__ void __launch_bounds__(kEvalThreads)
    k_evaluate(const uint32_t* __restrict__ bits, int n, int words, int pitch, long long edges, int k,
               const int32_t* __restrict__ all_labels, uint32_t* __restrict__ masks, int64_t* __restrict__ f_out,
               int32_t* __restrict__ sizes_out, int32_t* __restrict__ g_out) {
  constexpr int kWarps = kEvalThreads / kWarp;
  __shared__ int s_sizes[kMaxK];
  __shared__ int s_bad;
  __shared__ long long s_sum[kWarps];
  const int sol = blockIdx.x;
  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int warp = tid / kWarp;
  const int32_t* labels = all_labels + static_cast<size_t>(sol) * n;
  uint32_t* my_masks = masks + static_cast<size_t>(sol) * k * words;
  for (int c = tid; c < k; c += kEvalThreads) s_sizes[c] = 0;
  if (tid == 0) s_bad = 0;
  __syncthreads();

  for (int w = warp; w < words; w += kWarps) {
    const int v = w * kWarp + lane;
    const int l = v < n ? labels[v] : -1;
    if (v < n && (l < 0 || l >= k)) s_bad = 1;
    for (int c = 0; c < k; ++c) {
      const uint32_t m = __ballot_sync(kAllLanes, l == c);
      if (lane == (c % kWarp)) {
        my_masks[static_cast<size_t>(c) * words + w] = m;
        if (m) atomicAdd(&s_sizes[c], __popc(m));
      }
    }
  }
  __syncthreads();

  long long intra_twice = 0;
  for (int v = warp; v < n; v += kWarps) {
    const uint32_t* row = bits + static_cast<size_t>(v) * pitch;
    const int own = labels[v];
    for (int c0 = 0; c0 < k; c0 += kEvalChunk) {
      int acc[kEvalChunk];
#pragma unroll
      for (int i = 0; i < kEvalChunk; ++i) acc[i] = 0;
      for (int w = lane; w < words; w += kWarp) {
        const uint32_t a = __ldg(row + w);
#pragma unroll
        for (int i = 0; i < kEvalChunk; ++i)
          if (c0 + i < k) acc[i] += __popc(a & my_masks[static_cast<size_t>(c0 + i) * words + w]);
      }
#pragma unroll
      for (int i = 0; i < kEvalChunk; ++i) {
        if (c0 + i < k) {
          const int total = static_cast<int>(__reduce_add_sync(kAllLanes, static_cast<unsigned>(acc[i])));
          if (lane == 0) {
            if (g_out != nullptr) g_out[(static_cast<size_t>(sol) * k + c0 + i) * n + v] = total;
            if (own == c0 + i) intra_twice += total;
          }
        }
      }
    }
  }
  const long long sum = BlockSum<kWarps>(intra_twice, s_sum);
  if (tid == 0) {
    long long pairs = 0;
    for (int c = 0; c < k; ++c) pairs += static_cast<long long>(s_sizes[c]) * (s_sizes[c] - 1) / 2;
    f_out[sol] = s_bad ? -1 : edges + pairs - sum;
  }
  if (sizes_out != nullptr) {
    for (int c = tid; c < k; c += kEvalThreads) sizes_out[static_cast<size_t>(sol) * k + c] = s_sizes[c];
  }
}

const char* CheckEvaluateArgs(const uint32_t* bits, uint32_t n, uint32_t words_per_row, int32_t k, int32_t count,
                              const int32_t* labels, const int64_t* f_out) {
  if (k < 1 || k > CCB_MAX_CLUSTERS) return "k must be in [1, 64]";
  if (count < 0) return "count must be >= 0";
  if (n > (uint32_t)CCB_MAX_VERTICES_WIDE) return "n exceeds 1048576, the range of the packed move";
  if (n > 0 && words_per_row < (n + 31) / 32) return "words_per_row < ceil(n / 32)";
  if (count > 0 && n > 0 && (bits == nullptr || labels == nullptr)) return "null bitset or labels";
  if (count > 0 && f_out == nullptr) return "null f_out";
  return nullptr;
}

int Report(int status, const char* message) {
  SetLastError(message);
  return status;
}

}  // namespace
}  // namespace ccb

using namespace ccb;

extern "C" {

int ccb_evaluate_labelings(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges, int32_t k,
                           int32_t count, const int32_t* labels, int64_t* f_out, int32_t* sizes_out, int32_t* g_out,
                           void* stream) {
  if (const char* why = CheckEvaluateArgs(bits, n, words_per_row, k, count, labels, f_out)) {
    return Report(CCB_ERR_INVALID, why);
  }
  if (count == 0) return Report(CCB_OK, "");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int words = (int)((n + 31) / 32);
  const size_t mask_bytes = sizeof(uint32_t) * (size_t)count * k * words;
  uint32_t* masks = nullptr;
  cudaError_t e = cudaSuccess;
  if (mask_bytes > 0) {
    e = cudaMallocAsync(&masks, mask_bytes, st);
    if (e != cudaSuccess) return Report(CCB_ERR_DEVICE_MEMORY, cudaGetErrorString(e));
  }
  k_evaluate<<<count, kEvalThreads, 0, st>>>(bits, (int)n, words, (int)words_per_row, (long long)edges, k, labels,
                                             masks, f_out, sizes_out, g_out);
  e = cudaGetLastError();
  if (masks) cudaFreeAsync(masks, st);
  if (e != cudaSuccess) return Report(CCB_ERR_CUDA, cudaGetErrorString(e));
  return Report(CCB_OK, "");
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Allocation-free recount.
//
// Some callers cannot allocate device memory when they call in: a host application whose device
// memory is already reserved by its own pool allocator (a framework that took the free memory up
// front, where cudaMalloc fails or fragments that pool), or a latency-critical loop that must not pay
// cudaMalloc / cudaFree, which can synchronise the whole device.  For them the mask scratch of
// k_evaluate lives in a fixed array in device memory, loaded with the library: every GPU that loads
// libccb.so holds these kNoAllocMaskWords words (4 MiB) until the process exits.
//
// The array's host-side name is only a stand-in, not a device address, so the entry point looks the
// address up with cudaGetSymbolAddress once per device (on its first call on that device, with that
// device current) and passes it to the kernel.  Make that first call before any stream capture.
// Under CUDA's default lazy module loading the array is only allocated when that first call loads this
// module onto the device, so a caller that reserves the device's free memory for its own pool must make
// the first call before it does; a call with count = 0 does exactly this set-up and nothing else.  (With
// CUDA_MODULE_LOADING=EAGER the array is allocated when the library is loaded.)  The address is kept for
// the life of the process: after cudaDeviceReset on a device the module is loaded afresh and may sit
// elsewhere, so the entry point must not be used across a device reset.
// Every call shares the one array and finds the last call's contents there.  k_evaluate writes every
// mask word it later reads, so nothing needs clearing between calls; but two calls whose kernels
// overlap on the GPU (different streams, or different host threads) race on the array, so callers
// must order their calls.
// ------------------------------------------------------------------------------------------------
#include <mutex>

namespace ccb {
namespace {

constexpr size_t kNoAllocMaskWords = size_t(1) << 20;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_masks[kNoAllocMaskWords];

std::mutex g_noalloc_mutex;
uint32_t* g_noalloc_address[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_masks on the current device, looked up once per device.
cudaError_t NoAllocScratch(uint32_t** out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_address[device] == nullptr) {
    void* address = nullptr;
    e = cudaGetSymbolAddress(&address, g_noalloc_masks);
    if (e != cudaSuccess) return e;
    g_noalloc_address[device] = static_cast<uint32_t*>(address);
  }
  *out = g_noalloc_address[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace ccb

extern "C" {

int ccb_evaluate_labelings_noalloc(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges,
                                   int32_t k, int32_t count, const int32_t* labels, int64_t* f_out,
                                   int32_t* sizes_out, int32_t* g_out, void* stream) {
  if (const char* why = CheckEvaluateArgs(bits, n, words_per_row, k, count, labels, f_out)) {
    return Report(CCB_ERR_INVALID, why);
  }
  const size_t words = (n + 31) / 32;
  if ((size_t)count * (size_t)k * words > kNoAllocMaskWords) {
    return Report(CCB_ERR_INVALID,
                  "ccb_evaluate_labelings_noalloc: count * k * ceil(n / 32) exceeds the 1048576 mask words of "
                  "its static scratch; split the batch or use ccb_evaluate_labelings");
  }
  uint32_t* masks = nullptr;
  cudaError_t e = NoAllocScratch(&masks);  // also the whole of a count = 0 call: the per-device set-up
  if (e != cudaSuccess) return Report(CCB_ERR_CUDA, cudaGetErrorString(e));
  if (count == 0) return Report(CCB_OK, "");
  k_evaluate<<<count, kEvalThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      bits, (int)n, (int)words, (int)words_per_row, (long long)edges, k, labels, masks, f_out, sizes_out, g_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return Report(CCB_ERR_CUDA, cudaGetErrorString(e));
  return Report(CCB_OK, "");
}

}  // extern "C"
