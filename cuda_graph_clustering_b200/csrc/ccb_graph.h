// Device-resident graph shared by the translation units of libccb: allocation, degree count, generators.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "ccb_device.cuh"

struct ccb_graph {
  int device = 0;
  int n = 0;
  int words = 0;  // ceil(n / 32)
  int pitch = 0;  // words per row in memory (multiple of 4)
  int64_t edges = 0;
  uint32_t* bits = nullptr;
  int32_t* degrees = nullptr;

  ccb::GraphView View() const { return ccb::GraphView{bits, degrees, n, words, pitch, edges}; }
  ~ccb_graph() {
    if (bits) cudaFree(bits);
    if (degrees) cudaFree(degrees);
  }
};

namespace ccb {
// Zeroed rows of n vertices (16-byte pitch) and a degree array, after a device-memory budget check.
ccb_graph* AllocateGraph(uint32_t n, cudaStream_t stream);
// Counts degrees once the rows are filled, then waits for the stream.
void FinishGraph(ccb_graph& g, cudaStream_t stream);
}  // namespace ccb
