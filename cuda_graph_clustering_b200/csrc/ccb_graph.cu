// Device graphs: allocation, degrees, and generation on the device.
//
// Generation reproduces the host generators bit for bit (Graph::ErdosRenyi, src/cc_graph.cpp:168-177, and
// this project's planted partition): both draw pair by pair from one splitmix64 stream in the order
// (i ascending, j < i ascending), and splitmix64 jumps ahead in closed form, the state after t draws being
// seed + t * gamma.  Pair (i, j), j < i, is pair number i(i-1)/2 + j; the Erdős–Rényi graph uses its draw
// number t, the planted graph draws 2t (edge) and 2t + 1 (flip).  A warp computes one 32 x 32 tile of the
// lower triangle, one row word per lane, and writes the mirrored tile of the upper triangle from 32 warp
// ballots, so every pair is drawn once.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <numeric>
#include <vector>

#include "ccb.h"
#include "ccb_graph.h"
#include "ccb_streams.cuh"
#include "ccb_util.h"

namespace ccb {
namespace {

constexpr int kGenWarps = 8;

__global__ void k_graph_degrees(const uint32_t* __restrict__ bits, int n, int words, int pitch, int32_t* degrees) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const uint32_t* row = bits + static_cast<size_t>(v) * pitch;
  int d = 0;
  for (int w = 0; w < words; ++w) d += __popc(row[w]);
  degrees[v] = d;
}

// Unit draw number t (0-based) of the stream that starts at state s0.
__device__ __forceinline__ float UnitAt(uint64_t s0, uint64_t t) {
  const uint64_t z = Mix64(s0 + (t + 1) * kGamma);
  return static_cast<float>(static_cast<uint32_t>(z >> 32) >> 8) * (1.0f / 16777216.0f);
}

// kind 0: Erdős–Rényi with p_in; kind 1: planted (community[], p_in / p_out, flip).
__global__ void __launch_bounds__(kGenWarps * 32) k_generate(uint32_t* __restrict__ bits, int n, int pitch, int kind,
                                                            uint64_t s0, double p_in, double p_out, double flip,
                                                            const int32_t* __restrict__ community,
                                                            unsigned long long* edges) {
  const int tiles = (n + 31) / 32;
  const long long tile = static_cast<long long>(blockIdx.x) * kGenWarps + threadIdx.x / 32;
  const long long total = static_cast<long long>(tiles) * (tiles + 1) / 2;
  if (tile >= total) return;
  // tile -> (ti, tj), tj <= ti, row-major over the lower triangle
  int ti = static_cast<int>((sqrt(8.0 * static_cast<double>(tile) + 1.0) - 1.0) / 2.0);
  while (static_cast<long long>(ti) * (ti + 1) / 2 > tile) --ti;
  while (static_cast<long long>(ti + 1) * (ti + 2) / 2 <= tile) ++ti;
  const int tj = static_cast<int>(tile - static_cast<long long>(ti) * (ti + 1) / 2);
  const int lane = threadIdx.x % 32;
  const int i = ti * 32 + lane;
  uint32_t word = 0;
  if (i < n) {
    const uint64_t base = static_cast<uint64_t>(i) * (i - 1) / 2;
    const int ci = kind == 1 ? community[i] : 0;
    for (int b = 0; b < 32; ++b) {
      const int j = tj * 32 + b;
      if (j >= i || j >= n) break;
      const uint64_t t = base + static_cast<uint64_t>(j);
      bool e;
      if (kind == 0) {
        e = static_cast<double>(UnitAt(s0, t)) < p_in;
      } else {
        const double p = ci == community[j] ? p_in : p_out;
        e = (static_cast<double>(UnitAt(s0, 2 * t)) < p) != (static_cast<double>(UnitAt(s0, 2 * t + 1)) < flip);
      }
      word |= static_cast<uint32_t>(e) << b;
    }
  }
  const unsigned cnt = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(__popc(word)));
  if (lane == 0 && cnt) atomicAdd(edges, static_cast<unsigned long long>(cnt));
  // mirrored tile: lane c receives bit c of every row of this tile
  uint32_t mirror = 0;
  for (int c = 0; c < 32; ++c) {
    const uint32_t m = __ballot_sync(0xffffffffu, (word >> c) & 1u);
    if (lane == c) mirror = m;
  }
  if (ti == tj) {
    if (i < n) bits[static_cast<size_t>(i) * pitch + tj] = word | mirror;
  } else {
    if (i < n) bits[static_cast<size_t>(i) * pitch + tj] = word;
    const int j = tj * 32 + lane;
    if (j < n) bits[static_cast<size_t>(j) * pitch + ti] = mirror;
  }
}

ccb_graph* Generate(uint32_t n, int kind, uint64_t seed, double p_in, double p_out, double flip,
                    const std::vector<int32_t>& community, cudaStream_t st) {
  std::unique_ptr<ccb_graph> g(AllocateGraph(n, st));
  if (n > 0) {
    int32_t* d_comm = nullptr;
    unsigned long long* d_edges = nullptr;
    CCB_CUDA(cudaMalloc(&d_edges, sizeof(unsigned long long)));
    CCB_CUDA(cudaMemsetAsync(d_edges, 0, sizeof(unsigned long long), st));
    if (kind == 1) {
      CCB_CUDA(cudaMalloc(&d_comm, n * sizeof(int32_t)));
      CCB_CUDA(cudaMemcpyAsync(d_comm, community.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    }
    const uint64_t s0 = StreamSeed(seed, kind == 0 ? kErdosRenyiTag : kPlantedTag, kind == 0 ? 0 : 3);
    const long long tiles = (n + 31) / 32;
    const long long total = tiles * (tiles + 1) / 2;
    const long long blocks = (total + kGenWarps - 1) / kGenWarps;
    k_generate<<<(unsigned)blocks, kGenWarps * 32, 0, st>>>(g->bits, (int)n, g->pitch, kind, s0, p_in, p_out, flip,
                                                          d_comm, d_edges);
    CCB_CUDA(cudaGetLastError());
    unsigned long long edges = 0;
    CCB_CUDA(cudaMemcpyAsync(&edges, d_edges, sizeof(edges), cudaMemcpyDeviceToHost, st));
    CCB_CUDA(cudaStreamSynchronize(st));
    g->edges = (int64_t)edges;
    cudaFree(d_edges);
    if (d_comm) cudaFree(d_comm);
  }
  FinishGraph(*g, st);
  return g.release();
}

}  // namespace

ccb_graph* AllocateGraph(uint32_t n, cudaStream_t stream) {
  if (n > (uint32_t)CCB_MAX_VERTICES_WIDE) {
    Fail(CCB_ERR_INVALID, "n exceeds " + std::to_string(CCB_MAX_VERTICES_WIDE) + ", the range of the packed move");
  }
  std::unique_ptr<ccb_graph> g(new ccb_graph());
  CCB_CUDA(cudaGetDevice(&g->device));
  g->n = (int)n;
  g->words = (int)((n + 31) / 32);
  g->pitch = std::max(4, (g->words + 3) / 4 * 4);
  const size_t rows = std::max<uint32_t>(n, 1);
  const size_t bytes = rows * g->pitch * sizeof(uint32_t);
  size_t free_b = 0, total_b = 0;
  CCB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (bytes + rows * 4 > free_b) {
    Fail(CCB_ERR_DEVICE_MEMORY, "graph needs " + std::to_string((bytes + (1 << 20) - 1) >> 20) +
                                    " MiB of device memory, " + std::to_string(free_b >> 20) + " MiB free");
  }
  CCB_CUDA(cudaMalloc(&g->bits, bytes));
  CCB_CUDA(cudaMalloc(&g->degrees, rows * sizeof(int32_t)));
  CCB_CUDA(cudaMemsetAsync(g->bits, 0, bytes, stream));
  CCB_CUDA(cudaMemsetAsync(g->degrees, 0, rows * sizeof(int32_t), stream));
  return g.release();
}

void FinishGraph(ccb_graph& g, cudaStream_t stream) {
  if (g.n > 0) {
    k_graph_degrees<<<(g.n + 255) / 256, 256, 0, stream>>>(g.bits, g.n, g.words, g.pitch, g.degrees);
    CCB_CUDA(cudaGetLastError());
  }
  CCB_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace ccb

using namespace ccb;

extern "C" {

int ccb_graph_generate_erdos_renyi(uint32_t n, double density, uint64_t seed, void* stream, ccb_graph** out) {
  return Guard([&] {
    if (!out) Fail(CCB_ERR_STATE, "null output handle");
    *out = Generate(n, 0, seed, density, 0.0, 0.0, {}, static_cast<cudaStream_t>(stream));
  });
}

int ccb_graph_generate_planted(uint32_t n, int32_t parts, int32_t shuffle_split, double p_in, double p_out,
                               double flip, uint64_t seed, void* stream, ccb_graph** out, int32_t* community_out) {
  return Guard([&] {
    if (!out) Fail(CCB_ERR_STATE, "null output handle");
    // Communities on the host: the same sequential draws as ccb_generate_planted.
    std::vector<int32_t> community(n);
    if (shuffle_split) {
      std::vector<uint32_t> order(n);
      std::iota(order.begin(), order.end(), 0u);
      uint64_t s = StreamSeed(seed, kPlantedTag, 1);
      for (uint32_t i = n; i-- > 1;) std::swap(order[i], order[DrawBelow(s, i + 1)]);
      for (uint32_t pos = 0; pos < n; ++pos) community[order[pos]] = pos < n / 2 ? 0 : 1;
    } else {
      uint64_t s = StreamSeed(seed, kPlantedTag, 2);
      for (uint32_t v = 0; v < n; ++v) community[v] = (int32_t)DrawBelow(s, (uint32_t)std::max(parts, 1));
    }
    *out = Generate(n, 1, seed, p_in, p_out, flip, community, static_cast<cudaStream_t>(stream));
    if (community_out) std::copy(community.begin(), community.end(), community_out);
  });
}

int ccb_graph_download(const ccb_graph* g, uint32_t* bits, uint32_t words_per_row) {
  return Guard([&] {
    if (!g) Fail(CCB_ERR_STATE, "null graph");
    if (g->n == 0) return;
    if (words_per_row < (uint32_t)g->words) Fail(CCB_ERR_INVALID, "words_per_row < ceil(n / 32)");
    CCB_CUDA(cudaMemcpy2D(bits, words_per_row * sizeof(uint32_t), g->bits, g->pitch * sizeof(uint32_t),
                          g->words * sizeof(uint32_t), g->n, cudaMemcpyDeviceToHost));
    if (words_per_row > (uint32_t)g->words) {
      for (int v = 0; v < g->n; ++v) {
        for (uint32_t w = g->words; w < words_per_row; ++w) bits[(size_t)v * words_per_row + w] = 0;
      }
    }
  });
}

}  // extern "C"
