// Host instance generators of libccb: the reference's seeded Erdős–Rényi graph and this project's seeded
// planted partition.  Both draw from one sequential splitmix64 stream over the pairs (i ascending,
// j < i ascending), so any caller that passes the same seed gets the same bits.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "ccb.h"
#include "ccb_streams.cuh"

namespace {

inline void SetPair(uint32_t* bits, uint32_t words, uint32_t i, uint32_t j) {
  bits[(size_t)i * words + j / 32] |= 1u << (j % 32);
  bits[(size_t)j * words + i / 32] |= 1u << (i % 32);
}

}  // namespace

extern "C" {

// Graph::ErdosRenyi (src/cc_graph.cpp:168-177): pair (i, j) is an edge iff its draw is below `density`.
uint64_t ccb_generate_erdos_renyi(uint32_t n, double density, uint64_t seed, uint32_t* bits, uint32_t words_per_row) {
  std::memset(bits, 0, (size_t)n * words_per_row * sizeof(uint32_t));
  uint64_t state = ccb::StreamSeed(seed, ccb::kErdosRenyiTag, 0);
  uint64_t edges = 0;
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t j = 0; j < i; ++j) {
      if ((double)ccb::DrawUnit(state) < density) {
        SetPair(bits, words_per_row, i, j);
        ++edges;
      }
    }
  }
  return edges;
}

// Planted partition.  Communities: with shuffle_split a Fisher-Yates shuffle of the vertices (stream step
// 1; i from n-1 down to 1 swaps i with a draw below i + 1) puts the first n/2 positions in community 0
// and the rest in 1; otherwise each vertex in order draws one of `parts` communities (step 2).  Edges
// (step 3): per pair two draws, edge = (first < p_in or p_out) XOR (second < flip).
uint64_t ccb_generate_planted(uint32_t n, int32_t parts, int32_t shuffle_split, double p_in, double p_out,
                              double flip, uint64_t seed, uint32_t* bits, uint32_t words_per_row,
                              int32_t* community_out) {
  std::memset(bits, 0, (size_t)n * words_per_row * sizeof(uint32_t));
  std::vector<int32_t> community(n);
  if (shuffle_split) {
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    uint64_t s = ccb::StreamSeed(seed, ccb::kPlantedTag, 1);
    for (uint32_t i = n; i-- > 1;) std::swap(order[i], order[ccb::DrawBelow(s, i + 1)]);
    for (uint32_t pos = 0; pos < n; ++pos) community[order[pos]] = pos < n / 2 ? 0 : 1;
  } else {
    uint64_t s = ccb::StreamSeed(seed, ccb::kPlantedTag, 2);
    for (uint32_t v = 0; v < n; ++v) community[v] = (int32_t)ccb::DrawBelow(s, (uint32_t)std::max(parts, 1));
  }
  uint64_t state = ccb::StreamSeed(seed, ccb::kPlantedTag, 3);
  uint64_t edges = 0;
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t j = 0; j < i; ++j) {
      const double p = community[i] == community[j] ? p_in : p_out;
      const bool edge = (double)ccb::DrawUnit(state) < p;
      const bool flipped = (double)ccb::DrawUnit(state) < flip;
      if (edge != flipped) {
        SetPair(bits, words_per_row, i, j);
        ++edges;
      }
    }
  }
  if (community_out) std::copy(community.begin(), community.end(), community_out);
  return edges;
}

}  // extern "C"
