// Counter-based random streams and move algebra shared by the host planner and the kernels.
//
// The solver must walk the same trajectory as the reference CPU solver for the same seed, so the
// stream derivation is the reference's, bit for bit: splitmix64 (the published generator of
// Steele, Lea and Flood, 2014) advanced from a seed that the caller carries, with the reference's
// stream seeding, draw helpers and stream tags (include/cc_math.hpp:84-145).  The code is this
// project's own; only the constants and the order of the draws have to be the same.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define CCB_HD __host__ __device__ __forceinline__
#else
#define CCB_HD inline
#endif

namespace ccb {

// splitmix64 increment and finaliser constants.
constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kMix1 = 0xBF58476D1CE4E5B9ull;
constexpr uint64_t kMix2 = 0x94D049BB133111EBull;
// Stream-seed multipliers (cc_math.hpp:107-111).
constexpr uint64_t kStreamMul = 0xD1B54A32D192ED03ull;
constexpr uint64_t kStepMul = 0xA0761D6478BD642Full;
// Stream tags (cc_math.hpp:118-121, cc_graph.cpp:20).
constexpr uint64_t kInitTag = 0xA11CE;
constexpr uint64_t kSelectTag = 0x5E1EC7;
constexpr uint64_t kPerturbTag = 0xBEEF;
constexpr uint64_t kPerturbStepBase = 0x5000000;
constexpr uint64_t kErdosRenyiTag = 0xE4D05F;
// This project's planted-partition generator (no counterpart in the reference).
constexpr uint64_t kPlantedTag = 0x9A27ED;

CCB_HD uint64_t Mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * kMix1;
  z = (z ^ (z >> 27)) * kMix2;
  return z ^ (z >> 31);
}

// One draw: advance the carried state by the golden gamma and return its mix.
CCB_HD uint64_t Draw64(uint64_t& state) {
  state += kGamma;
  return Mix64(state);
}

CCB_HD uint32_t DrawU32(uint64_t& state) { return static_cast<uint32_t>(Draw64(state) >> 32); }

// Uniform integer in [0, bound) by a 32x32 multiply-shift; bound 0 gives 0.
CCB_HD uint32_t DrawBelow(uint64_t& state, uint32_t bound) {
  return bound == 0 ? 0u : static_cast<uint32_t>((static_cast<uint64_t>(DrawU32(state)) * bound) >> 32);
}

// Uniform float in [0, 1) with 24 random mantissa bits.  Exact in IEEE single precision, so host and
// device compare the same value against a probability.
CCB_HD float DrawUnit(uint64_t& state) {
  return static_cast<float>(DrawU32(state) >> 8) * (1.0f / 16777216.0f);
}

// The stream seed derived from (seed, stream, step): one finalisation round of the combined word.
CCB_HD uint64_t StreamBase(uint64_t seed, uint64_t stream, uint64_t step) {
  return seed ^ (stream * kStreamMul) ^ (step * kStepMul);
}

CCB_HD uint64_t StreamSeed(uint64_t seed, uint64_t stream, uint64_t step) {
  uint64_t s = StreamBase(seed, stream, step);
  Draw64(s);
  return s;
}

// Label of population entry `index` (= slot * n + vertex) in the initial population.
CCB_HD int InitialLabelOf(uint64_t base, uint64_t index, int k) {
  uint64_t s = StreamSeed(base, index, 0);
  return static_cast<int>(DrawBelow(s, static_cast<uint32_t>(k)));
}

// Tournament winner for `slot` of iteration `iteration`: the best f among `tournament` uniform draws;
// a later draw replaces the current one only if strictly better.
template <typename FitnessAt>
CCB_HD int TournamentWinner(uint64_t base, int slot, int iteration, int population, int tournament, FitnessAt f) {
  uint64_t s = StreamSeed(base, static_cast<uint64_t>(slot), static_cast<uint64_t>(iteration + 1));
  int chosen = static_cast<int>(DrawBelow(s, static_cast<uint32_t>(population)));
  int64_t best = f(chosen);
  for (int t = 1; t < tournament; ++t) {
    const int candidate = static_cast<int>(DrawBelow(s, static_cast<uint32_t>(population)));
    const int64_t fc = f(candidate);
    if (fc < best) {
      chosen = candidate;
      best = fc;
    }
  }
  return chosen;
}

// With probability p the label moves to a uniformly drawn other cluster, otherwise it stays.
CCB_HD int PerturbLabelOf(uint64_t base, uint64_t index, int iteration, int label, int k, float p) {
  uint64_t s = StreamSeed(base, index, static_cast<uint64_t>(iteration) + kPerturbStepBase);
  if (DrawUnit(s) >= p) return label;
  return (label + 1 + static_cast<int>(DrawBelow(s, static_cast<uint32_t>(k - 1)))) % k;
}

// Change of the disagreement count when a vertex with g_from neighbours in its cluster (of size
// size_from) moves to a cluster of size size_to holding g_to of its neighbours.
CCB_HD int MoveGain(int size_from, int size_to, int g_from, int g_to) {
  return (size_to - size_from + 1) - 2 * (g_to - g_from);
}

// sum over clusters of C(size, 2).
CCB_HD int64_t PairsInside(const int* sizes, int k) {
  int64_t acc = 0;
  for (int c = 0; c < k; ++c) acc += static_cast<int64_t>(sizes[c]) * (sizes[c] - 1) / 2;
  return acc;
}

}  // namespace ccb
