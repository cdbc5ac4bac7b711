// C entry points over the reference's own CPU code (test infrastructure only).
//
// oracle/Makefile compiles this file together with the reference sources src/cc_graph.cpp and
// src/cc_pbils_cpu.cpp, read in place from the reference checkout, into oracle/_ref/libccref.so.
// The tests load it with ctypes to pin the plain-C restatement in oracle/cc_oracle.c against the
// reference itself, case by case.  Nothing in the product loads it.
#include <cstdint>
#include <cstring>
#include <vector>

#include "cc_graph.hpp"
#include "cc_math.hpp"
#include "cc_pbils.hpp"

namespace {

// cc::Graph has no constructor from raw words, so the pairs are replayed through AddEdge.
cc::Graph FromBits(const uint32_t* bits, uint32_t n, uint32_t words) {
  cc::Graph g(n);
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = i + 1; j < n; ++j)
      if ((bits[(size_t)i * words + j / 32] >> (j % 32)) & 1u) g.AddEdge(i, j);
  return g;
}

}  // namespace

extern "C" {

struct ref_params {
  int32_t k, population, tournament, iterations, early_stop;
  double perturbation, gww;
  uint64_t seed;
};

struct ref_result {
  int64_t objective;
  int32_t iterations_done, clusters_used;
  int64_t local_searches, accepted_moves;
};

// Graph::ErdosRenyi (src/cc_graph.cpp:168-177); bits must hold n * max(1, ceil(n/32)) words.
uint64_t ref_erdos_renyi(uint32_t n, double density, uint64_t seed, uint32_t* bits) {
  const cc::Graph g = cc::Graph::ErdosRenyi(n, density, seed);
  std::memcpy(bits, g.Bits().data(), g.Bits().size() * sizeof(uint32_t));
  return g.EdgeCount();
}

// SolveCpu (src/cc_pbils_cpu.cpp:183-252).
int ref_pbils(const uint32_t* bits, uint32_t n, uint32_t words, const ref_params* p, int threads, int32_t* labels_out,
              ref_result* out) {
  const cc::Graph g = FromBits(bits, n, words);
  cc::PbilsParams params;
  params.k = p->k;
  params.population = p->population;
  params.tournament = p->tournament;
  params.iterations = p->iterations;
  params.early_stop = p->early_stop;
  params.perturbation = p->perturbation;
  params.gww = p->gww;
  params.seed = p->seed;
  params.threads = threads;
  try {
    const cc::PbilsResult r = cc::SolveCpu(g, params);
    for (uint32_t v = 0; v < n; ++v) labels_out[v] = r.labels[v];
    out->objective = r.objective;
    out->iterations_done = r.iterations_done;
    out->clusters_used = r.clusters_used;
    out->local_searches = r.local_searches;
    out->accepted_moves = r.accepted_moves;
  } catch (...) {
    return -1;
  }
  return 0;
}

// State::Rebuild (src/cc_pbils_cpu.cpp:74-95).
int64_t ref_rebuild(const uint32_t* bits, uint32_t n, uint32_t words, int k, const int32_t* labels, int32_t* g_out,
                    int32_t* sizes_out) {
  const cc::Graph g = FromBits(bits, n, words);
  cc::State s;
  s.Init((int)n, k);
  for (uint32_t v = 0; v < n; ++v) s.labels[v] = labels[v];
  s.Rebuild(g);
  if (g_out) std::memcpy(g_out, s.g.data(), s.g.size() * sizeof(int32_t));
  if (sizes_out) std::memcpy(sizes_out, s.sizes.data(), s.sizes.size() * sizeof(int32_t));
  return s.f;
}

// LocalSearch (src/cc_pbils_cpu.cpp:141-149) from `labels`, rebuilt first.
int64_t ref_local_search(const uint32_t* bits, uint32_t n, uint32_t words, int k, int32_t* labels, int64_t* moves) {
  const cc::Graph g = FromBits(bits, n, words);
  cc::State s;
  s.Init((int)n, k);
  for (uint32_t v = 0; v < n; ++v) s.labels[v] = labels[v];
  s.Rebuild(g);
  long long m = 0;
  cc::LocalSearch(g, s, &m);
  for (uint32_t v = 0; v < n; ++v) labels[v] = s.labels[v];
  *moves = m;
  return s.f;
}

// The sequential Neighborhood check of cuda/cc_verify_gpu.cu:21-35, on the reference's State.
int ref_neighborhood(const uint32_t* bits, uint32_t n, uint32_t words, int local_search, int32_t* labels_out,
                     ref_result* out) {
  const cc::Graph g = FromBits(bits, n, words);
  cc::State s;
  s.Init((int)n, 2);
  long long best = -1;
  long long moves = 0;
  std::vector<int> labels;
  for (uint32_t v = 0; v < n; ++v) {
    for (uint32_t u = 0; u < n; ++u) s.labels[u] = (u == v || g.IsJoined(v, u)) ? 0 : 1;
    s.Rebuild(g);
    if (local_search) cc::LocalSearch(g, s, &moves);
    if (best < 0 || s.f < best) {
      best = s.f;
      labels = s.labels;
    }
  }
  for (uint32_t v = 0; v < n; ++v) labels_out[v] = labels[v];
  out->objective = best;
  out->iterations_done = 0;
  out->clusters_used = cc::CountClustersUsed(labels, 2);
  out->local_searches = local_search ? n : 0;
  out->accepted_moves = moves;
  return 0;
}

// The same loop over start vertices [first, first + count) only: a bounded sample of the brute force, for
// timing the reference's CPU Neighborhood on the GPU box (bench.py's CPU baseline).  Returns the moves.
int64_t ref_neighborhood_range(const uint32_t* bits, uint32_t n, uint32_t words, int local_search, uint32_t first,
                               uint32_t count, int64_t* best_out) {
  const cc::Graph g = FromBits(bits, n, words);
  cc::State s;
  s.Init((int)n, 2);
  long long best = -1;
  long long moves = 0;
  for (uint32_t v = first; v < first + count && v < n; ++v) {
    for (uint32_t u = 0; u < n; ++u) s.labels[u] = (u == v || g.IsJoined(v, u)) ? 0 : 1;
    s.Rebuild(g);
    if (local_search) cc::LocalSearch(g, s, &moves);
    if (best < 0 || s.f < best) best = s.f;
  }
  *best_out = best;
  return moves;
}

// Graph::LoadTags (src/cc_graph.cpp:311-371): writes up to `capacity` vertices' rows (max(1, ceil(n/32)) words
// each) into bits and the edge count into edges_out; returns the vertex count, or -1 on an error.
int64_t ref_load_tags(const char* path, const char* similarity, double threshold, uint32_t n, uint64_t seed,
                      uint32_t capacity, uint32_t* bits, uint64_t* edges_out) {
  try {
    const cc::Graph g = cc::Graph::LoadTags(path, similarity, threshold, n, seed);
    if (g.Size() > capacity) return -1;
    std::memcpy(bits, g.Bits().data(), g.Bits().size() * sizeof(uint32_t));
    *edges_out = g.EdgeCount();
    return g.Size();
  } catch (...) {
    return -1;
  }
}

int64_t ref_objective_direct(const uint32_t* bits, uint32_t n, uint32_t words, const int32_t* labels) {
  const cc::Graph g = FromBits(bits, n, words);
  return cc::ObjectiveDirect(g, std::vector<int>(labels, labels + n));
}

int64_t ref_objective_bitwise(const uint32_t* bits, uint32_t n, uint32_t words, const int32_t* labels) {
  const cc::Graph g = FromBits(bits, n, words);
  return cc::ObjectiveBitwise(g, std::vector<int>(labels, labels + n));
}

void ref_rank_slots(const int64_t* f, int population, int32_t* order) {
  std::vector<long long> ff(f, f + population);
  const std::vector<int> o = cc::RankSlots(ff.data(), population);
  for (int i = 0; i < population; ++i) order[i] = o[i];
}

int ref_tournament(uint64_t base, int slot, int iteration, const int64_t* f, int population, int tournament) {
  std::vector<long long> ff(f, f + population);
  return cc::Tournament(base, slot, iteration, ff.data(), population, tournament);
}

int ref_perturbed_label(uint64_t base, uint64_t index, int iteration, int label, int k, float p) {
  return cc::PerturbedLabel(base, index, iteration, label, k, p);
}

int ref_initial_label(uint64_t base, uint64_t index, int k) { return cc::InitialLabel(base, index, k); }

uint64_t ref_stream_seed(uint64_t seed, uint64_t stream, uint64_t step) { return cc::StreamSeed(seed, stream, step); }

}  // extern "C"
