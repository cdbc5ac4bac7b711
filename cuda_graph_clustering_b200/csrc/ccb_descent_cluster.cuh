// Steepest descent for K <= 8 when one slot's packed state does not fit one SM's shared memory (the large
// narrow instances: n = 32000 at K = 8 is 512 KiB): the state is spread over the distributed shared memory of
// a thread-block cluster of C CTAs, CTA r holding the lanes of vertices [r * span, (r + 1) * span).  Same
// state, keys and trajectory as DescentStream (ccb_descent_stream.cuh) and the reference's BestMove/ApplyMove
// (src/cc_pbils_cpu.cpp:99-139): per move every CTA scans its own vertices from its shared memory and reduces
// its best key in the block, publishes it in its half of a double buffer, and after one cluster barrier reads
// the C candidates from the other CTAs' shared memory; all CTAs take the same minimum, so they agree on the
// move and on the end of the descent (every CTA runs the same number of cluster barriers).  Rows of the
// adjacency come from L2, each CTA reading only its own words.
#pragma once

#include <cooperative_groups.h>

#include <cstdint>

#include "ccb_descent_stream.cuh"

namespace ccb {

// Vertices per CTA: whole 32-vertex words, so that each CTA reads whole words of a row.
__host__ __device__ constexpr int ClusterSpan(int n, int c) { return ((n + c - 1) / c + 31) / 32 * 32; }

template <int K, int T, int C>
__device__ __forceinline__ void DescentCluster(const DescentArgs<int16_t>& a, int slot) {
  namespace cg = cooperative_groups;
  constexpr int KP = PackedLanes(K);
  constexpr int U = 4;  // vertices in flight per thread
  using P = PackedGains<KP>;
  using Vec = typename P::Vec;
  constexpr int kWarps = T / kWarp;
  constexpr int kPenalty = 1 << 20;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<uint32_t> s_records[2 * kWarps];
  __shared__ MoveRecord<uint32_t> s_candidate[2];  // this CTA's best of the move, read by the whole cluster

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = static_cast<int>(cluster.block_rank());
  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int n = a.gr.n;
  const int ld = a.ld;
  const int bits = a.key_bits;
  const int pitch = a.gr.pitch;
  const int span = ClusterSpan(n, C);
  const int u0 = rank * span;
  const int u1 = min(n, u0 + span);

  if (tid == 0) {  // every CTA of the cluster draws the same winner from the same stream
    s_stop = a.ctl->stop;
    if (!s_stop) {
      const int64_t* f = a.cur.f;
      s_winner = a.tournament > 0 ? TournamentWinner(a.select_stream, slot, a.iteration, a.population, a.tournament,
                                                     [f](int i) { return f[i]; })
                                  : slot;
    }
  }
  __syncthreads();
  if (s_stop) return;  // the same flag for every CTA of the cluster: none of them reaches a cluster barrier
  const int w = s_winner;

  Vec* gv = reinterpret_cast<Vec*>(smem);  // gv[u - u0]
  int off[K];
  {
    const int16_t* g_src = a.cur.g + static_cast<size_t>(w) * K * ld;
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
#pragma unroll
    for (int c = 0; c < K; ++c) off[c] = 16 * sizes[c] + c;
    for (int u = u0 + tid; u < u1; u += T) {
      const int own = l_src[u];
      uint32_t words[P::kWords];
#pragma unroll
      for (int i = 0; i < P::kWords; ++i) words[i] = 0;
#pragma unroll
      for (int c = 0; c < K; ++c) {
        const uint32_t gc = static_cast<uint16_t>(g_src[static_cast<size_t>(c) * ld + u]) + (c == own ? 0x8000u : 0u);
        words[c / 2] |= gc << (16 * (c & 1));
      }
      Vec v;
      if constexpr (KP == 2) {
        v = words[0];
      } else if constexpr (KP == 4) {
        v = make_uint2(words[0], words[1]);
      } else {
        v = make_uint4(words[0], words[1], words[2], words[3]);
      }
      gv[u - u0] = v;
    }
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  __syncthreads();

  unsigned long long applied = 0;
  int parity = 0;
  const uint32_t* prev_row = nullptr;
  uint32_t delta[P::kWords];
#pragma unroll
  for (int i = 0; i < P::kWords; ++i) delta[i] = 0;
  const uint32_t lane_bit = 1u << lane;
  const uint32_t key_base = (1u << bits) << bits;

  while (true) {
    uint32_t best = KeyTraits<uint32_t>::kNone;
    uint32_t payload = 0;
    for (int base = u0 + tid; base < u1; base += U * T) {
      Vec v[U];
      uint32_t rw[U];
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        if (u < u1) {
          v[i] = gv[u - u0];
          rw[i] = prev_row != nullptr ? prev_row[u >> 5] : 0u;
        } else {
          rw[i] = 0u;
        }
      }
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        if (u < u1) {
          if (rw[i] & lane_bit) {
            P::Add(v[i], delta);
            gv[u - u0] = v[i];
          }
          int keys[K];
          LaneKeys<K, KP, 0>::Run(v[i], off, keys);
          int lo, hi;
          LanesMinMax<K>(keys, lo, hi);
          const int gain = (lo >> 4) - (hi >> 4) + (kPenalty >> 4) + 1;
          const uint32_t mk = static_cast<uint32_t>(gain * (1 << bits)) + key_base + static_cast<uint32_t>(u);
          if (mk < best) {
            best = mk;
            payload = static_cast<uint32_t>(hi & 15) | (static_cast<uint32_t>(lo & 15) << 8);
          }
        }
      }
    }
    const MoveRecord<uint32_t> mine = BlockArgMin<uint32_t, kWarps>(best, payload, s_records + parity * kWarps);
    if (tid == 0) s_candidate[parity] = mine;
    cluster.sync();  // every CTA's candidate of this move is published
    MoveRecord<uint32_t> m{KeyTraits<uint32_t>::kNone, 0u};
#pragma unroll
    for (int r = 0; r < C; ++r) {
      const MoveRecord<uint32_t>* other = cluster.map_shared_rank(&s_candidate[parity], r);
      const MoveRecord<uint32_t> x = *other;
      if (x.key < m.key) m = x;  // keys hold distinct vertices: no ties between CTAs
    }
    if (m.key >= key_base) break;
    parity ^= 1;

    const int v = MoveVertex(m.key, bits);
    const int from = static_cast<int>(m.payload & 0xff);
    const int to = static_cast<int>(m.payload >> 8);
#pragma unroll
    for (int c = 0; c < K; ++c) off[c] += (c == to ? 16 : 0) - (c == from ? 16 : 0);
#pragma unroll
    for (int i = 0; i < P::kWords; ++i) {
      delta[i] = ((to >> 1) == i ? (1u << (16 * (to & 1))) : 0u) - ((from >> 1) == i ? (1u << (16 * (from & 1))) : 0u);
    }
    if (v >= u0 && v < u1 && (v - u0) % T == tid) {
      Vec x = gv[v - u0];
      ShiftLane<KP>(x, from, 0xFFFF8000u);  // the own-cluster bias leaves lane `from`
      ShiftLane<KP>(x, to, 0x8000u);        // and enters lane `to`
      gv[v - u0] = x;
    }
    prev_row = a.gr.bits + static_cast<size_t>(v) * pitch;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {  // the same count in every CTA: a uniform exit
      if (tid == 0 && rank == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
  }

  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
  for (int u = u0 + tid; u < u1; u += T) {
    const Vec x = gv[u - u0];
    int own = 0;
#pragma unroll
    for (int c = 0; c < K; ++c) {
      const uint32_t word = P::Word(x, c / 2);
      if ((word >> (16 * (c & 1) + 15)) & 1u) own = c;
    }
    dst[u] = static_cast<uint8_t>(own);
  }
  if (tid == 0 && rank == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
  cluster.sync();  // no CTA leaves while another may still read its candidates
}

// One slot per cluster of C CTAs (plain path).
template <int K, int T, int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(T, 1) k_descent_cluster(DescentArgs<int16_t> a) {
  DescentCluster<K, T, C>(a, static_cast<int>(blockIdx.x) / C);
}

}  // namespace ccb
