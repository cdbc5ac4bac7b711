// Steepest descent with the whole slot state in registers: compile-time K <= 8, four vertices per thread
// (u = tid + j * T, j < 4), n <= 4 * T <= 4096.  Same trajectory as k_descent and the reference's
// BestMove/ApplyMove (src/cc_pbils_cpu.cpp:99-139).
//
// Per owned vertex a thread keeps
//   g[j]    the K counters G_c(u) in 16-bit lanes of one 4/8/16-byte vector, the own cluster's lane with its
//           top bit set (G_a + 2^15, never carries: G <= n - 1 < 2^15);
//   lab[j]  the label a(u);
//   hown[j] h_a(u) = size_a - 2 G_a(u), kept up to date move by move;
// and every thread keeps off[c] = 16 size_c + c.  The key of moving u to c is off[c] - 32 G_c(u) =
// 16 h_c(u) + c; read through a sign-extending unpack, the own lane's key carries a +2^20 penalty, which for
// n <= 21844 exceeds the spread of all keys, so the best foreign target is a plain minimum over the lanes
// (smallest h, then lowest cluster: the reference's rule).  A move (v: from -> to) changes, for every u,
//   h_from += 2 adj - 1,  h_to += 1 - 2 adj      (adj = u is a neighbour of v),
// and for neighbours G_from -= 1, G_to += 1 (one packed add).  The moved vertex's own lane moves from `from`
// to `to` and its h_own becomes its old h_to (the uniform update then adds the size change).
#pragma once

#include <cstdint>

#include "ccb_descent_small_k.cuh"
#include "ccb_device.cuh"

namespace ccb {

constexpr int kRegVerticesPerThread = 4;
constexpr int kRegMaxVertices = 21844;  // limit of the own-lane penalty (48 n < 2^20 - 15)

// Key contribution 32 * lane c, read as a signed 16-bit value (so the own lane comes out negative).
template <int KP, int C>
__device__ __forceinline__ int Scaled32(const typename PackedGains<KP>::Vec& v) {
  const uint32_t word = PackedGains<KP>::Word(v, C / 2);
  if constexpr (C & 1) {
    return (static_cast<int>(word) >> 16) * 32;
  } else {
    return static_cast<int>(word << 16) >> 11;
  }
}

template <int K, int KP, int C>
struct LaneMin {
  __device__ __forceinline__ static int Run(const typename PackedGains<KP>::Vec& v, const int* off, int acc) {
    acc = min(acc, off[C] - Scaled32<KP, C>(v));
    return LaneMin<K, KP, C + 1>::Run(v, off, acc);
  }
};
template <int K, int KP>
struct LaneMin<K, KP, K> {
  __device__ __forceinline__ static int Run(const typename PackedGains<KP>::Vec&, const int*, int acc) { return acc; }
};

template <int KP>
__device__ __forceinline__ void AddLane(typename PackedGains<KP>::Vec& v, int lane, uint32_t amount) {
  uint32_t d[PackedGains<KP>::kWords];
#pragma unroll
  for (int i = 0; i < PackedGains<KP>::kWords; ++i) d[i] = (lane >> 1) == i ? (amount << (16 * (lane & 1))) : 0u;
  PackedGains<KP>::Add(v, d);
}

template <int K, int T, bool kSmemRows>
__global__ void __launch_bounds__(T, 1) k_descent_registers(DescentArgs<int16_t> a) {
  constexpr int KP = PackedLanes(K);
  constexpr int V = kRegVerticesPerThread;
  using P = PackedGains<KP>;
  using Vec = typename P::Vec;
  constexpr int kWarps = T / kWarp;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<uint32_t> s_records[2 * kWarps];

  const int slot = blockIdx.x;
  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int n = a.gr.n;
  const int ld = a.ld;
  const int bits = a.key_bits;

  if (tid == 0) {
    s_stop = a.ctl->stop;
    if (!s_stop) {
      const int64_t* f = a.cur.f;
      s_winner = a.tournament > 0 ? TournamentWinner(a.select_stream, slot, a.iteration, a.population, a.tournament,
                                                     [f](int i) { return f[i]; })
                                  : slot;
    }
  }
  const uint32_t* rows = a.gr.bits;
  if constexpr (kSmemRows) {
    const size_t row_words = static_cast<size_t>(n) * a.gr.pitch;
    const uint4* src = reinterpret_cast<const uint4*>(a.gr.bits);
    uint4* dst = reinterpret_cast<uint4*>(smem);
    for (size_t i = tid; i < row_words / 4; i += T) dst[i] = __ldg(src + i);
    rows = reinterpret_cast<const uint32_t*>(smem);
  }
  __syncthreads();
  if (s_stop) return;
  const int w = s_winner;

  int off[K];
  {
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
#pragma unroll
    for (int c = 0; c < K; ++c) off[c] = 16 * sizes[c] + c;
  }
  Vec g[V];
  int lab[V];
  int hown[V];
  int ucode[V];  // (2^B << B) | u: adding gain << B gives the move key
  unsigned valid = 0;
  {
    const int16_t* g_src = a.cur.g + static_cast<size_t>(w) * K * ld;
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int u = tid + j * T;
      uint32_t words[P::kWords];
#pragma unroll
      for (int i = 0; i < P::kWords; ++i) words[i] = 0;
      int own = 0, g_own = 0;
      if (u < n) {
        valid |= 1u << j;
        own = l_src[u];
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const int gc = g_src[static_cast<size_t>(c) * ld + u];
          words[c / 2] |= static_cast<uint32_t>(gc + (c == own ? 0x8000 : 0)) << (16 * (c & 1));
          if (c == own) g_own = gc;
        }
      }
      if constexpr (KP == 2) {
        g[j] = words[0];
      } else if constexpr (KP == 4) {
        g[j] = make_uint2(words[0], words[1]);
      } else {
        g[j] = make_uint4(words[0], words[1], words[2], words[3]);
      }
      lab[j] = own;
      int s_own = 0;
#pragma unroll
      for (int c = 0; c < K; ++c) s_own = (c == own) ? (off[c] >> 4) : s_own;
      hown[j] = s_own - 2 * g_own;
      ucode[j] = ((1 << bits) << bits) | u;
    }
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;

  unsigned long long applied = 0;
  int parity = 0;
  bool pending = false;  // a move whose neighbour update is still to be folded in
  int from = 0, to = 0;
  const uint32_t* prev_row = rows;
  uint32_t delta[P::kWords];
#pragma unroll
  for (int i = 0; i < P::kWords; ++i) delta[i] = 0;
  const uint32_t lane_bit = 1u << lane;

  while (true) {
    // Fold the previous move into the owned vertices, then score them.
    uint32_t rw[V];
#pragma unroll
    for (int j = 0; j < V; ++j) rw[j] = (pending && ((valid >> j) & 1)) ? prev_row[(tid + j * T) >> 5] : 0u;
    int kb[V];
    uint32_t key[V];
    uint32_t best = KeyTraits<uint32_t>::kNone;
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const bool adj = (rw[j] & lane_bit) != 0;
      if (adj) P::Add(g[j], delta);
      if (pending) {
        const int d = adj ? 1 : -1;  // h_from += 2 adj - 1, h_to -= 2 adj - 1
        hown[j] += (lab[j] == from ? d : 0) - (lab[j] == to ? d : 0);
      }
      kb[j] = LaneMin<K, KP, 0>::Run(g[j], off, 0x7fffffff);
      const int gain = (kb[j] >> 4) - hown[j] + 1;
      key[j] = (gain < 0 && ((valid >> j) & 1)) ? static_cast<uint32_t>(gain * (1 << bits) + ucode[j])
                                                : KeyTraits<uint32_t>::kNone;
      best = min(best, key[j]);
    }
    uint32_t payload = 0;
#pragma unroll
    for (int j = V - 1; j >= 0; --j) {
      if (key[j] == best) payload = static_cast<uint32_t>(lab[j]) | (static_cast<uint32_t>(kb[j] & 15) << 8);
    }
    const MoveRecord<uint32_t> m = BlockArgMin<uint32_t, kWarps>(best, payload, s_records + parity * kWarps);
    if (m.key == KeyTraits<uint32_t>::kNone) break;
    parity ^= 1;

    const int v = MoveVertex(m.key, bits);
    from = static_cast<int>(m.payload & 0xff);
    to = static_cast<int>(m.payload >> 8);
#pragma unroll
    for (int c = 0; c < K; ++c) off[c] += (c == to ? 16 : 0) - (c == from ? 16 : 0);
#pragma unroll
    for (int i = 0; i < P::kWords; ++i) {
      delta[i] = ((to >> 1) == i ? (1u << (16 * (to & 1))) : 0u) - ((from >> 1) == i ? (1u << (16 * (from & 1))) : 0u);
    }
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if (v == tid + j * T) {
        // the moved vertex: own lane from -> to, h_own = its old h_to (the size change is added above)
        AddLane<KP>(g[j], from, 0xFFFF8000u);  // - 2^15 in lane `from` (its top bit is set: no borrow)
        AddLane<KP>(g[j], to, 0x8000u);
        hown[j] = kb[j] >> 4;
        lab[j] = to;
      }
    }
    prev_row = rows + static_cast<size_t>(v) * a.gr.pitch;
    pending = true;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, 1);
      break;
    }
  }

  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    if ((valid >> j) & 1) dst[tid + j * T] = static_cast<uint8_t>(lab[j]);
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

}  // namespace ccb
