// Steepest descent for 4096 < n <= 32767 and K <= 8: the slot's state streams from shared memory when it
// fits, else from its rows of `next` in global memory (L2 resident: 16 bytes per vertex at K <= 8).
// Same trajectory as k_descent and the reference's BestMove/ApplyMove (src/cc_pbils_cpu.cpp:99-139).
//
// A vertex is one packed vector of KP 16-bit lanes: lane c holds G_c(u), and the lane of u's own cluster
// holds G_a(u) + 2^15 (no label array).  Every thread keeps off[c] = 16 size_c + c.  Read as signed 16-bit,
// the own lane gives key_a = off[a] - 32 G_a + 2^20, i.e. h_a + 65536 in units of h; since a foreign
// h_c = size_c - 2 G_c <= n - size_a and h_a >= 2 - size_a, foreign minus own h is at most n - 2 < 2^15,
// so over the lanes the minimum key is the best foreign target (smallest h, then lowest cluster: the
// reference's rule) and the maximum is the own cluster.  A move (v: from -> to) adds a packed +1 / -1 to
// lanes to / from of every neighbour (no carries: G_from >= 1 there, and lanes stay below 2^16), moves
// the bias of v from lane `from` to lane `to`, and changes off[from], off[to] by -16 / +16.  The update is
// folded into the next scan; vertices are taken four at a time with their loads issued first.
// With the state in global memory and kHint, its accesses carry an L2 evict_last priority and the bitset rows
// evict_first: the population's packed state (128 slots x 32000 vertices x 16 bytes = 64 MB) then stays in L2
// while the rows (128 MB at n = 32000) stream past it, instead of the rows evicting dirty state lines.
#pragma once

#include <cstdint>

#include "ccb_descent_registers.cuh"
#include "ccb_descent_small_k.cuh"
#include "ccb_device.cuh"

namespace ccb {

template <int KP, int C>
__device__ __forceinline__ int SignedLane32(const typename PackedGains<KP>::Vec& v) {
  const uint32_t word = PackedGains<KP>::Word(v, C / 2);
  if constexpr (C & 1) {
    return (static_cast<int>(word) >> 16) * 32;
  } else {
    return static_cast<int>(word << 16) >> 11;
  }
}

template <int K, int KP, int C>
struct LaneKeys {
  __device__ __forceinline__ static void Run(const typename PackedGains<KP>::Vec& v, const int* off, int* keys) {
    keys[C] = off[C] - SignedLane32<KP, C>(v);
    LaneKeys<K, KP, C + 1>::Run(v, off, keys);
  }
};
template <int K, int KP>
struct LaneKeys<K, KP, K> {
  __device__ __forceinline__ static void Run(const typename PackedGains<KP>::Vec&, const int*, int*) {}
};

template <int KP>
__device__ __forceinline__ void ShiftLane(typename PackedGains<KP>::Vec& v, int lane, uint32_t amount) {
  uint32_t d[PackedGains<KP>::kWords];
#pragma unroll
  for (int i = 0; i < PackedGains<KP>::kWords; ++i) d[i] = (lane >> 1) == i ? (amount << (16 * (lane & 1))) : 0u;
  PackedGains<KP>::Add(v, d);
}

template <int K, int T, bool kSmemState, bool kHint = false>
__device__ __forceinline__ void DescentStream(const DescentArgs<int16_t>& a, int slot) {
  static_assert(!(kSmemState && kHint), "L2 hints are for state in global memory");
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

  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int n = a.gr.n;
  const int ld = a.ld;
  const int bits = a.key_bits;
  const int pitch = a.gr.pitch;

  if (tid == 0) {
    s_stop = a.ctl->stop;
    if (!s_stop) {
      const int64_t* f = a.cur.f;
      s_winner = a.tournament > 0 ? TournamentWinner(a.select_stream, slot, a.iteration, a.population, a.tournament,
                                                     [f](int i) { return f[i]; })
                                  : slot;
    }
  }
  __syncthreads();
  if (s_stop) return;
  const int w = s_winner;

  Vec* gv = kSmemState ? reinterpret_cast<Vec*>(smem) : reinterpret_cast<Vec*>(a.next.g) + static_cast<size_t>(slot) * ld;
  [[maybe_unused]] uint64_t keep = 0, drop = 0;
  if constexpr (kHint) {
    keep = L2PolicyEvictLast();
    drop = L2PolicyEvictFirst();
  }
  auto load = [&](int u) -> Vec {
    if constexpr (kHint) {
      return LoadL2Hint(gv + u, keep);
    } else {
      return gv[u];
    }
  };
  auto store = [&](int u, const Vec& x) {
    if constexpr (kHint) {
      StoreL2Hint(gv + u, x, keep);
    } else {
      gv[u] = x;
    }
  };
  int off[K];
  {
    const int16_t* g_src = a.cur.g + static_cast<size_t>(w) * K * ld;
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
#pragma unroll
    for (int c = 0; c < K; ++c) off[c] = 16 * sizes[c] + c;
    for (int u = tid; u < n; u += T) {
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
      store(u, v);
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
    for (int base = tid; base < n; base += U * T) {
      Vec v[U];
      uint32_t rw[U];
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        if (u < n) {
          v[i] = load(u);
          if constexpr (kHint) {
            rw[i] = prev_row != nullptr ? LoadL2Hint(prev_row + (u >> 5), drop) : 0u;
          } else {
            rw[i] = prev_row != nullptr ? prev_row[u >> 5] : 0u;
          }
        } else {
          rw[i] = 0u;
        }
      }
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        if (u < n) {
          if (rw[i] & lane_bit) {
            P::Add(v[i], delta);
            store(u, v[i]);
          }
          int keys[K];
          LaneKeys<K, KP, 0>::Run(v[i], off, keys);
          int lo, hi;
          LanesMinMax<K>(keys, lo, hi);
          const int gain = (lo >> 4) - (hi >> 4) + (kPenalty >> 4) + 1;
          // improving moves sort below 2^(2B), the rest above it (gain <= n - 1 keeps it below 2^32)
          const uint32_t mk = static_cast<uint32_t>(gain * (1 << bits)) + key_base + static_cast<uint32_t>(u);
          if (mk < best) {
            best = mk;
            payload = static_cast<uint32_t>(hi & 15) | (static_cast<uint32_t>(lo & 15) << 8);
          }
        }
      }
    }
    const MoveRecord<uint32_t> m = BlockArgMin<uint32_t, kWarps>(best, payload, s_records + parity * kWarps);
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
    if (v % T == tid) {
      Vec x = load(v);
      ShiftLane<KP>(x, from, 0xFFFF8000u);  // the own-cluster bias leaves lane `from` (no borrow: bit 15 set)
      ShiftLane<KP>(x, to, 0x8000u);        // and enters lane `to` (no carry: G_to < 2^15)
      store(v, x);
    }
    prev_row = a.gr.bits + static_cast<size_t>(v) * pitch;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
  }

  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
  for (int u = tid; u < n; u += T) {
    Vec x;
    if constexpr (kHint) {
      x = LoadL2Hint(gv + u, drop);  // the last read of this launch: the line may leave first now
    } else {
      x = gv[u];
    }
    int own = 0;
#pragma unroll
    for (int c = 0; c < K; ++c) {
      const uint32_t word = P::Word(x, c / 2);
      if ((word >> (16 * (c & 1) + 15)) & 1u) own = c;
    }
    dst[u] = static_cast<uint8_t>(own);
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

// One slot per block (plain path).
template <int K, int T, bool kSmemState, bool kHint>
__global__ void __launch_bounds__(T, 1) k_descent_stream(DescentArgs<int16_t> a) {
  DescentStream<K, T, kSmemState, kHint>(a, blockIdx.x);
}

}  // namespace ccb
