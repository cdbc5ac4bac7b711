// Steepest descent specialised for a compile-time number of clusters K <= 8 (narrow path, n <= 32767).
//
// Same trajectory as k_descent (and as the reference's BestMove/ApplyMove, src/cc_pbils_cpu.cpp:99-139);
// what changes is how much work a move costs:
//
//  * G is vertex-major: the K counters of a vertex are KP (= 2, 4 or 8) 16-bit lanes packed in one
//    4/8/16-byte vector, so the scan reads one vector per vertex instead of K scattered entries.
//  * The cluster part of every candidate key lives in registers: off[c] = 16 * size_c + c, identical in
//    all threads, updated by the two clusters of each move.  The key of moving u to c is
//    off[c] - 32 * G_c(u) = 16 * h_c(u) + c with h_c = size_c - 2 G_c, so one multiply-add per candidate,
//    and the smallest key is the smallest h, then the lowest cluster: the reference's target rule.
//  * The gain of u's best move is (best >> 4) - (own >> 4) + 1 (the cluster index sits in the low 4 bits).
//  * The G update of move i is applied while scanning for move i + 1: a neighbour u of the moved vertex
//    adds a packed delta (+1 in lane `to`, -1 in lane `from`) to the vector it just loaded.  G_from(u) >= 1
//    for such u (the moved vertex itself is counted there) and G_to(u) + 1 <= n - 1 < 2^15, so lanes never
//    borrow or carry into each other.
#pragma once

#include <cstdint>

#include "ccb_device.cuh"

namespace ccb {

template <int KP>
struct PackedGains;
template <>
struct PackedGains<2> {
  using Vec = uint32_t;
  static constexpr int kWords = 1;
  __device__ static uint32_t Word(const Vec& v, int) { return v; }
  __device__ static void Add(Vec& v, const uint32_t* d) { v += d[0]; }
};
template <>
struct PackedGains<4> {
  using Vec = uint2;
  static constexpr int kWords = 2;
  __device__ static uint32_t Word(const Vec& v, int i) { return i == 0 ? v.x : v.y; }
  __device__ static void Add(Vec& v, const uint32_t* d) {
    v.x += d[0];
    v.y += d[1];
  }
};
template <>
struct PackedGains<8> {
  using Vec = uint4;
  static constexpr int kWords = 4;
  __device__ static uint32_t Word(const Vec& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }
  __device__ static void Add(Vec& v, const uint32_t* d) {
    v.x += d[0];
    v.y += d[1];
    v.z += d[2];
    v.w += d[3];
  }
};

constexpr int PackedLanes(int k) { return k <= 2 ? 2 : (k <= 4 ? 4 : 8); }

template <int K, int T, bool kSmemState, bool kSmemRows>
__global__ void __launch_bounds__(T, 1) k_descent_small_k(DescentArgs<int16_t> a) {
  constexpr int KP = PackedLanes(K);
  using P = PackedGains<KP>;
  using Vec = typename P::Vec;
  constexpr int kWarps = T / kWarp;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;

  const int slot = blockIdx.x;
  const int tid = threadIdx.x;
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
  __syncthreads();
  if (s_stop) return;
  const int w = s_winner;

  // Shared memory: rows | packed G | labels | move records.
  unsigned char* p = smem;
  const uint32_t* rows = a.gr.bits;
  if constexpr (kSmemRows) {
    const size_t row_words = static_cast<size_t>(n) * a.gr.pitch;
    const uint4* src = reinterpret_cast<const uint4*>(a.gr.bits);
    uint4* dst = reinterpret_cast<uint4*>(p);
    for (size_t i = tid; i < row_words / 4; i += T) dst[i] = __ldg(src + i);
    rows = reinterpret_cast<const uint32_t*>(p);
    p += (row_words * 4 + 15) / 16 * 16;
  }
  Vec* gv;
  uint8_t* lab;
  if constexpr (kSmemState) {
    gv = reinterpret_cast<Vec*>(p);
    p += static_cast<size_t>(ld) * sizeof(Vec);
    lab = p;
    p += (ld + 15) / 16 * 16;
  } else {
    gv = reinterpret_cast<Vec*>(a.next.g) + static_cast<size_t>(slot) * ld;
    lab = a.next.labels + static_cast<size_t>(slot) * ld;
  }
  MoveRecord<uint32_t>* records = reinterpret_cast<MoveRecord<uint32_t>*>(p);

  // Copy-in: the winner's cluster-major G becomes packed vectors; labels as they are.
  {
    const int16_t* g_src = a.cur.g + static_cast<size_t>(w) * K * ld;
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
    for (int u = tid; u < n; u += T) {
      uint32_t words[P::kWords];
#pragma unroll
      for (int i = 0; i < P::kWords; ++i) {
        const int c0 = 2 * i, c1 = 2 * i + 1;
        const uint32_t lo = c0 < K ? static_cast<uint16_t>(g_src[static_cast<size_t>(c0) * ld + u]) : 0u;
        const uint32_t hi = c1 < K ? static_cast<uint16_t>(g_src[static_cast<size_t>(c1) * ld + u]) : 0u;
        words[i] = lo | (hi << 16);
      }
      Vec v;
      if constexpr (KP == 2) {
        v = words[0];
      } else if constexpr (KP == 4) {
        v = make_uint2(words[0], words[1]);
      } else {
        v = make_uint4(words[0], words[1], words[2], words[3]);
      }
      gv[u] = v;
      lab[u] = l_src[u];
    }
  }
  int off[K];
  {
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
#pragma unroll
    for (int c = 0; c < K; ++c) off[c] = 16 * sizes[c] + c;
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  __syncthreads();

  unsigned long long applied = 0;
  int parity = 0;
  const uint32_t* prev_row = nullptr;  // row of the last applied move, still to be folded into G
  uint32_t delta[P::kWords];
#pragma unroll
  for (int i = 0; i < P::kWords; ++i) delta[i] = 0;

  while (true) {
    uint32_t best = KeyTraits<uint32_t>::kNone;
    uint32_t payload = 0;
    for (int u = tid; u < n; u += T) {
      Vec v = gv[u];
      if (prev_row != nullptr && Bit(prev_row, u)) {
        P::Add(v, delta);
        gv[u] = v;
      }
      const int own = lab[u];
      int k_own = 0;
      int k_best = 0x7fffffff;
#pragma unroll
      for (int c = 0; c < K; ++c) {
        const uint32_t word = P::Word(v, c / 2);
        const int g = (c & 1) ? static_cast<int>(word >> 16) : static_cast<int>(word & 0xffffu);
        const int key = off[c] - 32 * g;
        if (c == own) {
          k_own = key;
        } else {
          k_best = min(k_best, key);
        }
      }
      const int gain = (k_best >> 4) - (k_own >> 4) + 1;
      if (gain < 0) {
        const uint32_t key = PackMove<uint32_t>(gain, u, bits);
        if (key < best) {
          best = key;
          payload = static_cast<uint32_t>(own) | (static_cast<uint32_t>(k_best & 15) << 8);
        }
      }
    }
    const MoveRecord<uint32_t> m = BlockArgMin<uint32_t, kWarps>(best, payload, records + parity * kWarps);
    if (m.key == KeyTraits<uint32_t>::kNone) break;
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
    prev_row = rows + static_cast<size_t>(v) * a.gr.pitch;
    if (v % T == tid) lab[v] = static_cast<uint8_t>(to);
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, 1);
      break;
    }
  }

  if constexpr (kSmemState) {
    uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
    for (int u = tid; u < n; u += T) dst[u] = lab[u];
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

}  // namespace ccb
