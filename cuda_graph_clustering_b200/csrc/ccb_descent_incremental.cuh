// Steepest descent for 9 <= k <= 64 on the narrow path (n <= 32767) with incrementally maintained best moves.
// Same trajectory as k_descent and the reference's BestMove/ApplyMove (src/cc_pbils_cpu.cpp:99-139).
//
// Keys are key_c(u) = 64 h_c(u) + c with h_c = size_c - 2 G_c(u), so the smallest key is the smallest h, then
// the lowest cluster: the reference's target rule.  Every warp keeps off[c] = 64 size_c + c in its own
// shared-memory row, so key_c(u) = off[c] - 128 G_c(u).  Per vertex the slot state holds
//   g[c][u]   the counters G_c(u), 16-bit, cluster-major (a move touches lanes from and to of many vertices,
//             contiguous in this layout; the rare full rescan reads k strided entries);
//   lab[u]    the label a(u);
//   kbest[u]  min over c != a(u) of key_c(u);   kown[u] = key_a(u)(u).
// A move (v: from -> to) changes, for every u, only key_from and key_to (and G_from, G_to of neighbours of v).
// So the cached minimum is updated from those two keys, and all K lanes are rescanned only when the cached
// best target is `from` or `to` and its key grew (on average about one vertex in K - 1), or for v itself,
// whose set of foreign clusters changed.  The update is folded into the next move's scan.
#pragma once

#include <cstdint>

#include "ccb_device.cuh"

namespace ccb {

// Smallest key over c != own of vertex u; the counters are cluster-major with leading dimension ld.
__device__ __forceinline__ int RescanBest(const uint16_t* g, int ld, int u, const int* off, int k, int own) {
  int best = 0x7fffffff;
  for (int c = 0; c < k; ++c) {
    const int key = off[c] - 128 * static_cast<int>(g[static_cast<size_t>(c) * ld + u]);
    if (c != own) best = min(best, key);
  }
  return best;
}

// Shared or global layout of one slot's incremental state (all arrays indexed by vertex, leading dimension ld).
struct IncState {
  uint16_t* g;    // [k][ld] counters G_c(u), cluster-major: the two lanes a move touches are contiguous
  int* kbest;     // [ld]
  int* kown;      // [ld]
  uint8_t* lab;   // [ld]

  __host__ __device__ static size_t Bytes(int k, int ld) {
    return static_cast<size_t>(ld) * (static_cast<size_t>(k) * 2 + 4 + 4 + 1);
  }
  __device__ void Carve(unsigned char* base, int k, int ld) {
    g = reinterpret_cast<uint16_t*>(base);
    kbest = reinterpret_cast<int*>(base + static_cast<size_t>(k) * ld * 2);
    kown = kbest + ld;
    lab = reinterpret_cast<uint8_t*>(kown + ld);
  }
};

template <int T, bool kSmemState>
__device__ __forceinline__ void DescentIncremental(const DescentArgs<int16_t>& a, int slot) {
  constexpr int kWarps = T / kWarp;
  constexpr int U = 4;
  constexpr int KP = kMaxK;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<uint32_t> s_records[2 * kWarps];
  __shared__ int s_off[kWarps][KP];

  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int warp = tid / kWarp;
  const int n = a.gr.n;
  const int k = a.k;
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

  IncState st;
  st.Carve(kSmemState ? smem
                      : reinterpret_cast<unsigned char*>(a.next.g) + static_cast<size_t>(slot) * IncState::Bytes(k, ld),
           k, ld);
  int* off = s_off[warp];
  {
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
    for (int c = lane; c < KP; c += kWarp) off[c] = c < k ? 64 * sizes[c] + c : 0x3fffffff;
    __syncwarp();
    const uint4* g_src = reinterpret_cast<const uint4*>(a.cur.g + static_cast<size_t>(w) * k * ld);
    uint4* g_dst = reinterpret_cast<uint4*>(st.g);
    for (size_t i = tid; i < static_cast<size_t>(k) * ld / 8; i += T) g_dst[i] = g_src[i];
    __syncthreads();
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
    for (int u = tid; u < n; u += T) {
      const int own = l_src[u];
      st.lab[u] = static_cast<uint8_t>(own);
      st.kown[u] = off[own] - 128 * static_cast<int>(st.g[static_cast<size_t>(own) * ld + u]);
      st.kbest[u] = RescanBest(st.g, ld, u, off, k, own);
    }
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  __syncthreads();

  unsigned long long applied = 0;
  int parity = 0;
  int from = -1, to = -1, moved = -1;
  const uint32_t* prev_row = nullptr;
  const uint32_t lane_bit = 1u << lane;
  const uint32_t key_base = (1u << bits) << bits;

  while (true) {
    uint32_t best = KeyTraits<uint32_t>::kNone;
    uint32_t payload = 0;
    for (int base = tid; base < n; base += U * T) {
      int own[U], kb[U], ko[U];
      uint32_t rw[U];
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        if (u < n) {
          own[i] = st.lab[u];
          kb[i] = st.kbest[u];
          ko[i] = st.kown[u];
          rw[i] = prev_row != nullptr ? prev_row[u >> 5] : 0u;
        }
      }
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        if (u >= n) continue;
        if (prev_row != nullptr) {
          uint16_t* g_from = st.g + static_cast<size_t>(from) * ld + u;
          uint16_t* g_to = st.g + static_cast<size_t>(to) * ld + u;
          int gf = *g_from;
          int gt = *g_to;
          if (rw[i] & lane_bit) {
            *g_from = static_cast<uint16_t>(--gf);
            *g_to = static_cast<uint16_t>(++gt);
          }
          const int kf = off[from] - 128 * gf;
          const int kt = off[to] - 128 * gt;
          if (u == moved) {
            // its own cluster changed: foreign set is new, rescan
            own[i] = to;
            st.lab[u] = static_cast<uint8_t>(to);
            ko[i] = kt;
            kb[i] = RescanBest(st.g, ld, u, off, k, to);
          } else {
            if (own[i] == from) ko[i] = kf;
            if (own[i] == to) ko[i] = kt;
            const int b = kb[i] & 63;
            const bool from_foreign = own[i] != from;
            const bool to_foreign = own[i] != to;
            if ((b == from && kf > kb[i]) || (b == to && kt > kb[i])) {
              kb[i] = RescanBest(st.g, ld, u, off, k, own[i]);
            } else {
              int m = (b == from || b == to) ? 0x7fffffff : kb[i];
              if (from_foreign) m = min(m, kf);
              if (to_foreign) m = min(m, kt);
              kb[i] = m;
            }
          }
          st.kbest[u] = kb[i];
          st.kown[u] = ko[i];
        }
        const int gain = (kb[i] >> 6) - (ko[i] >> 6) + 1;
        const uint32_t mk = static_cast<uint32_t>(gain * (1 << bits)) + key_base + static_cast<uint32_t>(u);
        if (mk < best) {
          best = mk;
          payload = static_cast<uint32_t>(own[i]) | (static_cast<uint32_t>(kb[i] & 63) << 8);
        }
      }
    }
    const MoveRecord<uint32_t> m = BlockArgMin<uint32_t, kWarps>(best, payload, s_records + parity * kWarps);
    if (m.key >= key_base) break;
    parity ^= 1;

    moved = MoveVertex(m.key, bits);
    from = static_cast<int>(m.payload & 0xff);
    to = static_cast<int>(m.payload >> 8);
    if (lane == 0) {
      off[from] -= 64;
      off[to] += 64;
    }
    __syncwarp();
    prev_row = a.gr.bits + static_cast<size_t>(moved) * pitch;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, 1);
      break;
    }
  }

  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
  for (int u = tid; u < n; u += T) dst[u] = st.lab[u];
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

// One slot per block (plain path).
template <int T, bool kSmemState>
__global__ void __launch_bounds__(T, 1) k_descent_incremental(DescentArgs<int16_t> a) {
  DescentIncremental<T, kSmemState>(a, blockIdx.x);
}

}  // namespace ccb
