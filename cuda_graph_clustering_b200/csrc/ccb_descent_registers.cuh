// Steepest descent with the slot state in registers as move keys: compile-time K <= 8, V vertices per thread
// (u = tid + j * T, j < V), n <= V * T.  Same trajectory as k_descent and the reference's BestMove/ApplyMove
// (src/cc_pbils_cpu.cpp:99-139).
//
// For each owned vertex u a thread keeps K 32-bit keys
//     key_c(u) = 16 h_c(u) + c  (+ 2^20 for c = the label of u),   h_c(u) = size_c - 2 G_c(u),
// so the key of moving u to c orders candidates by h, then by the lower cluster: the reference's rule
// (MoveDelta, cc_math.hpp:75-77: the gain of a -> c is h_c - h_a + 1).  A foreign h_c <= n - size_a and the
// own h_a >= 2 - size_a, so foreign minus own h is at most n - 2 < 2^15 on the narrow path; the penalty
// (2^16 in units of h) therefore makes the minimum over the K lanes the best foreign target and the
// maximum the vertex's own cluster: no label, no G, no per-cluster offset is stored.
//
// A move (v: from -> to) shifts, for every vertex u, key_from by +16 if u is a neighbour of v and -16
// otherwise (size_from - 1, and G_from - 1 for neighbours), and key_to by the opposite amount; with the
// per-move coefficients coef_c = [c = from] - [c = to] that is one multiply-add per lane, folded into the
// scan of the next move.  The moved vertex itself (not its own neighbour) also moves its penalty from lane
// `from` to lane `to`.
#pragma once

#include <cstdint>

#include "ccb_device.cuh"

namespace ccb {

constexpr int kRegPenalty = 1 << 20;

// Minimum and maximum of K lanes with three-input min / max (DPX on sm_90 and later).
template <int K>
__device__ __forceinline__ void LanesMinMax(const int* x, int& lo, int& hi) {
  lo = x[0];
  hi = x[0];
  int c = 1;
#pragma unroll
  for (; c + 1 < K; c += 2) {
    lo = __vimin3_s32(lo, x[c], x[c + 1]);
    hi = __vimax3_s32(hi, x[c], x[c + 1]);
  }
  if (c < K) {
    lo = min(lo, x[c]);
    hi = max(hi, x[c]);
  }
}

// ---- compact keys (n <= 1023) ---------------------------------------------------------------------------
// With B = bit width of n <= 10 and S = B + 8, a vertex's lanes are
//     foreign c:  L_c = (h_c << S) + c          own a:  L_a = ((h_a + P) << S) - 16 a,    P = 2^(B+1)
// (|h| <= n < 2^B, so every foreign lane is below 2^(B+S) and the own lane above it: max = own, min = the best
// foreign target, smaller cluster first).  Then the block's move key of the vertex is a single add:
//     kmin - kmax + ((P + 1 + 2^B) << S) + (u << 8) = ((gain + 2^B) << S) | (u << 8) | (a << 4) | to,
// gain + 2^B in [2, 2^(B+1)) since the gain is in [1 - n, n - 1]: smaller gain, then smaller vertex, as the
// reference orders moves, with both clusters riding in the low byte.  A move (v: from -> to) changes lanes
// `from` and `to` of every vertex by -/+ 2^S (sign by adjacency to v), folded into the next scan.  Keys are
// unsigned so that the lanes of absent vertices (u >= n, ignored) wrap instead of overflowing.
constexpr int kCompactMaxBits = 10;

// One scan of the vertices: fold the last move into lanes (coef[c] = [c = from] - [c = to] times the signed step,
// by adjacency to the moved vertex), then each vertex's move key.
template <int K, int V>
__device__ __forceinline__ uint32_t CompactScan(uint32_t (&key)[V][K], const uint32_t (&rw)[V], uint32_t lane_bit,
                                                const uint32_t (&cu)[V], unsigned valid, const int (&coef)[K],
                                                int step) {
  uint32_t best = ~0u;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int d = (rw[j] & lane_bit) ? step : -step;
    int lanes[K];
#pragma unroll
    for (int c = 0; c < K; ++c) {
      key[j][c] += static_cast<uint32_t>(coef[c] * d);
      lanes[c] = static_cast<int>(key[j][c]);
    }
    int kmin, kmax;
    LanesMinMax<K>(lanes, kmin, kmax);
    const uint32_t mk = static_cast<uint32_t>(kmin - kmax) + cu[j];
    best = min(best, ((valid >> j) & 1) ? mk : ~0u);
  }
  return best;
}

template <int K, int T, int V>
__device__ __forceinline__ void DescentRegistersCompact(const DescentArgs<int16_t>& a, int slot, int w,
                                                        const uint32_t* rows, MoveRecord<uint32_t>* s_records) {
  constexpr int kWarps = T / kWarp;
  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int n = a.gr.n;
  const int ld = a.ld;
  const int bits = a.key_bits;
  const int shift = bits + 8;
  const uint32_t step = 1u << shift;
  const uint32_t penalty = (2u << bits) << shift;

  uint32_t key[V][K];
  uint32_t cu[V];
  unsigned valid = 0;
  {
    const int16_t* g_src = a.cur.g + static_cast<size_t>(w) * K * ld;
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
    int sz[K];
#pragma unroll
    for (int c = 0; c < K; ++c) sz[c] = sizes[c];
    const uint32_t base = ((2u << bits) + 1u + (1u << bits)) << shift;
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int u = tid + j * T;
      const bool ok = u < n;
      valid |= ok ? (1u << j) : 0u;
      const int own = ok ? l_src[u] : 0;
#pragma unroll
      for (int c = 0; c < K; ++c) {
        const int h = sz[c] - 2 * (ok ? static_cast<int>(g_src[static_cast<size_t>(c) * ld + u]) : 0);
        const uint32_t lane_key = (static_cast<uint32_t>(h) << shift) + static_cast<uint32_t>(c);
        key[j][c] = c == own ? lane_key + penalty - 17u * static_cast<uint32_t>(c) : lane_key;
      }
      cu[j] = base + (static_cast<uint32_t>(ok ? u : 0) << 8);
    }
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  unsigned long long applied = 0;
  int parity = 0;
  const uint32_t lane_bit = 1u << lane;
  const uint32_t no_move = (1u << bits) << shift;
  const uint32_t vmask = (1u << bits) - 1u;

  uint32_t rw[V];
  int coef[K];
#pragma unroll
  for (int j = 0; j < V; ++j) rw[j] = 0u;
#pragma unroll
  for (int c = 0; c < K; ++c) coef[c] = 0;
  uint32_t best = CompactScan<K, V>(key, rw, lane_bit, cu, valid, coef, static_cast<int>(step));
  while (true) {
    const uint32_t mkey = BlockArgMin<uint32_t, kWarps>(best, 0u, s_records + parity * kWarps).key;
    if (mkey >= no_move) break;
    parity ^= 1;
    const int v = static_cast<int>((mkey >> 8) & vmask);
    const int from = static_cast<int>((mkey >> 4) & 15u);
    const int to = static_cast<int>(mkey & 15u);
    if ((v % T) == tid) {  // the moved vertex's own lane moves from `from` to `to`
      const int jv = v / T;
#pragma unroll
      for (int j = 0; j < V; ++j) {
        if (j == jv) {
#pragma unroll
          for (int c = 0; c < K; ++c) {
            if (c == from) key[j][c] += 17u * static_cast<uint32_t>(c) - penalty;
            if (c == to) key[j][c] += penalty - 17u * static_cast<uint32_t>(c);
          }
        }
      }
    }
    objective += static_cast<long long>(static_cast<int>(mkey >> shift) - (1 << bits));
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
    const uint32_t* row = rows + static_cast<size_t>(v) * a.gr.pitch;
#pragma unroll
    for (int j = 0; j < V; ++j) rw[j] = ((valid >> j) & 1) ? row[(tid + j * T) >> 5] : 0u;  // words < ceil(n/32)
#pragma unroll
    for (int c = 0; c < K; ++c) coef[c] = (c == from ? 1 : 0) - (c == to ? 1 : 0);
    best = CompactScan<K, V>(key, rw, lane_bit, cu, valid, coef, static_cast<int>(step));
  }

  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    if ((valid >> j) & 1) {
      int lanes[K];
#pragma unroll
      for (int c = 0; c < K; ++c) lanes[c] = static_cast<int>(key[j][c]);
      int kmin, kmax;
      LanesMinMax<K>(lanes, kmin, kmax);
      dst[tid + j * T] = static_cast<uint8_t>(((0u - static_cast<uint32_t>(kmax)) >> 4) & 15u);
    }
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

template <int K, int T, int V, bool kSmemRows>
__device__ __forceinline__ void DescentRegisters(const DescentArgs<int16_t>& a, int slot) {
  constexpr int kWarps = T / kWarp;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<uint32_t> s_records[2 * kWarps];

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
  if constexpr (T * V <= 1024) {
    if (a.key_bits <= kCompactMaxBits) {
      DescentRegistersCompact<K, T, V>(a, slot, w, rows, s_records);
      return;
    }
  }

  int key[V][K];
  int ucode[V];  // (2^B << B) | u: adding gain << B gives the block-wide move key
  unsigned valid = 0;
  {
    const int16_t* g_src = a.cur.g + static_cast<size_t>(w) * K * ld;
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
    int s16[K];
#pragma unroll
    for (int c = 0; c < K; ++c) s16[c] = 16 * sizes[c] + c;
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int u = tid + j * T;
      const bool ok = u < n;
      valid |= ok ? (1u << j) : 0u;
      const int own = ok ? l_src[u] : 0;
#pragma unroll
      for (int c = 0; c < K; ++c) {
        const int gc = ok ? g_src[static_cast<size_t>(c) * ld + u] : 0;
        key[j][c] = s16[c] - 32 * gc + (c == own ? kRegPenalty : 0);
      }
      ucode[j] = ok ? (((1 << bits) << bits) | u) : (1 << 30);
    }
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;

  unsigned long long applied = 0;
  int parity = 0;
  bool pending = false;  // a move still to be folded into the keys
  int coef[K];           // [c = from] - [c = to] of that move
#pragma unroll
  for (int c = 0; c < K; ++c) coef[c] = 0;
  const uint32_t* prev_row = rows;
  const uint32_t lane_bit = 1u << lane;
  const uint32_t no_move = (1u << bits) << bits;

  while (true) {
    uint32_t rw[V];
#pragma unroll
    for (int j = 0; j < V; ++j) rw[j] = (pending && ((valid >> j) & 1)) ? prev_row[(tid + j * T) >> 5] : 0u;
    uint32_t best = KeyTraits<uint32_t>::kNone;
    uint32_t payload = 0;
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int d = (rw[j] & lane_bit) ? 16 : -16;
#pragma unroll
      for (int c = 0; c < K; ++c) key[j][c] += coef[c] * d;
      int kmin, kmax;
      LanesMinMax<K>(key[j], kmin, kmax);
      const int gain = (kmin >> 4) - (kmax >> 4) + (kRegPenalty >> 4) + 1;
      // (gain + 2^B) << B | u for every vertex: improving moves sort below 2^(2B), the rest above it
      // (gain <= n - 1), and absent vertices carry 2^31 in ucode.
      const uint32_t mk = static_cast<uint32_t>(gain * (1 << bits)) + static_cast<uint32_t>(ucode[j]);
      if (mk < best) {
        best = mk;
        payload = static_cast<uint32_t>(kmax & 15) | (static_cast<uint32_t>(kmin & 15) << 8);
      }
    }
    const MoveRecord<uint32_t> m = BlockArgMin<uint32_t, kWarps>(best, payload, s_records + parity * kWarps);
    if (m.key >= no_move) break;
    parity ^= 1;

    const int v = MoveVertex(m.key, bits);
    const int from = static_cast<int>(m.payload & 0xff);
    const int to = static_cast<int>(m.payload >> 8);
#pragma unroll
    for (int c = 0; c < K; ++c) coef[c] = (c == from ? 1 : 0) - (c == to ? 1 : 0);
    if (v % T == tid) {
      const int jv = v / T;
#pragma unroll
      for (int j = 0; j < V; ++j) {
        if (j == jv) {
#pragma unroll
          for (int c = 0; c < K; ++c) key[j][c] -= coef[c] * kRegPenalty;
        }
      }
    }
    prev_row = rows + static_cast<size_t>(v) * a.gr.pitch;
    pending = true;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
  }

  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    if ((valid >> j) & 1) {
      int kmin, kmax;
      LanesMinMax<K>(key[j], kmin, kmax);
      dst[tid + j * T] = static_cast<uint8_t>(kmax & 15);
    }
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

// One slot per block (plain path).
template <int K, int T, int V, bool kSmemRows>
__global__ void __launch_bounds__(T, 1) k_descent_registers(DescentArgs<int16_t> a) {
  DescentRegisters<K, T, V, kSmemRows>(a, blockIdx.x);
}

}  // namespace ccb
