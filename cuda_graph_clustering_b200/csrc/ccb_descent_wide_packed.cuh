// Steepest descent on the wide path (32767 < n <= 2^20) for k = 2 and k = 3 with the slot's state packed into
// one word per vertex, so the whole population's state stays resident in L2 (k = 2: 4 bytes per vertex,
// 32 MiB for n = 65536 and 128 slots; k = 3: 8 bytes, 64 MiB).  Same trajectory as k_descent and the
// reference's BestMove/ApplyMove (src/cc_pbils_cpu.cpp:99-139); the reference's own packed wide kernels are
// KernelLocalSearch2Wide / KernelLocalSearch3Wide (cuda/cc_local_search_k2.cuh:132-221,
// cuda/cc_local_search_k3.cuh:28-127).
//
// k = 2: word = 2 e + a with e = G_1(u) - G_0(u) and a the label.  With s = size_1 - size_0 the only move of
//        u has gain d = s + 1 - 2e (a = 0) or 2 - d (a = 1).  A move of v to cluster t adds +-2 to e of every
//        neighbour (word +-4) and flips a(v).
// k = 3: word = G_0 | G_1 << 20 | G_2 << 40 | a << 60.  Per vertex h_c = size_c - 2 G_c, the best foreign
//        target is the smallest 4 h_c + c over c != a and its gain is h_c - h_a + 1.  A move of v from f to t
//        adds 2^(20 t) - 2^(20 f) to every neighbour's word (no borrow: G_f >= 1 there) and rewrites a(v).
// Each thread owns the vertices u = j T + tid; the update of the previous move is folded into the next scan
// (one pass over the state per move), and a word is stored back only when it changed.
#pragma once

#include <cstdint>
#include <type_traits>

#include "ccb_device.cuh"
#include "ccb_streams.cuh"

namespace ccb {

template <int K>
struct WidePacked;

template <>
struct WidePacked<2> {
  using Word = int32_t;
  static constexpr int kGroup = 16;  // vertices whose loads are in flight together
  struct Sizes {
    int s;  // size_1 - size_0
  };
  __device__ static Word Make(const int32_t* g, int ld, int u, int a) {
    return 2 * (g[ld + u] - g[u]) + a;
  }
  __device__ static int Label(Word w) { return w & 1; }
  __device__ static void LoadSizes(const int32_t* sizes, Sizes& z) { z.s = sizes[1] - sizes[0]; }
  __device__ static void Apply(Sizes& z, int from, int to) { z.s += to == 1 ? 2 : -2; }
  // neighbour of the moved vertex / the moved vertex itself
  __device__ static Word Neighbour(Word w, int from, int to) { return w + (to == 1 ? 4 : -4); }
  __device__ static Word Moved(Word w, int to) { return (w & ~1) | to; }
  // gain of the vertex's best move and its target
  __device__ static int Gain(Word w, const Sizes& z, int& target) {
    const int a = w & 1;
    const int d = z.s + 1 - (w >> 1) * 2;
    target = a ^ 1;
    return a ? 2 - d : d;
  }
};

template <>
struct WidePacked<3> {
  using Word = unsigned long long;
  static constexpr int kGroup = 8;
  struct Sizes {
    int n0, n1, n2;
  };
  __device__ static Word Make(const int32_t* g, int ld, int u, int a) {
    return static_cast<Word>(g[u]) | static_cast<Word>(g[ld + u]) << 20 | static_cast<Word>(g[2 * ld + u]) << 40 |
           static_cast<Word>(a) << 60;
  }
  __device__ static int Label(Word w) { return static_cast<int>(w >> 60); }
  __device__ static void LoadSizes(const int32_t* sizes, Sizes& z) {
    z.n0 = sizes[0];
    z.n1 = sizes[1];
    z.n2 = sizes[2];
  }
  __device__ static void Apply(Sizes& z, int from, int to) {
    z.n0 += (to == 0) - (from == 0);
    z.n1 += (to == 1) - (from == 1);
    z.n2 += (to == 2) - (from == 2);
  }
  __device__ static Word Neighbour(Word w, int from, int to) {
    return w + (static_cast<Word>(1) << (20 * to)) - (static_cast<Word>(1) << (20 * from));
  }
  __device__ static Word Moved(Word w, int to) {
    return (w & ((static_cast<Word>(1) << 60) - 1)) | static_cast<Word>(to) << 60;
  }
  __device__ static int Gain(Word w, const Sizes& z, int& target) {
    constexpr Word kMask = (1u << 20) - 1;
    const int a = static_cast<int>(w >> 60);
    const int h0 = z.n0 - 2 * static_cast<int>(w & kMask);
    const int h1 = z.n1 - 2 * static_cast<int>((w >> 20) & kMask);
    const int h2 = z.n2 - 2 * static_cast<int>((w >> 40) & kMask);
    const int k0 = a == 0 ? 0x7fffffff : 4 * h0;
    const int k1 = a == 1 ? 0x7fffffff : 4 * h1 + 1;
    const int k2 = a == 2 ? 0x7fffffff : 4 * h2 + 2;
    const int best = min(k0, min(k1, k2));
    const int ha = a == 0 ? h0 : (a == 1 ? h1 : h2);
    target = best & 3;
    return (best >> 2) - ha + 1;
  }
};

template <int K, int T>
__device__ __forceinline__ void DescentWidePacked(const DescentArgs<int32_t>& a, int slot) {
  using P = WidePacked<K>;
  using Word = typename P::Word;
  using Key = unsigned long long;
  constexpr int kWarps = T / kWarp;
  constexpr int U = P::kGroup;
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<Key> s_records[2 * kWarps];

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

  // the slot's words in its rows of `next` (k * ld int32 per slot: room for ld words of 4 or 8 bytes)
  Word* state = reinterpret_cast<Word*>(a.next.g + static_cast<size_t>(slot) * a.k * ld);
  {
    const int32_t* g = a.cur.g + static_cast<size_t>(w) * a.k * ld;
    const uint8_t* lab = a.cur.labels + static_cast<size_t>(w) * ld;
    for (int u = tid; u < n; u += T) state[u] = P::Make(g, ld, u, lab[u]);
  }
  typename P::Sizes z;
  P::LoadSizes(a.cur.sizes + static_cast<size_t>(w) * a.kpad, z);
  long long objective = a.cur.f[w];
  const long long move_budget = objective;

  unsigned long long applied = 0;
  int parity = 0;
  int from = 0, to = 0, moved = -1;
  bool pending = false;
  const uint32_t* prev_row = a.gr.bits;
  const uint32_t lane_bit = 1u << lane;
  const Key key_base = (static_cast<Key>(1) << bits) << bits;

  while (true) {
    Key best = KeyTraits<Key>::kNone;
    uint32_t payload = 0;
    for (int j0 = 0; j0 * T < n; j0 += U) {  // block-uniform trip count
      Word wd[U];
      uint32_t rw[U];
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = (j0 + i) * T + tid;
        const bool live = u < n;
        wd[i] = live ? state[u] : Word{};
        rw[i] = live && pending ? prev_row[u >> 5] : 0u;
      }
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = (j0 + i) * T + tid;
        if (u >= n) continue;
        if (pending) {
          const Word old = wd[i];
          if (rw[i] & lane_bit) wd[i] = P::Neighbour(wd[i], from, to);
          if (u == moved) wd[i] = P::Moved(wd[i], to);
          if (wd[i] != old) state[u] = wd[i];
        }
        int target;
        const int gain = P::Gain(wd[i], z, target);
        if (gain < 0) {
          const Key mk = (static_cast<Key>(gain + (1 << bits)) << bits) + static_cast<Key>(u);
          if (mk < best) {
            best = mk;
            payload = static_cast<uint32_t>(P::Label(wd[i])) | static_cast<uint32_t>(target) << 8;
          }
        }
      }
    }
    const MoveRecord<Key> m = BlockArgMin<Key, kWarps>(best, payload, s_records + parity * kWarps);
    if (m.key >= key_base) break;
    parity ^= 1;
    moved = MoveVertex(m.key, bits);
    from = static_cast<int>(m.payload & 0xff);
    to = static_cast<int>(m.payload >> 8);
    P::Apply(z, from, to);
    prev_row = a.gr.bits + static_cast<size_t>(moved) * pitch;
    pending = true;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
  }

  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
  for (int u = tid; u < n; u += T) dst[u] = static_cast<uint8_t>(P::Label(state[u]));
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

template <int K, int T>
__global__ void __launch_bounds__(T, 1) k_descent_wide_packed(DescentArgs<int32_t> a) {
  DescentWidePacked<K, T>(a, blockIdx.x);
}

// k = 2 with work per move proportional to the moved vertex's degree instead of n.  With s = size_1 - size_0
// the gain of a vertex is s + 1 - 2e in cluster 0 and 1 - s + 2e in cluster 1, so within a cluster the best
// move is the largest e (cluster 0) or the smallest e (cluster 1), ties to the lower vertex, whatever s is.
// Every thread keeps, for the vertices it owns, the best vertex of each cluster; the block minimum over the
// threads' two candidates is the move (smallest gain, then lowest vertex).  A move of v to cluster t changes
// e by the same +-2 for every neighbour: in one cluster all neighbours get better (a compare against the
// thread's best), in the other they get worse (the thread rescans its vertices only if its best was among
// them), and v changes cluster.  A thread owns the row words {32 W j + 32 i + lane : i < W} of its warp's
// stretch (W words per thread), so the row of v is read coalesced and a rescan reads 128-byte runs.
// Best moves of the sparse k = 2 descent, one pair per thread (the owner of whole row words), kept in shared
// memory so that any lane of the owner's warp can improve them: cluster 0's best is the largest
// (e + 2^20) << 11 | (2047 - j) over the owner's cluster-0 vertices (largest e, then lowest vertex), cluster 1's the
// smallest (e + 2^20) << 11 | j over its cluster-1 vertices (smallest e, then lowest vertex), with j = 32 i + bit the
// vertex's place among the owner's (word i of the owner, lower j = lower vertex); 0 and ~0 mean none (e > -2^20
// keeps both out of reach).
__device__ __forceinline__ uint32_t Wide2Key0(int wd, uint32_t j) {
  return static_cast<uint32_t>((wd >> 1) + (1 << 20)) << 11 | (2047u - j);
}
__device__ __forceinline__ uint32_t Wide2Key1(int wd, uint32_t j) {
  return static_cast<uint32_t>((wd >> 1) + (1 << 20)) << 11 | j;
}

// Recomputes lane `owner`'s two best keys with the whole warp: the owner's vertices are the 32 of each of its row
// words, lane l reads vertex l of every word (128-byte runs), two warp reductions pick the best of each cluster,
// and the owner stores them.
template <int W, typename StateT>
__device__ __forceinline__ void WarpRescanWide2(const StateT* state, int n, int words, int owner_word0, int owner,
                                                uint32_t* k0_out, uint32_t* k1_out) {
  const int lane = threadIdx.x % kWarp;
  uint32_t k0 = 0u, k1 = ~0u;
#pragma unroll(W < 8 ? W : 8)
  for (int i = 0; i < W; ++i) {
    const int q = owner_word0 + i * kWarp;
    const int u = 32 * q + lane;
    if (q < words && u < n) {
      const int wd = state[u];
      const uint32_t j = static_cast<uint32_t>(i * kWarp + lane);
      if (wd & 1) {
        k1 = min(k1, Wide2Key1(wd, j));
      } else {
        k0 = max(k0, Wide2Key0(wd, j));
      }
    }
  }
  k0 = __reduce_max_sync(kAllLanes, k0);
  k1 = __reduce_min_sync(kAllLanes, k1);
  if (lane == owner) {
    *k0_out = k0;
    *k1_out = k1;
  }
}

// kSmem16: the slot's words 2e + label as int16 in shared memory (n * 2 bytes), exact while every degree is below
// 16384 (|2e + label| <= 2 deg + 1 < 2^15); else int32 in the slot's rows of `next` (global memory, L2).  Every
// vertex belongs to the thread that owns its row word; the two placements run the same code.
//
// Per move the neighbours of the moved vertex v are processed by the whole warp rather than each owner alone (a
// thread holds about one neighbour per move at p = 0.02, so per-thread loops left most lanes idle): the warp
// writes the set bits of its row words into a short list (owner, word, bit) in shared memory, in rounds of
// kWide2List entries, and its lanes take the entries in turn.  A neighbour's word changes by +-4 (e +- 2); if that
// makes it better, its owner's key is improved with a shared-memory atomic max / min; if worse and it was the
// owner's best, the owner is flagged and the warp rescans the owner's vertices after the round.  Keys, ties and
// the order of moves are those of the per-thread form (largest / smallest e, then the lowest vertex).
constexpr int kWide2List = 128;  // list entries per warp and round

template <int T, int W, bool kSmem16>
__device__ __forceinline__ void DescentWide2Sparse(const DescentArgs<int32_t>& a, int slot) {
  using Key = unsigned long long;
  using StateT = typename std::conditional<kSmem16, int16_t, int32_t>::type;
  constexpr int kWarps = T / kWarp;
  static_assert(W <= 32, "list entries hold the word index in 5 bits");
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<Key> s_records[2 * kWarps];
  __shared__ uint32_t s_k0[T];       // each thread's best key of cluster 0 (largest)
  __shared__ uint32_t s_k1[T];       // and of cluster 1 (smallest)
  __shared__ uint8_t s_rescan[T];    // the thread's best of the worsened cluster was a neighbour of the move
  __shared__ uint16_t s_list[kWarps][kWide2List];

  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int warp = tid / kWarp;
  const int n = a.gr.n;
  const int ld = a.ld;
  const int bits = a.key_bits;
  const int pitch = a.gr.pitch;
  const int words = (n + 31) / 32;
  const int warp_word0 = warp * kWarp * W;  // the warp's row words: warp_word0 + lane + 32 i, i < W
  const int word0 = warp_word0 + lane;      // this thread's row words: word0 + 32 i, i < W

  if (tid == 0) {
    s_stop = a.ctl->stop;
    if (!s_stop) {
      const int64_t* f = a.cur.f;
      s_winner = a.tournament > 0 ? TournamentWinner(a.select_stream, slot, a.iteration, a.population, a.tournament,
                                                     [f](int i) { return f[i]; })
                                  : slot;
    }
  }
  s_rescan[tid] = 0;
  __syncthreads();
  if (s_stop) return;
  const int w = s_winner;

  StateT* state = kSmem16 ? reinterpret_cast<StateT*>(smem)
                          : reinterpret_cast<StateT*>(a.next.g + static_cast<size_t>(slot) * a.k * ld);
  {
    const int32_t* g = a.cur.g + static_cast<size_t>(w) * a.k * ld;
    const uint8_t* lab = a.cur.labels + static_cast<size_t>(w) * ld;
    // the warp builds its owners' words 32 at a time (vertex 32 q + lane of each of its words q)
#pragma unroll 1
    for (int q = warp_word0; q < min(words, warp_word0 + kWarp * W); ++q) {
      const int u = 32 * q + lane;
      if (u < n) state[u] = static_cast<StateT>(2 * (g[ld + u] - g[u]) + lab[u]);
    }
    __syncwarp();
#pragma unroll 1
    for (int owner = 0; owner < kWarp; ++owner) {
      WarpRescanWide2<W>(state, n, words, warp_word0 + owner, owner, &s_k0[warp * kWarp + owner],
                         &s_k1[warp * kWarp + owner]);
    }
    __syncwarp();
  }
  const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
  int s = sizes[1] - sizes[0];
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  unsigned long long applied = 0;
  int parity = 0;
  const Key key_base = (static_cast<Key>(1) << bits) << bits;

  while (true) {
    Key best = KeyTraits<Key>::kNone;
    uint32_t payload = 0;
    const uint32_t k0 = s_k0[tid], k1 = s_k1[tid];
    if (k0 != 0u) {  // this thread's best move out of cluster 0
      const int e0 = static_cast<int>(k0 >> 11) - (1 << 20);
      const int j = 2047 - static_cast<int>(k0 & 2047u);
      const int u0 = 32 * (word0 + (j / kWarp) * kWarp) + j % kWarp;
      const int gain = s + 1 - 2 * e0;
      if (gain < 0) {
        best = (static_cast<Key>(gain + (1 << bits)) << bits) + static_cast<Key>(u0);
        payload = 0u | 1u << 8;
      }
    }
    if (k1 != ~0u) {  // and out of cluster 1
      const int e1 = static_cast<int>(k1 >> 11) - (1 << 20);
      const int j = static_cast<int>(k1 & 2047u);
      const int u1 = 32 * (word0 + (j / kWarp) * kWarp) + j % kWarp;
      const int gain = 1 - s + 2 * e1;
      if (gain < 0) {
        const Key mk = (static_cast<Key>(gain + (1 << bits)) << bits) + static_cast<Key>(u1);
        if (mk < best) {
          best = mk;
          payload = 1u;
        }
      }
    }
    const MoveRecord<Key> m = BlockArgMin<Key, kWarps>(best, payload, s_records + parity * kWarps);
    if (m.key >= key_base) break;
    parity ^= 1;
    const int v = MoveVertex(m.key, bits);
    const int to = static_cast<int>(m.payload >> 8);
    s += to == 1 ? 2 : -2;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
    // neighbours of v: e += 2 (to = 1) or -= 2 (to = 0); the cluster whose best gets worse is 1 resp. 0
    const int step = to == 1 ? 4 : -4;
    const int worse = to;  // e up hurts cluster 1 (smallest e wanted), e down hurts cluster 0
    const uint32_t* row = a.gr.bits + static_cast<size_t>(v) * pitch;
    uint16_t* list = s_list[warp];
    constexpr int kChunk = W < 4 ? W : 4;  // row words in flight together (one memory latency per chunk)
#pragma unroll 1
    for (int i0 = 0; i0 < W; i0 += kChunk) {
      uint32_t rw[kChunk];
#pragma unroll
      for (int t = 0; t < kChunk; ++t) {
        const int q = word0 + (i0 + t) * kWarp;
        rw[t] = q < words ? row[q] : 0u;
      }
      int cnt = 0;
#pragma unroll
      for (int t = 0; t < kChunk; ++t) cnt += __popc(rw[t]);
      int incl = cnt;  // inclusive prefix of the lanes' neighbour counts
#pragma unroll
      for (int o = 1; o < kWarp; o <<= 1) {
        const int y = __shfl_up_sync(kAllLanes, incl, o);
        if (lane >= o) incl += y;
      }
      const int total = __shfl_sync(kAllLanes, incl, kWarp - 1);
      int pos = incl - cnt;  // this lane's next list position (its entries are [incl - cnt, incl))
#pragma unroll 1
      for (int r0 = 0; r0 < total; r0 += kWide2List) {
        const int r1 = r0 + kWide2List;
#pragma unroll
        for (int t = 0; t < kChunk; ++t) {
          while (rw[t] != 0u && pos < r1) {
            const int bit = __ffs(rw[t]) - 1;
            rw[t] &= rw[t] - 1;
            list[pos - r0] = static_cast<uint16_t>(lane << 10 | (i0 + t) << 5 | bit);
            ++pos;
          }
        }
        __syncwarp();
        const int here = min(kWide2List, total - r0);
        for (int p = lane; p < here; p += kWarp) {
          const int entry = list[p];
          const int owner = entry >> 10, i = (entry >> 5) & 31, bit = entry & 31;
          const int u = 32 * (warp_word0 + owner + i * kWarp) + bit;
          const uint32_t j = static_cast<uint32_t>(i * kWarp + bit);
          const int otid = warp * kWarp + owner;
          const int wd = state[u] + step;
          state[u] = static_cast<StateT>(wd);
          if ((wd & 1) == worse) {  // u got worse: a rescan of its owner if u was the owner's best
            if (wd & 1) {
              const uint32_t kb = s_k1[otid];
              if (kb != ~0u && (kb & 2047u) == j) s_rescan[otid] = 1;
            } else {
              const uint32_t kb = s_k0[otid];
              if (kb != 0u && (kb & 2047u) == 2047u - j) s_rescan[otid] = 1;
            }
          } else if (wd & 1) {  // u got better: it may become its owner's best
            atomicMin(&s_k1[otid], Wide2Key1(wd, j));
          } else {
            atomicMax(&s_k0[otid], Wide2Key0(wd, j));
          }
        }
        __syncwarp();
      }
    }
    // v itself changes cluster (its e is unchanged: no self-loops)
    const int qv = v >> 5;
    bool rescan = false;
    if (qv >= warp_word0 && qv < warp_word0 + kWarp * W && (qv - warp_word0) % kWarp == lane) {
      const int wd = state[v] ^ 1;
      state[v] = static_cast<StateT>(wd);
      const uint32_t jv = static_cast<uint32_t>(((qv - warp_word0) / kWarp) * kWarp + (v & 31));
      if (to == 1) {  // v left cluster 0 and joins cluster 1
        rescan = s_k0[tid] != 0u && (s_k0[tid] & 2047u) == 2047u - jv;
        s_k1[tid] = min(s_k1[tid], Wide2Key1(wd, jv));
      } else {
        rescan = s_k1[tid] != ~0u && (s_k1[tid] & 2047u) == jv;
        s_k0[tid] = max(s_k0[tid], Wide2Key0(wd, jv));
      }
    }
    __syncwarp();  // every lane's stores and flags are visible to the warp's rescans
    rescan |= s_rescan[tid] != 0;
    s_rescan[tid] = 0;
    unsigned pending = __ballot_sync(kAllLanes, rescan);
    while (pending) {
      const int owner = __ffs(pending) - 1;
      pending &= pending - 1;
      WarpRescanWide2<W>(state, n, words, warp_word0 + owner, owner, &s_k0[warp * kWarp + owner],
                         &s_k1[warp * kWarp + owner]);
    }
    __syncwarp();
  }

  __syncwarp();
  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
#pragma unroll 1
  for (int q = warp_word0; q < min(words, warp_word0 + kWarp * W); ++q) {
    const int u = 32 * q + lane;
    if (u < n) dst[u] = static_cast<uint8_t>(state[u] & 1);
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

template <int T, int W, bool kSmem16>
__global__ void __launch_bounds__(T, 1) k_descent_wide2_sparse(DescentArgs<int32_t> a) {
  DescentWide2Sparse<T, W, kSmem16>(a, blockIdx.x);
}

// k = 3 in the same degree-proportional form.  For a vertex in cluster a the gain of target c is
// (size_c - size_a + 1) - 2 d with d = G_c - G_a, so within each of the six (a, c) classes the best vertex is
// the largest d, ties to the lower vertex, whatever the sizes are.  Each thread keeps one key per class,
// (d + 2^20) << 11 | (2047 - j) (j = the vertex's place among the thread's, 0: none), and its candidate is the
// smallest (gain, vertex, target) over the six.  A move of v from f to t changes d of every neighbour in class
// (a, c) by [c = t] - [c = f] - [a = t] + [a = f], the same for all of them: better (a compare), worse (a
// rescan if the class's best is among them) or unchanged; v leaves the classes of f and joins those of t.
// Vertex words as in WidePacked<3>.  Class (a, c) is 2a + (c > a ? c - 1 : c): a's two classes are 2a (its lower
// foreign target) and 2a + 1 (the higher).
__device__ __forceinline__ int Wide3Target(int cls) {
  const int a = cls >> 1, r = cls & 1;
  return r < a ? r : r + 1;
}
__device__ __forceinline__ int Wide3G(unsigned long long w, int c) {
  return static_cast<int>((w >> (20 * c)) & ((1u << 20) - 1));
}

// The keys of vertex word wd (place j) in its two classes: (a, lower foreign target) = class 2a and (a, higher
// foreign target) = class 2a + 1.
struct Wide3Keys {
  int a;
  uint32_t lo, hi;
};
__device__ __forceinline__ Wide3Keys Wide3KeysOf(unsigned long long wd, uint32_t j) {
  const int a = static_cast<int>(wd >> 60);
  const int ga = Wide3G(wd, a);
  const int clo = a == 0 ? 1 : 0, chi = a == 2 ? 1 : 2;
  const uint32_t tail = 2047u - j;
  return Wide3Keys{a, static_cast<uint32_t>(Wide3G(wd, clo) - ga + (1 << 20)) << 11 | tail,
                   static_cast<uint32_t>(Wide3G(wd, chi) - ga + (1 << 20)) << 11 | tail};
}

// Folds vertex word wd (place j) into the keys of its two classes.  The six keys are indexed by compile-time
// class only (one branch per cluster) so that they stay in registers.
__device__ __forceinline__ void Wide3Offer(unsigned long long wd, uint32_t j, uint32_t (&key)[6]) {
  const Wide3Keys kk = Wide3KeysOf(wd, j);
  if (kk.a == 0) {
    key[0] = max(key[0], kk.lo);
    key[1] = max(key[1], kk.hi);
  } else if (kk.a == 1) {
    key[2] = max(key[2], kk.lo);
    key[3] = max(key[3], kk.hi);
  } else {
    key[4] = max(key[4], kk.lo);
    key[5] = max(key[5], kk.hi);
  }
}

// A neighbour's change to its two class keys (lower and higher foreign target): better (dl / dh > 0) raises the
// key, worse (< 0) asks for a rescan when the class's best is this vertex (tail = 2047 - its place).
__device__ __forceinline__ void Wide3Fold(uint32_t& klo, uint32_t& khi, const Wide3Keys& kk, int dl, int dh,
                                          uint32_t tail, bool& rescan) {
  if (dl > 0) {
    klo = max(klo, kk.lo);
  } else if (dl < 0) {
    rescan |= (klo & 2047u) == tail;
  }
  if (dh > 0) {
    khi = max(khi, kk.hi);
  } else if (dh < 0) {
    rescan |= (khi & 2047u) == tail;
  }
}

// Where a k = 3 slot keeps its vertex words.  Wide3Global: the 64-bit words (three 20-bit counters + label) in
// the slot's rows of `next` (global memory, L2).  Wide3Smem26: a 26-bit record per vertex in shared memory, the
// label a and the two foreign differences d_c = G_c - G_a (lower foreign cluster first) as 12-bit values offset
// by 2048, exact while every degree is below 2048 (|d| <= degree).  The descent only ever needs these differences,
// so the record holds no degree and a load touches shared memory only.  The record of vertex u sits at bit 26u:
// the 32 vertices of a row word q fill exactly the 26 words [26q, 26q + 26), so every thread writes only words
// of its own.  Both present a 64-bit word of three 20-bit counters + label to the descent; Wide3Smem26's has
// G_a = 2^19 and G_c = 2^19 + d_c (the same differences; a move's +-1 steps stay inside the fields), and its
// store takes the differences of whatever word it is given, re-based on that word's label.
struct Wide3Global {
  unsigned long long* p;
  __device__ __forceinline__ unsigned long long Load(int u) const { return p[u]; }
  __device__ __forceinline__ void Store(int u, unsigned long long w) const { p[u] = w; }
};

struct Wide3Smem26 {
  uint32_t* words;
  static constexpr uint32_t kMask = (1u << 26) - 1u;
  static constexpr unsigned long long kBase = 1ull << 19;
  // The raw record: d_lo + 2048 | (d_hi + 2048) << 12 | a << 24.
  __device__ __forceinline__ uint32_t LoadRec(int u) const {
    const int o = 26 * u;
    const int wi = o >> 5, sh = o & 31;
    uint32_t rec = words[wi] >> sh;
    if (sh > 6) rec |= words[wi + 1] << (32 - sh);
    return rec & kMask;
  }
  __device__ __forceinline__ void StoreRec(int u, uint32_t rec) const {
    const int o = 26 * u;
    const int wi = o >> 5, sh = o & 31;
    words[wi] = (words[wi] & ~(kMask << sh)) | (rec << sh);
    if (sh > 6) {
      const uint32_t hi_mask = kMask >> (32 - sh);
      words[wi + 1] = (words[wi + 1] & ~hi_mask) | (rec >> (32 - sh));
    }
  }
  __device__ __forceinline__ unsigned long long Load(int u) const {
    const uint32_t rec = LoadRec(u);
    const int a = static_cast<int>(rec >> 24);
    const int clo = a == 0 ? 1 : 0, chi = a == 2 ? 1 : 2;
    const unsigned long long glo = kBase + (rec & 4095u) - 2048u, ghi = kBase + ((rec >> 12) & 4095u) - 2048u;
    return kBase << (20 * a) | glo << (20 * clo) | ghi << (20 * chi) | static_cast<unsigned long long>(a) << 60;
  }
  __device__ __forceinline__ void Store(int u, unsigned long long w) const {
    const int a = static_cast<int>(w >> 60);
    const int ga = Wide3G(w, a);
    const int clo = a == 0 ? 1 : 0, chi = a == 2 ? 1 : 2;
    StoreRec(u, static_cast<uint32_t>(Wide3G(w, clo) - ga + 2048) |
                    static_cast<uint32_t>(Wide3G(w, chi) - ga + 2048) << 12 | static_cast<uint32_t>(a) << 24);
  }
};

template <int W, typename State>
__device__ __forceinline__ void WarpRescanWide3(const State& state, int n, int words, int owner_word0, int owner,
                                                uint32_t (&key)[6]) {
  const int lane = threadIdx.x % kWarp;
  uint32_t k[6] = {0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll(W < 8 ? W : 8)
  for (int i = 0; i < W; ++i) {
    const int q = owner_word0 + i * kWarp;
    const int u = 32 * q + lane;
    if (q < words && u < n) Wide3Offer(state.Load(u), static_cast<uint32_t>(i * kWarp + lane), k);
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    const uint32_t m = __reduce_max_sync(kAllLanes, k[c]);
    if (lane == owner) key[c] = m;
  }
}

template <int T, int W, bool kSmem26>
__device__ __forceinline__ void DescentWide3Sparse(const DescentArgs<int32_t>& a, int slot) {
  using Key = unsigned long long;
  using Word = unsigned long long;
  using State = typename std::conditional<kSmem26, Wide3Smem26, Wide3Global>::type;
  constexpr int kWarps = T / kWarp;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<Key> s_records[2 * kWarps];

  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int warp = tid / kWarp;
  const int n = a.gr.n;
  const int ld = a.ld;
  const int bits = a.key_bits;
  const int pitch = a.gr.pitch;
  const int words = (n + 31) / 32;
  const int warp_word0 = warp * kWarp * W;
  const int word0 = warp_word0 + lane;  // this thread's row words: word0 + 32 i, i < W

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

  State state;
  if constexpr (kSmem26) {
    state = State{reinterpret_cast<uint32_t*>(smem)};
  } else {
    state = State{reinterpret_cast<Word*>(a.next.g + static_cast<size_t>(slot) * a.k * ld)};
  }
  uint32_t key[6] = {0u, 0u, 0u, 0u, 0u, 0u};
  {
    const int32_t* g = a.cur.g + static_cast<size_t>(w) * a.k * ld;
    const uint8_t* lab = a.cur.labels + static_cast<size_t>(w) * ld;
    if constexpr (kSmem26) {
      // a thread writes the vertices of its own row words only (the 26-bit records of a word's 32 vertices share
      // memory words with nothing else): the vertices of word q = word0 + 32 i are written by this thread
#pragma unroll 1
      for (int i = 0; i < W; ++i) {
        const int q = word0 + i * kWarp;
        if (q >= words) continue;
#pragma unroll 1
        for (int b = 0; b < 32; ++b) {
          const int u = 32 * q + b;
          if (u < n) {
            state.Store(u, static_cast<Word>(g[u]) | static_cast<Word>(g[ld + u]) << 20 |
                               static_cast<Word>(g[2 * ld + u]) << 40 | static_cast<Word>(lab[u]) << 60);
          }
        }
      }
    } else {
      // the warp builds its owners' words 32 at a time (vertex 32 q + lane of each of its words q)
#pragma unroll 1
      for (int q = warp_word0; q < min(words, warp_word0 + kWarp * W); ++q) {
        const int u = 32 * q + lane;
        if (u < n) {
          state.Store(u, static_cast<Word>(g[u]) | static_cast<Word>(g[ld + u]) << 20 |
                             static_cast<Word>(g[2 * ld + u]) << 40 | static_cast<Word>(lab[u]) << 60);
        }
      }
    }
    __syncwarp();
#pragma unroll 1
    for (int owner = 0; owner < kWarp; ++owner) WarpRescanWide3<W>(state, n, words, warp_word0 + owner, owner, key);
  }
  const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
  int sz[3] = {sizes[0], sizes[1], sizes[2]};
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  unsigned long long applied = 0;
  int parity = 0;
  const Key key_base = (static_cast<Key>(1) << bits) << bits;

  while (true) {
    Key best = KeyTraits<Key>::kNone;
    uint32_t payload = 0;
#pragma unroll
    for (int cls = 0; cls < 6; ++cls) {  // ascending (a, c): among equal (gain, vertex) the lower target stays
      if (key[cls] == 0u) continue;
      const int ca = cls >> 1, cc = Wide3Target(cls);
      const int d = static_cast<int>(key[cls] >> 11) - (1 << 20);
      const int gain = (sz[cc] - sz[ca] + 1) - 2 * d;
      if (gain >= 0) continue;
      const int j = 2047 - static_cast<int>(key[cls] & 2047u);
      const int u = 32 * (word0 + (j / kWarp) * kWarp) + j % kWarp;
      const Key mk = (static_cast<Key>(gain + (1 << bits)) << bits) + static_cast<Key>(u);
      if (mk < best) {
        best = mk;
        payload = static_cast<uint32_t>(ca) | static_cast<uint32_t>(cc) << 8;
      }
    }
    const MoveRecord<Key> m = BlockArgMin<Key, kWarps>(best, payload, s_records + parity * kWarps);
    if (m.key >= key_base) break;
    parity ^= 1;
    const int v = MoveVertex(m.key, bits);
    const int from = static_cast<int>(m.payload & 0xff);
    const int to = static_cast<int>(m.payload >> 8);
#pragma unroll
    for (int c = 0; c < 3; ++c) sz[c] += (c == to) - (c == from);  // compile-time indices: sz stays in registers
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
    const Word step = (static_cast<Word>(1) << (20 * to)) - (static_cast<Word>(1) << (20 * from));
    const uint32_t* row = a.gr.bits + static_cast<size_t>(v) * pitch;
    bool rescan = false;
    constexpr int kChunk = W < 4 ? W : 4;  // row words in flight together (one memory latency per chunk)
#pragma unroll 1
    for (int i0 = 0; i0 < W; i0 += kChunk) {
      uint32_t rwords[kChunk];
#pragma unroll
      for (int t = 0; t < kChunk; ++t) {
        const int q = word0 + (i0 + t) * kWarp;
        rwords[t] = q < words ? row[q] : 0u;
      }
      // two row words at a time as one 64-bit mask (word i low, word i + 1 high), as in the k = 2 form
#pragma unroll
      for (int t = 0; t < kChunk; t += 2) {
        const int i = i0 + t;
        unsigned long long mbits = rwords[t];
        if (t + 1 < kChunk) mbits |= static_cast<unsigned long long>(rwords[t + 1]) << 32;
        const int base = 32 * (word0 + i * kWarp);
        while (mbits) {
          int us[4];
          uint32_t js[4];  // the vertex's place among the thread's: (word index) * 32 + bit
          Word ws[4];      // 64-bit counter words (state in global memory)
          uint32_t rs[4];  // or the raw 26-bit records (shared memory)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            us[c] = -1;
            js[c] = 0u;
            if (mbits) {
              const int bit = __ffsll(mbits) - 1;
              us[c] = base + (bit >> 5) * (32 * kWarp) + (bit & 31);
              js[c] = static_cast<uint32_t>((i + (bit >> 5)) * kWarp + (bit & 31));
              mbits &= mbits - 1;
            }
          }
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            if constexpr (kSmem26) {
              rs[c] = us[c] >= 0 ? state.LoadRec(us[c]) : 0u;
            } else {
              ws[c] = us[c] >= 0 ? state.Load(us[c]) : Word{};
            }
          }
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            if (us[c] < 0) continue;
            const uint32_t j = js[c];
            const uint32_t tail = 2047u - j;
            Wide3Keys kk;
            if constexpr (kSmem26) {
              kk.a = static_cast<int>(rs[c] >> 24);
            } else {
              const Word wd = ws[c] + step;
              state.Store(us[c], wd);
              kk = Wide3KeysOf(wd, j);
            }
            const int au = kk.a;
            const int own = (au == from) - (au == to);
            const int clo = au == 0 ? 1 : 0, chi = au == 2 ? 1 : 2;
            const int dl = (clo == to) - (clo == from) + own;  // change of d for the class (au, clo)
            const int dh = (chi == to) - (chi == from) + own;  // and (au, chi)
            if constexpr (kSmem26) {
              // the record holds the two differences themselves: add the changes in place (|d| <= degree < 2048
              // keeps both fields inside [1, 4095], so no borrow or carry crosses a field)
              const uint32_t rec = rs[c] + static_cast<uint32_t>(dl) + (static_cast<uint32_t>(dh) << 12);
              state.StoreRec(us[c], rec);
              kk.lo = static_cast<uint32_t>(static_cast<int>(rec & 4095u) - 2048 + (1 << 20)) << 11 | tail;
              kk.hi = static_cast<uint32_t>(static_cast<int>((rec >> 12) & 4095u) - 2048 + (1 << 20)) << 11 | tail;
            }
            if (au == 0) {  // classes 2 au and 2 au + 1
              Wide3Fold(key[0], key[1], kk, dl, dh, tail, rescan);
            } else if (au == 1) {
              Wide3Fold(key[2], key[3], kk, dl, dh, tail, rescan);
            } else {
              Wide3Fold(key[4], key[5], kk, dl, dh, tail, rescan);
            }
          }
        }
      }
    }
    // v changes cluster (its counters are unchanged: no self-loops)
    const int qv = v >> 5;
    if (qv >= warp_word0 && qv < warp_word0 + kWarp * W && (qv - warp_word0) % kWarp == lane) {
      const Word old = state.Load(v);
      const Word wd = (old & ((static_cast<Word>(1) << 60) - 1)) | static_cast<Word>(to) << 60;
      state.Store(v, wd);
      const uint32_t j = static_cast<uint32_t>(((qv - warp_word0) / kWarp) * kWarp + (v & 31));
#pragma unroll
      for (int cls = 0; cls < 6; ++cls) {  // v leaves the two classes of `from`
        if ((cls >> 1) == from) rescan |= (key[cls] & 2047u) == (2047u - j) && key[cls];
      }
      Wide3Offer(wd, j, key);
    }
    __syncwarp();
    unsigned pending = __ballot_sync(kAllLanes, rescan);
    while (pending) {
      const int owner = __ffs(pending) - 1;
      pending &= pending - 1;
      WarpRescanWide3<W>(state, n, words, warp_word0 + owner, owner, key);
    }
  }

  __syncwarp();
  uint8_t* dst = a.next.labels + static_cast<size_t>(slot) * ld;
#pragma unroll 1
  for (int q = warp_word0; q < min(words, warp_word0 + kWarp * W); ++q) {
    const int u = 32 * q + lane;
    if (u < n) dst[u] = static_cast<uint8_t>(state.Load(u) >> 60);
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

template <int T, int W, bool kSmem26>
__global__ void __launch_bounds__(T, 1) k_descent_wide3_sparse(DescentArgs<int32_t> a) {
  DescentWide3Sparse<T, W, kSmem26>(a, blockIdx.x);
}

}  // namespace ccb
