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
// So the cached minimum is updated from those two keys; with a lower bound on the second-best key also
// cached, all K lanes are rescanned only when the best known key reaches that bound, or for v itself, whose
// set of foreign clusters changed.
// Empty clusters are kept out of the per-vertex caches: an empty cluster's key is its index for every vertex,
// so the best empty target is the lowest empty cluster, one value per block (with k far above the number of
// communities, most vertices' best target is empty, and a cluster filling up would otherwise send them all
// to rescan).  The update is folded into the next move's scan.
#pragma once

#include <cstdint>

#include "ccb_device.cuh"

namespace ccb {

// Smallest and second smallest key over the non-empty clusters c != own of vertex u (off[c] >= 64 iff
// size_c >= 1); the counters are cluster-major with leading dimension ld.  INT_MAX where there is none.
__device__ __forceinline__ int2 RescanBest2(const uint16_t* g, int ld, int u, const int* off, int k, int own) {
  int b1 = 0x7fffffff, b2 = 0x7fffffff;
#pragma unroll 8
  for (int c = 0; c < k; ++c) {
    const int o = off[c];
    const int key = o - 128 * static_cast<int>(g[static_cast<size_t>(c) * ld + u]);
    if (c != own && o >= 64) {
      b2 = min(b2, max(b1, key));
      b1 = min(b1, key);
    }
  }
  return make_int2(b1, b2);
}

// Smallest and second smallest key over the non-empty clusters c != own of vertex u, computed by the whole
// warp for one vertex: lane l reads clusters l and l + 32, then two warp reductions.  Every lane gets the
// result.  Keys are distinct (the cluster index is in the low bits), so exactly one lane holds the minimum.
__device__ __forceinline__ int2 WarpRescan2(const uint16_t* g, int ld, int u, const int* off, int k, int own) {
  const int lane = threadIdx.x % kWarp;
  int k1 = 0x7fffffff, k2 = 0x7fffffff;
  if (lane < k) {
    const int o = off[lane];
    if (lane != own && o >= 64) k1 = o - 128 * static_cast<int>(g[static_cast<size_t>(lane) * ld + u]);
  }
  if (lane + kWarp < k) {
    const int o = off[lane + kWarp];
    if (lane + kWarp != own && o >= 64) {
      k2 = o - 128 * static_cast<int>(g[static_cast<size_t>(lane + kWarp) * ld + u]);
    }
  }
  const int lo = min(k1, k2);
  const int hi = max(k1, k2);
  const int b1 = __reduce_min_sync(kAllLanes, lo);
  const int b2 = __reduce_min_sync(kAllLanes, lo == b1 ? hi : lo);
  return make_int2(b1, b2);
}

// Lowest-index empty cluster from a warp's off[] row, or -1.  An empty cluster c has size 0 and no
// neighbours of any vertex in it, so its key is just c for every vertex: among empty targets the lowest
// index always wins, and it is the same for all vertices.
__device__ __forceinline__ int LowestEmpty(const int* off, int k) {
  const int lane = threadIdx.x % kWarp;
  const unsigned lo = __ballot_sync(kAllLanes, lane < k && off[lane] == lane);
  const unsigned hi = __ballot_sync(kAllLanes, lane + 32 < k && off[lane + 32] == lane + 32);
  return lo ? __ffs(lo) - 1 : (hi ? 32 + __ffs(hi) - 1 : -1);
}

// Folds the move (from -> to, `moved` = the vertex that moved) into the cached keys of vertex u, given its
// new keys kf = key_from(u) and kt = key_to(u).  kb is the smallest key over the non-empty foreign
// clusters, lb a lower bound on the second smallest, ko the key of u's own cluster (label = ko & 63).
// Only key_from and key_to changed; every other foreign cluster but kb's is still >= lb.  So the best
// known key is exact whenever it stays below lb.  Returns true when it does not (the cached best got worse
// than the bound) or for the moved vertex, whose foreign set changed: then kb and lb must be rescanned.
// After the move `to` is non-empty; if `from` became empty it leaves the set.
__device__ __forceinline__ bool FoldMove(int u, int kf, int kt, int from, int to, int moved, bool from_empty,
                                         int& kb, int& lb, int& ko) {
  if (u == moved) {
    ko = kt;
    return true;
  }
  const int own = ko & 63;
  const bool of = own == from, ot = own == to;
  ko = of ? kf : (ot ? kt : ko);
  // known keys: the cached best if its cluster is neither from nor to (kb = INT_MAX, no best, reads as
  // cluster 63 and stays INT_MAX either way), key_from if foreign and non-empty, key_to if foreign
  const int b = kb & 63;
  const int m1 = (b == from || b == to) ? 0x7fffffff : kb;
  const int cf = (of || from_empty) ? 0x7fffffff : kf;
  const int ct = ot ? 0x7fffffff : kt;
  const int lo = min(cf, ct), hi = max(cf, ct);
  const int n1 = min(m1, lo);
  const int n2 = min(max(m1, lo), hi);  // second smallest of the three
  if (n1 < lb) {
    kb = n1;
    lb = min(lb, n2);
    return false;
  }
  return true;
}
// Shared or global layout of one slot's incremental state (all arrays indexed by vertex, leading dimension ld).
struct IncState {
  uint16_t* g;    // [k][ld] counters G_c(u), cluster-major: the two lanes a move touches are contiguous
  int* kbest;     // [ld]
  int* kown;      // [ld]
  int* kbound;    // [ld] lower bound on the second-best foreign key
  uint8_t* lab;   // [ld]

  __host__ __device__ static size_t Bytes(int k, int ld) {
    return static_cast<size_t>(ld) * (static_cast<size_t>(k) * 2 + 4 + 4 + 4 + 1);
  }
  __device__ void Carve(unsigned char* base, int k, int ld) {
    g = reinterpret_cast<uint16_t*>(base);
    kbest = reinterpret_cast<int*>(base + static_cast<size_t>(k) * ld * 2);
    kown = kbest + ld;
    kbound = kown + ld;
    lab = reinterpret_cast<uint8_t*>(kbound + ld);
  }
};

// GainT is the population's G type (int16 narrow, int32 wide); the slot state keeps G as uint16 counters,
// exact for every n <= 65536 (a counter is at most the degree).  Key is the move-key width: 32 bits while
// 2 * key_bits <= 32, else 64.
template <int T, bool kSmemState, typename GainT = int16_t, typename Key = uint32_t>
__device__ __forceinline__ void DescentIncremental(const DescentArgs<GainT>& a, int slot) {
  constexpr int kWarps = T / kWarp;
  constexpr int U = 4;
  constexpr int KP = kMaxK;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<Key> s_records[2 * kWarps];
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
    if constexpr (sizeof(GainT) == 2) {
      const uint4* g_src = reinterpret_cast<const uint4*>(a.cur.g + static_cast<size_t>(w) * k * ld);
      uint4* g_dst = reinterpret_cast<uint4*>(st.g);
      for (size_t i = tid; i < static_cast<size_t>(k) * ld / 8; i += T) g_dst[i] = g_src[i];
    } else {
      // int32 counters (all < 65536) narrowed to uint16, four per step
      const int4* g_src = reinterpret_cast<const int4*>(a.cur.g + static_cast<size_t>(w) * k * ld);
      uint2* g_dst = reinterpret_cast<uint2*>(st.g);
      for (size_t i = tid; i < static_cast<size_t>(k) * ld / 4; i += T) {
        const int4 x = g_src[i];
        g_dst[i] = make_uint2((static_cast<uint32_t>(x.x) & 0xffffu) | (static_cast<uint32_t>(x.y) << 16),
                              (static_cast<uint32_t>(x.z) & 0xffffu) | (static_cast<uint32_t>(x.w) << 16));
      }
    }
    __syncthreads();
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
    for (int u = tid; u < n; u += T) {
      const int own = l_src[u];
      st.lab[u] = static_cast<uint8_t>(own);
      st.kown[u] = off[own] - 128 * static_cast<int>(st.g[static_cast<size_t>(own) * ld + u]);
      const int2 r = RescanBest2(st.g, ld, u, off, k, own);
      st.kbest[u] = r.x;
      st.kbound[u] = r.y;
    }
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  __syncthreads();

  unsigned long long applied = 0;
  int parity = 0;
  int from = -1, to = -1, moved = -1;
  bool from_empty = false;
  int empty = LowestEmpty(off, k);
  const uint32_t* prev_row = nullptr;
  const uint32_t lane_bit = 1u << lane;
  const Key key_base = (static_cast<Key>(1) << bits) << bits;

  while (true) {
    Key best = KeyTraits<Key>::kNone;
    uint32_t payload = 0;
    const bool fold = prev_row != nullptr;
    const int offf = fold ? off[from] : 0;
    const int offt = fold ? off[to] : 0;
    // warp-uniform trip count: the rescans below are warp-cooperative
    for (int base0 = tid - lane; base0 < n; base0 += U * T) {
      const int base = base0 + lane;
      int kb[U], ko[U], lbd[U], gf[U], gt[U];
      uint32_t rw[U];
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        const bool live = u < n;
        kb[i] = live ? st.kbest[u] : 0x7fffffff;
        ko[i] = live ? st.kown[u] : 0;
        lbd[i] = live ? st.kbound[u] : 0x7fffffff;
        rw[i] = live && fold ? prev_row[u >> 5] : 0u;
        gf[i] = live && fold ? st.g[static_cast<size_t>(from) * ld + u] : 0;
        gt[i] = live && fold ? st.g[static_cast<size_t>(to) * ld + u] : 0;
      }
      unsigned need = 0, chg = 0;  // bit i: rescan needed / cached keys changed
      if (fold) {
#pragma unroll
        for (int i = 0; i < U; ++i) {
          const int u = base + i * T;
          if (u >= n) continue;
          if (rw[i] & lane_bit) {
            st.g[static_cast<size_t>(from) * ld + u] = static_cast<uint16_t>(--gf[i]);
            st.g[static_cast<size_t>(to) * ld + u] = static_cast<uint16_t>(++gt[i]);
          }
          const int kb0 = kb[i], ko0 = ko[i], lb0 = lbd[i];
          if (FoldMove(u, offf - 128 * gf[i], offt - 128 * gt[i], from, to, moved, from_empty, kb[i], lbd[i],
                       ko[i])) {
            need |= 1u << i;
          }
          chg |= static_cast<unsigned>(kb[i] != kb0 || ko[i] != ko0 || lbd[i] != lb0) << i;
          if (u == moved) st.lab[u] = static_cast<uint8_t>(to);
        }
#pragma unroll
        for (int i = 0; i < U; ++i) {
          unsigned m = __ballot_sync(kAllLanes, (need >> i) & 1u);
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const int own_l = __shfl_sync(kAllLanes, ko[i] & 63, l);
            const int2 r = WarpRescan2(st.g, ld, base0 + l + i * T, off, k, own_l);
            if (lane == l) {
              kb[i] = r.x;
              lbd[i] = r.y;
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < U; ++i) {
        const int u = base + i * T;
        if (u >= n) continue;
        if ((chg | need) >> i & 1u) {
          st.kbest[u] = kb[i];
          st.kown[u] = ko[i];
          st.kbound[u] = lbd[i];
        }
        const int kbest = min(kb[i], empty >= 0 ? empty : 0x7fffffff);
        const int gain = (kbest >> 6) - (ko[i] >> 6) + 1;
        const Key mk = static_cast<Key>(static_cast<long long>(gain) * (1ll << bits)) + key_base + static_cast<Key>(u);
        if (mk < best) {
          best = mk;
          payload = static_cast<uint32_t>(ko[i] & 63) | (static_cast<uint32_t>(kbest & 63) << 8);
        }
      }
    }
    const MoveRecord<Key> m = BlockArgMin<Key, kWarps>(best, payload, s_records + parity * kWarps);
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
    from_empty = off[from] == from;
    empty = LowestEmpty(off, k);
    prev_row = a.gr.bits + static_cast<size_t>(moved) * pitch;
    objective += MoveDelta(m.key, bits);
    ++applied;
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
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

// The wide form (32767 < n <= 65536, int32 population G): state in the slot's rows of `next`, 64-bit keys.
template <int T>
__global__ void __launch_bounds__(T, 1) k_descent_incremental_wide(DescentArgs<int32_t> a) {
  DescentIncremental<T, false, int32_t, unsigned long long>(a, blockIdx.x);
}

// The same descent with the cached keys owned per thread: thread t owns vertices u = t + j T, j < V
// (n <= V T), and holds kbest, the second-best bound and kown of each (the label is kown & 63), in registers,
// or for V >= 16 in [V][T] shared-memory arrays that only their owner touches (read eight at a time).  A move then costs, per owned vertex, the two
// counter lanes `from` and `to` (one 16-bit load each, all of a thread's loads issued together) and the
// adjacency word; the counters stay in shared memory when k * n * 2 bytes fit, else in the slot's rows of
// `next` (L2).
template <int T, int V, bool kSmemG, bool kSmemKeys>
__device__ __forceinline__ void DescentIncrementalRegs(const DescentArgs<int16_t>& a, int slot) {
  constexpr int kWarps = T / kWarp;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;
  __shared__ MoveRecord<uint32_t> s_records[2 * kWarps];
  __shared__ int s_off[kWarps][kMaxK];

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

  // dynamic shared memory: [cached keys: best, bound, own, each V x T ints, when kSmemKeys] [counters when kSmemG]
  int* skb = reinterpret_cast<int*>(smem);
  int* slb = skb + V * T;
  int* sko = slb + V * T;
  unsigned char* after_keys = smem + (kSmemKeys ? static_cast<size_t>(V) * T * 3 * sizeof(int) : 0);
  uint16_t* g = kSmemG ? reinterpret_cast<uint16_t*>(after_keys)
                       : reinterpret_cast<uint16_t*>(a.next.g) + static_cast<size_t>(slot) * k * ld;
  int* off = s_off[warp];
  const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
  for (int c = lane; c < kMaxK; c += kWarp) off[c] = c < k ? 64 * sizes[c] + c : 0x3fffffff;
  __syncwarp();
  {
    const uint4* g_src = reinterpret_cast<const uint4*>(a.cur.g + static_cast<size_t>(w) * k * ld);
    uint4* g_dst = reinterpret_cast<uint4*>(g);
    for (size_t i = tid; i < static_cast<size_t>(k) * ld / 8; i += T) g_dst[i] = g_src[i];
  }
  __syncthreads();
  constexpr int VR = kSmemKeys ? 1 : V;  // cached keys held in registers
  int kb[VR], ko[VR], lbr[VR];
  unsigned valid = 0;
  {
    const uint8_t* l_src = a.cur.labels + static_cast<size_t>(w) * ld;
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const int u = tid + j * T;
      int2 b = make_int2(0, 0);
      int o = 0;
      if (u < n) {
        valid |= 1u << j;
        const int own = l_src[u];
        o = off[own] - 128 * static_cast<int>(g[static_cast<size_t>(own) * ld + u]);
        b = RescanBest2(g, ld, u, off, k, own);
      }
      if constexpr (kSmemKeys) {
        skb[j * T + tid] = b.x;
        slb[j * T + tid] = b.y;
        sko[j * T + tid] = o;
      } else {
        kb[j] = b.x;
        lbr[j] = b.y;
        ko[j] = o;
      }
    }
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;

  unsigned long long applied = 0;
  int parity = 0;
  int from = 0, to = 0, moved = -1;
  bool pending = false;
  bool from_empty = false;
  int empty = LowestEmpty(off, k);
  const uint32_t* prev_row = a.gr.bits;
  const uint32_t lane_bit = 1u << lane;
  const uint32_t key_base = (1u << bits) << bits;

  constexpr int kGroup = V < 8 ? V : 8;  // vertices whose loads are in flight together
  while (true) {
    uint32_t best = KeyTraits<uint32_t>::kNone;
    uint32_t payload = 0;
    const int offf = pending ? off[from] : 0;
    const int offt = pending ? off[to] : 0;
    const int empty_key = empty >= 0 ? empty : 0x7fffffff;
    // with the keys in shared memory nothing is indexed by j in registers: one group body, looped
#pragma unroll(kSmemKeys ? 1 : V / kGroup)
    for (int j0 = 0; j0 < V; j0 += kGroup) {
      uint32_t rw[kGroup];
      int gf[kGroup], gt[kGroup];
#pragma unroll
      for (int i = 0; i < kGroup; ++i) {
        const int u = tid + (j0 + i) * T;
        const bool live = pending && ((valid >> (j0 + i)) & 1);
        rw[i] = live ? prev_row[u >> 5] : 0u;
        gf[i] = live ? g[static_cast<size_t>(from) * ld + u] : 0;
        gt[i] = live ? g[static_cast<size_t>(to) * ld + u] : 0;
      }
      int ckb[kGroup], clb[kGroup], cko[kGroup];
      if constexpr (kSmemKeys) {
#pragma unroll
        for (int i = 0; i < kGroup; ++i) {
          ckb[i] = skb[(j0 + i) * T + tid];
          clb[i] = slb[(j0 + i) * T + tid];
          cko[i] = sko[(j0 + i) * T + tid];
        }
      }
      unsigned need = 0;  // bit i: rescan needed
      if (pending) {
#pragma unroll
        for (int i = 0; i < kGroup; ++i) {
          const int j = j0 + i;
          if (!((valid >> j) & 1)) continue;
          const int u = tid + j * T;
          int& kbj = kSmemKeys ? ckb[i] : kb[kSmemKeys ? 0 : j];
          int& lbj = kSmemKeys ? clb[i] : lbr[kSmemKeys ? 0 : j];
          int& koj = kSmemKeys ? cko[i] : ko[kSmemKeys ? 0 : j];
          if (rw[i] & lane_bit) {
            g[static_cast<size_t>(from) * ld + u] = static_cast<uint16_t>(--gf[i]);
            g[static_cast<size_t>(to) * ld + u] = static_cast<uint16_t>(++gt[i]);
          }
          if (FoldMove(u, offf - 128 * gf[i], offt - 128 * gt[i], from, to, moved, from_empty, kbj, lbj, koj)) {
            need |= 1u << i;
          }
        }
        // warp-cooperative rescans, one vertex at a time
#pragma unroll
        for (int i = 0; i < kGroup; ++i) {
          const int j = j0 + i;
          int& kbj = kSmemKeys ? ckb[i] : kb[kSmemKeys ? 0 : j];
          int& lbj = kSmemKeys ? clb[i] : lbr[kSmemKeys ? 0 : j];
          const int koj = kSmemKeys ? cko[i] : ko[kSmemKeys ? 0 : j];
          unsigned m = __ballot_sync(kAllLanes, (need >> i) & 1u);
          while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const int own_l = __shfl_sync(kAllLanes, koj & 63, l);
            const int2 r = WarpRescan2(g, ld, tid - lane + l + j * T, off, k, own_l);
            if (lane == l) {
              kbj = r.x;
              lbj = r.y;
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < kGroup; ++i) {
        const int j = j0 + i;
        if (!((valid >> j) & 1)) continue;
        const int u = tid + j * T;
        const int kbj = kSmemKeys ? ckb[i] : kb[kSmemKeys ? 0 : j];
        const int lbj = kSmemKeys ? clb[i] : lbr[kSmemKeys ? 0 : j];
        const int koj = kSmemKeys ? cko[i] : ko[kSmemKeys ? 0 : j];
        if constexpr (kSmemKeys) {
          if (pending) {  // cheaper than testing what changed: the three words are this thread's own
            skb[j * T + tid] = kbj;
            slb[j * T + tid] = lbj;
            sko[j * T + tid] = koj;
          }
        }
        const int kbest = min(kbj, empty_key);
        const int gain = (kbest >> 6) - (koj >> 6) + 1;
        const uint32_t mk = static_cast<uint32_t>(gain * (1 << bits)) + key_base + static_cast<uint32_t>(u);
        if (mk < best) {
          best = mk;
          payload = static_cast<uint32_t>(koj & 63) | (static_cast<uint32_t>(kbest & 63) << 8);
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
    from_empty = off[from] == from;
    empty = LowestEmpty(off, k);
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
#pragma unroll
  for (int j = 0; j < V; ++j) {
    if ((valid >> j) & 1) {
      const int o = kSmemKeys ? sko[j * T + tid] : ko[kSmemKeys ? 0 : j];
      dst[tid + j * T] = static_cast<uint8_t>(o & 63);
    }
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

template <int T, int V, bool kSmemG, bool kSmemKeys>
__global__ void __launch_bounds__(T, 1) k_descent_incremental_regs(DescentArgs<int16_t> a) {
  DescentIncrementalRegs<T, V, kSmemG, kSmemKeys>(a, blockIdx.x);
}

}  // namespace ccb
