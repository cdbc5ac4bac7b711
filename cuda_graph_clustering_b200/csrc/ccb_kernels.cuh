// Kernels of the PBILS iteration (one launch each, stream-ordered, no host round trip):
//
//   k_init_labels      initial population labels                       (cc_population_kernels.cuh:26-30)
//   k_rebuild          [perturb | copy | neighbourhood labels] + G = A*Z, sizes, f per slot
//                                                                      (cc_population_kernels.cuh:32-136)
//   k_descent          tournament select + steepest descent per slot   (cc_local_search.cuh:15-121,
//                                                                       cc_population_kernels.cuh:140-161)
//   k_record           record, stall / early stop, GWW source map      (cc_pbils_gpu.cu:325-345,
//                                                                       cc_pbils.hpp:69-78)
//   k_degrees          vertex degrees                                  (cc_population_kernels.cuh:82-89)
//
// The iteration is  descent(it) -> record(it) -> rebuild(perturb, it):  descent reads the current
// population and writes the next one, rebuild reads the next one and writes the current one back, so
// the two buffers never swap.  The GWW copy (cc_pbils_cpu.cpp:234-239) is folded into the rebuild:
// slot s perturbs the labels of its source src[s], which is s except for the worst `copies` slots,
// whose source is the matching winner.
#pragma once

#include <cstdint>

#include "ccb_device.cuh"

namespace ccb {

enum RebuildMode : int {
  kRebuildInPlace = 0,     // labels already in `cur`
  kRebuildPerturb = 1,     // cur[s] = perturb(next[src[s]])
  kRebuildCopy = 2,        // cur[s] = next[src[s]]            (no perturbation: k < 2 or p = 0)
  kRebuildNeighborhood = 3 // cur[s] = {v, N(v)} vs rest with v = first + s
};

static __global__ void k_mark_start(Control* ctl) {
  ctl->t0_ns = GlobalTimerNs();
}

static __global__ void k_clock(unsigned long long* t) { *t = GlobalTimerNs(); }

static __global__ void k_degrees(const uint32_t* __restrict__ bits, int n, int words, int pitch, int32_t* degrees) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const uint32_t* row = bits + static_cast<size_t>(v) * pitch;
  int d = 0;
  for (int w = 0; w < words; ++w) d += __popc(row[w]);
  degrees[v] = d;
}

// labels[slot][v] = InitialLabel(stream, slot * n + v, k) over a grid-stride loop.
static __global__ void k_init_labels(uint8_t* labels, int pop, int n, int ld, int k, uint64_t stream) {
  const long long total = static_cast<long long>(pop) * n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long slot = i / n;
    const int v = static_cast<int>(i - slot * n);
    labels[slot * ld + v] = static_cast<uint8_t>(InitialLabelOf(stream, static_cast<uint64_t>(i), k));
  }
}

// Rebuild of one slot per block.  Phase 1 writes the slot's labels (per mode), phase 2 packs one bit
// mask per cluster with warp ballots (masks live in a global scratch [slot][k][words], read back
// through L1), phase 3 gives each warp whole rows: lanes stride over the row's words, AND it with the
// masks of a chunk of clusters, count bits, and reduce across the warp in hardware.  The last
// cluster's row of G is the degree minus the others, so only k - 1 masks are intersected.
template <typename GainT>
struct RebuildArgs {
  GraphView gr;
  PopView<GainT> cur;
  const uint8_t* next_labels;
  const int32_t* src_map;
  uint32_t* masks;
  int k;
  int kpad;
  int ld;
  int mode;
  uint64_t stream;
  int iteration;
  float probability;
  int first;
  const Control* ctl;  // checked for the stop flag in the perturb / copy modes (may be null)
  int64_t* intra = nullptr;  // tiled form: labels, masks and sizes only; intra[slot] zeroed for the tiles
};

template <typename GainT, int kThreads>
__device__ __forceinline__ void RebuildBody(const RebuildArgs<GainT>& a, int slot) {
  const GraphView& gr = a.gr;
  const PopView<GainT>& cur = a.cur;
  // plain (coherent) loads: in the batched flow kernel these are written by other blocks of the same launch
  const uint8_t* next_labels = a.next_labels;
  const int32_t* src_map = a.src_map;
  uint32_t* __restrict__ masks = a.masks;
  const int k = a.k, kpad = a.kpad, ld = a.ld, mode = a.mode;
  const uint64_t stream = a.stream;
  const int iteration = a.iteration;
  const float probability = a.probability;
  const int first = a.first;
  const Control* ctl = a.ctl;
  constexpr int kWarps = kThreads / kWarp;
  constexpr int kChunk = 8;
  __shared__ int s_sizes[kMaxK];
  __shared__ long long s_sum[kWarps];
  if (ctl != nullptr && (mode == kRebuildPerturb || mode == kRebuildCopy) && ctl->stop) return;

  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int warp = tid / kWarp;
  const int n = gr.n;
  const int words = gr.words;
  uint8_t* labels = cur.labels + static_cast<size_t>(slot) * ld;

  if (mode == kRebuildPerturb || mode == kRebuildCopy) {
    const int src = src_map != nullptr ? src_map[slot] : slot;
    const uint8_t* from = next_labels + static_cast<size_t>(src) * ld;
    for (int v = tid; v < n; v += kThreads) {
      int l = from[v];
      if (mode == kRebuildPerturb) {
        l = PerturbLabelOf(stream, static_cast<uint64_t>(slot) * n + v, iteration, l, k, probability);
      }
      labels[v] = static_cast<uint8_t>(l);
    }
  } else if (mode == kRebuildNeighborhood) {
    const int center = first + slot;
    const uint32_t* crow = gr.bits + static_cast<size_t>(center) * gr.pitch;
    for (int v = tid; v < n; v += kThreads) labels[v] = (v == center || Bit(crow, v)) ? 0 : 1;
  }
  for (int c = tid; c < k; c += kThreads) s_sizes[c] = 0;
  __syncthreads();

  // Phase 2: masks of clusters 0 .. k-2 (and sizes of all clusters) by ballots over 32 labels.  Mask rows
  // have the graph's pitch; their pad words are never written, which is harmless because the matching
  // adjacency pad words are zero.
  const int pitch = gr.pitch;
  uint32_t* my_masks = masks + static_cast<size_t>(slot) * k * pitch;
  for (int w = warp; w < words; w += kWarps) {
    const int v = w * kWarp + lane;
    const int l = v < n ? labels[v] : -1;
    for (int c = 0; c < k; ++c) {
      const uint32_t m = __ballot_sync(kAllLanes, l == c);
      if (lane == (c % kWarp)) {
        if (c < k - 1) my_masks[static_cast<size_t>(c) * pitch + w] = m;
        if (m) atomicAdd(&s_sizes[c], __popc(m));
      }
    }
  }
  __syncthreads();
  if (a.intra != nullptr) {  // the tiled form computes G and f in k_rebuild_tiles / k_rebuild_finish
    for (int c = tid; c < k; c += kThreads) cur.sizes[static_cast<size_t>(slot) * kpad + c] = s_sizes[c];
    if (tid == 0) a.intra[slot] = 0;
    return;
  }

  // Phase 3: one row per thread.  The row streams in as 16-byte vectors (L1 keeps its line while the
  // thread walks it); every thread of the block reads the same mask vector at the same step, a broadcast.
  GainT* g = cur.g + static_cast<size_t>(slot) * k * ld;
  const int quads = pitch / 4;
  long long intra_twice = 0;
  for (int v = tid; v < n; v += kThreads) {
    const uint4* row = reinterpret_cast<const uint4*>(gr.bits + static_cast<size_t>(v) * pitch);
    int rest = gr.degrees[v];
    const int own = labels[v];
    int g_own = 0;
    for (int c0 = 0; c0 < k - 1; c0 += kChunk) {
      int acc[kChunk];
#pragma unroll
      for (int i = 0; i < kChunk; ++i) acc[i] = 0;
      for (int q = 0; q < quads; ++q) {
        const uint4 r = __ldg(row + q);
#pragma unroll
        for (int i = 0; i < kChunk; ++i) {
          if (c0 + i < k - 1) {
            const uint4 m = reinterpret_cast<const uint4*>(my_masks + static_cast<size_t>(c0 + i) * pitch)[q];
            acc[i] += __popc(r.x & m.x) + __popc(r.y & m.y) + __popc(r.z & m.z) + __popc(r.w & m.w);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < kChunk; ++i) {
        if (c0 + i < k - 1) {
          g[static_cast<size_t>(c0 + i) * ld + v] = static_cast<GainT>(acc[i]);
          rest -= acc[i];
          if (own == c0 + i) g_own = acc[i];
        }
      }
    }
    g[static_cast<size_t>(k - 1) * ld + v] = static_cast<GainT>(rest);
    intra_twice += (own == k - 1) ? rest : g_own;
  }
  const long long sum = BlockSum<kWarps>(intra_twice, s_sum);
  if (tid == 0) {
    long long pairs = 0;
    for (int c = 0; c < k; ++c) pairs += static_cast<long long>(s_sizes[c]) * (s_sizes[c] - 1) / 2;
    cur.f[slot] = gr.edges + pairs - sum;
  }
  for (int c = tid; c < k; c += kThreads) cur.sizes[static_cast<size_t>(slot) * kpad + c] = s_sizes[c];
}

template <typename GainT, int kThreads>
__global__ void __launch_bounds__(kThreads) k_rebuild(RebuildArgs<GainT> a) {
  RebuildBody<GainT, kThreads>(a, blockIdx.x);
}

// G = A*Z for every slot with each adjacency row read from memory once per rebuild (the one-block-per-slot
// form reads all n rows once per slot: at n = 65536 that is 512 MiB per slot).  A block stages a tile of
// kRows rows (one per warp) in shared memory, then walks the slots: warp w popcounts its row against the
// slot's cluster masks (read through L1, shared by the block's warps), writes G_c of its vertex for
// c < k - 1, derives G_{k-1} from the degree, and adds G_own to the slot's intra sum (one atomic per block
// and slot).  Runs after k_rebuild in its tiled form (labels, masks, sizes); k_rebuild_finish turns the
// intra sums into f.
struct RebuildTilesArgs {
  GraphView gr;
  const uint8_t* labels;  // [slot][ld]
  const uint32_t* masks;  // [slot][k][pitch]
  int32_t* g;             // [slot][k][ld]
  int64_t* intra;         // [slot]
  int count, k, ld;
  int mode;
  const Control* ctl;
};

template <int kThreads>
__global__ void __launch_bounds__(kThreads, 1) k_rebuild_tiles(RebuildTilesArgs a) {
  constexpr int kRows = kThreads / kWarp;
  extern __shared__ __align__(16) uint4 s_rows[];  // kRows x pitch words
  __shared__ long long s_part[kRows];
  if (a.ctl != nullptr && (a.mode == kRebuildPerturb || a.mode == kRebuildCopy) && a.ctl->stop) return;
  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int warp = tid / kWarp;
  const int n = a.gr.n;
  const int pitch = a.gr.pitch;
  const int quads = pitch / 4;
  const int r0 = blockIdx.x * kRows;
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.gr.bits) + static_cast<size_t>(r0) * quads;
    const int total = kRows * quads;
    for (int i = tid; i < total; i += kThreads) {
      const int row = r0 + i / quads;
      s_rows[i] = row < n ? src[i] : make_uint4(0u, 0u, 0u, 0u);
    }
  }
  __syncthreads();
  const int v = r0 + warp;
  const uint4* row = s_rows + static_cast<size_t>(warp) * quads;
  const int degree = v < n ? a.gr.degrees[v] : 0;
  for (int slot = 0; slot < a.count; ++slot) {
    long long own_g = 0;
    if (v < n) {
      const int own = a.labels[static_cast<size_t>(slot) * a.ld + v];
      const uint4* m = reinterpret_cast<const uint4*>(a.masks + static_cast<size_t>(slot) * a.k * pitch);
      int32_t* g = a.g + static_cast<size_t>(slot) * a.k * a.ld + v;
      int rest = degree;
      for (int c = 0; c < a.k - 1; ++c) {
        int acc = 0;
        for (int q = lane; q < quads; q += kWarp) {
          const uint4 r = row[q];
          const uint4 x = __ldg(m + static_cast<size_t>(c) * quads + q);
          acc += __popc(r.x & x.x) + __popc(r.y & x.y) + __popc(r.z & x.z) + __popc(r.w & x.w);
        }
        acc = __reduce_add_sync(kAllLanes, acc);
        if (lane == 0) g[static_cast<size_t>(c) * a.ld] = acc;
        rest -= acc;
        if (own == c) own_g = acc;
      }
      if (lane == 0) g[static_cast<size_t>(a.k - 1) * a.ld] = rest;
      if (own == a.k - 1) own_g = rest;
    }
    if (lane == 0) s_part[warp] = own_g;
    __syncthreads();
    if (tid == 0) {
      long long sum = 0;
#pragma unroll
      for (int w = 0; w < kRows; ++w) sum += s_part[w];
      if (sum != 0) atomicAdd(reinterpret_cast<unsigned long long*>(a.intra + slot), static_cast<unsigned long long>(sum));
    }
    __syncthreads();
  }
}

// f = m + sum_c C(size_c, 2) - (twice the intra-cluster edges) per slot, after k_rebuild_tiles.
template <typename GainT>
__global__ void k_rebuild_finish(PopView<GainT> cur, const int64_t* intra, int count, int k, int kpad, int64_t edges,
                                 int mode, const Control* ctl) {
  if (ctl != nullptr && (mode == kRebuildPerturb || mode == kRebuildCopy) && ctl->stop) return;
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  long long pairs = 0;
  for (int c = 0; c < k; ++c) {
    const long long sz = cur.sizes[static_cast<size_t>(slot) * kpad + c];
    pairs += sz * (sz - 1) / 2;
  }
  cur.f[slot] = edges + pairs - intra[slot];
}

// Steepest descent of one slot per block until no strictly improving single-vertex move remains.
//
// Thread t owns vertices u = t, t + T, t + 2T, ...  A move (v: from -> to) changes every vertex's
// h_c(u) = size_c - 2 G_c(u) for c in {from, to}; the gain of moving u from a to c is
// h_c - h_a + 1 (cc_math.hpp:75-77).  Per move each thread scans its vertices for its best (gain, u)
// with the target of u as payload, the block takes the minimum in one barrier (BlockArgMin), and
// every thread applies the move to the G entries of its own vertices from row v of the adjacency.
// Sizes live in a private copy per warp so that no second barrier is needed.
//
//   kSmemState: labels (1 B) and G of the slot sit in shared memory for the whole descent,
//               otherwise in the slot's rows of `next` (global memory, L2 resident).
//   kSmemRows:  the whole bitset is staged in shared memory (small n), otherwise rows come from L2.
template <typename GainT, typename Key, bool kSmemState, bool kSmemRows, int kThreads>
__global__ void __launch_bounds__(kThreads, 1) k_descent(DescentArgs<GainT> a) {
  constexpr int kWarps = kThreads / kWarp;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_winner;
  __shared__ int s_stop;

  const int slot = blockIdx.x;
  const int tid = threadIdx.x;
  const int lane = tid % kWarp;
  const int warp = tid / kWarp;
  const int n = a.gr.n;
  const int k = a.k;
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

  // Shared-memory carve-up (the host sizes it the same way): rows | G | labels | warp sizes | records.
  unsigned char* p = smem;
  const uint32_t* rows = a.gr.bits;
  if constexpr (kSmemRows) {
    uint32_t* srows = reinterpret_cast<uint32_t*>(p);
    const size_t row_words = static_cast<size_t>(n) * a.gr.pitch;
    const uint4* src = reinterpret_cast<const uint4*>(a.gr.bits);
    uint4* dst = reinterpret_cast<uint4*>(srows);
    for (size_t i = tid; i < row_words / 4; i += kThreads) dst[i] = __ldg(src + i);
    rows = srows;
    p += (row_words * 4 + 15) / 16 * 16;
  }
  GainT* g;
  uint8_t* lab;
  const size_t g_entries = static_cast<size_t>(k) * ld;
  if constexpr (kSmemState) {
    g = reinterpret_cast<GainT*>(p);
    p += (g_entries * sizeof(GainT) + 15) / 16 * 16;
    lab = p;
    p += (ld + 15) / 16 * 16;
  } else {
    g = a.next.g + static_cast<size_t>(slot) * g_entries;
    lab = a.next.labels + static_cast<size_t>(slot) * ld;
  }
  int* szw = reinterpret_cast<int*>(p);
  p += static_cast<size_t>(kWarps) * a.kpad * sizeof(int);
  MoveRecord<Key>* records = reinterpret_cast<MoveRecord<Key>*>((reinterpret_cast<uintptr_t>(p) + 15) / 16 * 16);

  {
    const uint4* gs = reinterpret_cast<const uint4*>(a.cur.g + static_cast<size_t>(w) * g_entries);
    uint4* gd = reinterpret_cast<uint4*>(g);
    for (size_t i = tid; i < g_entries * sizeof(GainT) / 16; i += kThreads) gd[i] = gs[i];
    const uint4* ls = reinterpret_cast<const uint4*>(a.cur.labels + static_cast<size_t>(w) * ld);
    uint4* ldst = reinterpret_cast<uint4*>(lab);
    for (int i = tid; i < ld / 16; i += kThreads) ldst[i] = ls[i];
    const int32_t* sizes = a.cur.sizes + static_cast<size_t>(w) * a.kpad;
    for (int i = tid; i < kWarps * k; i += kThreads) szw[(i / k) * a.kpad + i % k] = sizes[i % k];
  }
  long long objective = a.cur.f[w];
  const long long move_budget = objective;
  __syncthreads();

  int* sz = szw + warp * a.kpad;
  unsigned long long applied = 0;
  int parity = 0;
  while (true) {
    // Scan: best target of each owned vertex (smallest h, lowest cluster on ties), then the best
    // improving (gain, vertex) of the thread; vertices ascend, so strict < keeps the smallest vertex.
    Key best = KeyTraits<Key>::kNone;
    uint32_t payload = 0;
    for (int u = tid; u < n; u += kThreads) {
      const int from = lab[u];
      int h_from = 0;
      int h_best = 0x7fffffff;
      int to = 0;
      for (int c = 0; c < k; ++c) {
        const int h = sz[c] - 2 * static_cast<int>(g[static_cast<size_t>(c) * ld + u]);
        if (c == from) {
          h_from = h;
        } else if (h < h_best) {
          h_best = h;
          to = c;
        }
      }
      const int delta = h_best - h_from + 1;
      if (delta < 0) {
        const Key key = PackMove<Key>(delta, u, bits);
        if (key < best) {
          best = key;
          payload = static_cast<uint32_t>(from) | (static_cast<uint32_t>(to) << 8);
        }
      }
    }
    const MoveRecord<Key> m = BlockArgMin<Key, kWarps>(best, payload, records + parity * kWarps);
    if (m.key == KeyTraits<Key>::kNone) break;
    parity ^= 1;

    const int v = MoveVertex(m.key, bits);
    const int from = static_cast<int>(m.payload & 0xff);
    const int to = static_cast<int>(m.payload >> 8);
    if (lane == 0) {
      sz[from] -= 1;
      sz[to] += 1;
    }
    __syncwarp();
    if (v % kThreads == tid) lab[v] = static_cast<uint8_t>(to);
    const uint32_t* row = rows + static_cast<size_t>(v) * a.gr.pitch;
    GainT* g_from = g + static_cast<size_t>(from) * ld;
    GainT* g_to = g + static_cast<size_t>(to) * ld;
    for (int u = tid; u < n; u += kThreads) {
      if (Bit(row, u)) {
        g_from[u] -= 1;
        g_to[u] += 1;
      }
    }
    objective += MoveDelta(m.key, bits);
    ++applied;
    // Every accepted move lowers f by at least one and f >= 0, so f of the start state bounds the
    // number of moves; passing it means an inconsistent state, reported instead of looping on.
    if (static_cast<long long>(applied) > move_budget) {
      if (tid == 0) atomicExch(&a.ctl->error, kErrorMoveBound);
      break;
    }
  }

  if constexpr (kSmemState) {
    uint4* ldst = reinterpret_cast<uint4*>(a.next.labels + static_cast<size_t>(slot) * ld);
    const uint4* ls = reinterpret_cast<const uint4*>(lab);
    for (int i = tid; i < ld / 16; i += kThreads) ldst[i] = ls[i];
  }
  if (tid == 0) {
    a.next.f[slot] = objective;
    if (applied) atomicAdd(&a.ctl->moves, applied);
  }
}

enum RecordMode : int {
  kRecordInitial = 0,      // first offer (always taken), no iteration bookkeeping
  kRecordIteration = 1,    // record + Progress::Next + GWW source map
  kRecordNeighborhood = 2  // record only (strict improvement across batches)
};

struct RecordArgs {
  const int64_t* f;       // objective per slot
  const uint8_t* labels;  // labels per slot, leading dimension ld
  int ld;
  int n;
  int count;              // slots to consider
  Control* ctl;
  uint8_t* record_labels; // n labels of the record
  int mode;
  int iteration;
  int early_stop;
  int copies;             // GWW: WinnerCopies(gww, population) (cc_pbils_cpu.cpp:168)
  int32_t* src_map;       // GWW source of each slot's next member (null when copies == 0)
  int32_t* order;         // scratch: slots by (f, slot)
  TraceEntry* trace;      // progress log, one entry per iteration (may be null)
  unsigned long long time_limit_ns;  // 0 = none
};

// One block.  The record takes the first slot of minimum f on a strict improvement
// (cc_pbils_cpu.cpp:208-215); the stall counter and stop rule follow Progress::Next
// (cc_pbils.hpp:69-78); the GWW map ranks slots by (f, slot) as RankSlots does
// (cc_pbils_cpu.cpp:170-175) and sends the i-th best to the i-th worst for i < copies.
template <int kThreads>
__device__ __forceinline__ void RecordBody(const RecordArgs& a) {
  constexpr int kWarps = kThreads / kWarp;
  __shared__ long long s_f[kWarps];
  __shared__ int s_slot[kWarps];
  __shared__ int s_take;
  __shared__ int s_best;
  __shared__ int s_stop;
  const int tid = threadIdx.x;
  if (a.mode == kRecordIteration && a.ctl->stop) return;

  long long bf = 0x7fffffffffffffffll;
  int bs = 0x7fffffff;
  for (int s = tid; s < a.count; s += kThreads) {
    const long long f = a.f[s];
    if (f < bf) {
      bf = f;
      bs = s;
    }
  }
  for (int o = kWarp / 2; o > 0; o /= 2) {
    const long long of = __shfl_xor_sync(kAllLanes, bf, o);
    const int os = __shfl_xor_sync(kAllLanes, bs, o);
    if (of < bf || (of == bf && os < bs)) {
      bf = of;
      bs = os;
    }
  }
  if (tid % kWarp == 0) {
    s_f[tid / kWarp] = bf;
    s_slot[tid / kWarp] = bs;
  }
  __syncthreads();
  if (tid == 0) {
    long long f = s_f[0];
    int s = s_slot[0];
    for (int w = 1; w < kWarps; ++w) {
      if (s_f[w] < f || (s_f[w] == f && s_slot[w] < s)) {
        f = s_f[w];
        s = s_slot[w];
      }
    }
    Control* c = a.ctl;
    const int take = (a.mode == kRecordInitial) || !c->have_record || f < c->record_f;
    if (take) {
      c->record_f = f;
      c->have_record = 1;
      c->record_slot = s;
    }
    int stop = 0;
    if (a.mode == kRecordIteration) {
      c->iterations_done = a.iteration + 1;
      c->stall = take ? 0 : c->stall + 1;
      const unsigned long long now = GlobalTimerNs();
      if (a.trace != nullptr) a.trace[a.iteration] = TraceEntry{c->record_f, c->stall, 0, now - c->t0_ns};
      stop = c->stall >= a.early_stop || (a.time_limit_ns > 0 && now - c->t0_ns >= a.time_limit_ns);
      if (stop) c->stop = 1;
    }
    s_take = take;
    s_best = s;
    s_stop = stop;
  }
  __syncthreads();
  if (s_take) {
    const uint8_t* src = a.labels + static_cast<size_t>(s_best) * a.ld;
    for (int v = tid; v < a.n; v += kThreads) a.record_labels[v] = src[v];
  }
  if (a.mode != kRecordIteration || s_stop || a.copies <= 0) return;

  for (int s = tid; s < a.count; s += kThreads) {
    const long long f = a.f[s];
    int rank = 0;
    for (int t = 0; t < a.count; ++t) {
      const long long ft = a.f[t];
      rank += (ft < f) || (ft == f && t < s);
    }
    a.order[rank] = s;
    a.src_map[s] = s;
  }
  __syncthreads();
  for (int i = tid; i < a.copies; i += kThreads) a.src_map[a.order[a.count - 1 - i]] = a.order[i];
}

template <int kThreads>
__global__ void __launch_bounds__(kThreads) k_record(RecordArgs a) {
  RecordBody<kThreads>(a);
}

}  // namespace ccb
