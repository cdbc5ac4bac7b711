// G = A*Z on the tensor cores: the one-hot builder, the tcgen05 contraction kernel, and the recount entry
// point ccb_evaluate_labelings_tensor.  See ccb_rebuild_tensor.h for the data flow.
#include "ccb_rebuild_tensor.h"

#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "ccb.h"
#include "ccb_error.h"

namespace ccb {
namespace {

constexpr int kTileK = 128;                         // vertices u per pipeline stage: one 128-byte row
constexpr int kStages = 3;
constexpr int kSubTiles = 2;                        // 128-row accumulators per CTA, sharing each Z stage
constexpr int kMmaK = 32;                           // K of one kind::i8 MMA, in bytes
constexpr int kThreads = 192;                       // warp 0 TMA, warp 1 MMA + TMEM, warps 2..5 expand + epilogue
constexpr int kATileBytes = kTensorTileM * kTileK;  // int8 A sub-tile per stage: 16 KiB
constexpr int kBitsTileBytes = kTensorTileM * 16;   // adjacency words of a sub-tile per stage: 4 per row, 2 KiB
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // a wait gives up after 2 s ...
constexpr uint32_t kWaitSpinLimit = 1u << 24;               // ... or this many polls

// ---- PTX wrappers ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void BarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void BarArrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(bar)) : "memory");
}

__device__ __forceinline__ void BarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool BarTryWait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(SmemAddr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the phase of `bar` with the given parity.  Gives up (false) after kWaitLimitNs or kWaitSpinLimit
// polls, or as soon as another role of the CTA gave up (*abort, when given).
__device__ __noinline__ bool BarWait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  if (BarTryWait(bar, parity)) return true;
  const unsigned long long t0 = GlobalTimerNs();
  for (uint32_t spin = 1;; ++spin) {
    if (BarTryWait(bar, parity)) return true;
    if ((spin & 63) == 0) {
      if (abort != nullptr && *abort) return false;
      if (spin >= kWaitSpinLimit || GlobalTimerNs() - t0 > kWaitLimitNs) return false;
    }
  }
}

__device__ __forceinline__ void FenceBarrierInit() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Generic-proxy shared-memory writes become visible to the async proxy (the tensor cores' operand reads).
__device__ __forceinline__ void FenceProxyAsyncShared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 2-D tiled TMA load into this CTA's shared memory, completing on `bar` (no multicast).
__device__ __forceinline__ void TmaLoad2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(SmemAddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(SmemAddr(bar))
      : "memory");
}

__device__ __forceinline__ void TmemAlloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(slot)), "r"(cols)
               : "memory");
}
__device__ __forceinline__ void TmemRelinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void TmemDealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void TcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void TcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, unsigned 8-bit operands, int32 accumulators.
__device__ __forceinline__ void MmaI8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                      uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrives on `bar` once every MMA this thread issued so far has completed.
__device__ __forceinline__ void MmaCommit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(bar))
               : "memory");
}

// 16 consecutive 32-bit accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void TmemLoad16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzled layout: rows of 128 bytes,
// 8-row atoms of 1024 bytes (stride byte offset), 1024-byte aligned tile base.  Fields: start address >> 4
// (bits 0-13), leading byte offset 1 (unused for swizzled K-major), stride byte offset 1024 >> 4 (bits
// 32-45), descriptor version 1 (bits 46-47), base offset 0, layout 2 = 128-byte swizzle (bits 61-63).
// Advancing K by 32 bytes inside the atom adds 2 to the start field.
__device__ __forceinline__ uint64_t Sw128Desc(uint32_t smem_addr) {
  const uint64_t lo = ((smem_addr >> 4) & 0x3FFFu) | (1u << 16);
  const uint64_t hi = (1024u >> 4) | (1u << 14) | (2u << 29);
  return lo | (hi << 32);
}

// Instruction descriptor of kind::i8: int32 accumulator (bits 4-5 = 2), unsigned 8-bit A and B (bits 7-12 =
// 0), both K-major, N >> 3 (bits 17-22), M >> 4 (bits 24-28).
__host__ __device__ constexpr uint32_t IdescI8(int m, int n) {
  return (2u << 4) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

// Four adjacency bits -> four bytes 0/1 (bit j -> byte j): the multiply places bit j at bit 8j with no carries.
__device__ __forceinline__ uint32_t Spread4(uint32_t nibble) { return (nibble * 0x00204081u) & 0x01010101u; }

struct TensorArgs {
  int32_t* g;          // [col][ld], may be null
  int ld;
  int n;               // vertices (labels exist for v < n)
  int n_store;         // rows written per column
  int columns;         // live columns (count * k)
  int k;
  int bn;
  int ktiles;
  int tmem_cols;
  const void* labels;  // [slot][label_ld]
  int label_ld;
  int64_t* intra;      // [slot]
  int32_t* error;
  const Control* stop; // null: always run
};

template <typename LabelT>
__global__ void __launch_bounds__(kThreads, 1)
    k_rebuild_tensor(const __grid_constant__ CUtensorMap bits_map, const __grid_constant__ CUtensorMap z_map,
                     TensorArgs a) {
  if (a.stop != nullptr && a.stop->stop) return;  // uniform: before any barrier or TMEM use
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int bn = a.bn;
  uint8_t* s_a = base;                                        // [stage][sub][128 rows][128 B], swizzled
  uint8_t* s_b = s_a + kStages * kSubTiles * kATileBytes;     // [stage][bn rows][128 B], swizzled by TMA
  uint8_t* s_bits = s_b + kStages * bn * kTileK;              // [stage][sub][128 rows][16 B]
  uint64_t* full = reinterpret_cast<uint64_t*>(s_bits + kStages * kSubTiles * kBitsTileBytes);
  uint64_t* a_ready = full + kStages;
  uint64_t* empty = a_ready + kStages;
  uint64_t* accum = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x / kWarp;
  const int lane = threadIdx.x % kWarp;
  const int m0 = blockIdx.x * kTensorTileM * kSubTiles;
  const int n0 = blockIdx.y * bn;
  const int ktiles = a.ktiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      BarInit(&full[s], 1);
      BarInit(&a_ready[s], 4);
      BarInit(&empty[s], 1);
    }
    BarInit(accum, 1);
    *abort = 0;
    FenceBarrierInit();
  }
  if (warp == 1) {
    TmemAlloc(tmem_slot, a.tmem_cols);
    TmemRelinquish();
  }
  TcFenceBefore();
  __syncthreads();
  TcFenceAfter();
  const uint32_t tmem = *tmem_slot;

  auto give_up = [&]() {
    *abort = 1;
    atomicExch(a.error, kErrorWaitTimeout);
  };

  if (warp == 0) {
    if (lane == 0) {
      // TMA producer: stage s holds the adjacency words of K step kt and the Z block's bytes of it.
      const uint32_t bytes = kSubTiles * kBitsTileBytes + bn * kTileK;
      int issued = 0;
      for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt % kStages;
        if (kt >= kStages && !BarWait(&empty[s], ((kt / kStages) - 1) & 1, abort)) {
          give_up();
          break;
        }
        BarArriveExpectTx(&full[s], bytes);
#pragma unroll
        for (int sub = 0; sub < kSubTiles; ++sub) {  // a box past the last row reads zeros
          TmaLoad2d(s_bits + (s * kSubTiles + sub) * kBitsTileBytes, &bits_map, kt * 4, m0 + sub * kTensorTileM,
                    &full[s]);
        }
        TmaLoad2d(s_b + s * bn * kTileK, &z_map, kt * kTileK, n0, &full[s]);
        issued = kt + 1;
      }
      // drain: every copy issued has landed before the CTA may exit
      for (int kt = std::max(0, issued - kStages); kt < issued; ++kt) {
        if (!BarWait(&full[kt % kStages], (kt / kStages) & 1, nullptr)) give_up();
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = IdescI8(kTensorTileM, bn);
      const uint32_t a_base = SmemAddr(s_a);
      const uint32_t b_base = SmemAddr(s_b);
      for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt % kStages;
        const uint32_t par = (kt / kStages) & 1;
        if (!BarWait(&full[s], par, abort) || !BarWait(&a_ready[s], par, abort)) {
          give_up();
          break;
        }
        TcFenceAfter();
        const uint64_t bd = Sw128Desc(b_base + s * bn * kTileK);
#pragma unroll
        for (int sub = 0; sub < kSubTiles; ++sub) {  // accumulator `sub` in TMEM columns [sub * bn, (sub + 1) * bn)
          const uint64_t ad = Sw128Desc(a_base + (s * kSubTiles + sub) * kATileBytes);
#pragma unroll
          for (int j = 0; j < kTileK / kMmaK; ++j) {
            MmaI8(tmem + sub * bn, ad + 2 * j, bd + 2 * j, idesc, (kt > 0 || j > 0) ? 1u : 0u);
          }
        }
        MmaCommit(&empty[s]);  // the stage is free once these MMAs have read it
      }
      MmaCommit(accum);  // every MMA issued has completed: the accumulator is final (or, on abort, idle)
      if (!BarWait(accum, 0, nullptr)) give_up();
    }
    __syncwarp();
  } else {
    // Expansion: thread r turns row r's 128 adjacency bits of the stage into 128 bytes of the A tile, in the
    // 128-byte swizzle (16-byte chunk q of row r at chunk q ^ (r % 8) of its 1024-byte atom).
    const int r = (warp - 2) * kWarp + lane;
    for (int kt = 0; kt < ktiles; ++kt) {
      const int s = kt % kStages;
      if (!__all_sync(kAllLanes, BarWait(&full[s], (kt / kStages) & 1, abort))) {  // warp-uniform outcome
        if (lane == 0) give_up();
        break;
      }
#pragma unroll
      for (int sub = 0; sub < kSubTiles; ++sub) {
        const int t = s * kSubTiles + sub;
        const uint4 w = *reinterpret_cast<const uint4*>(s_bits + t * kBitsTileBytes + r * 16);
        const uint32_t words[4] = {w.x, w.y, w.z, w.w};
        uint8_t* row = s_a + t * kATileBytes + (r >> 3) * 1024 + (r & 7) * kTileK;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const uint32_t h = (words[q >> 1] >> ((q & 1) * 16)) & 0xFFFFu;
          uint4 out;
          out.x = Spread4(h & 0xFu);
          out.y = Spread4((h >> 4) & 0xFu);
          out.z = Spread4((h >> 8) & 0xFu);
          out.w = Spread4(h >> 12);
          *reinterpret_cast<uint4*>(row + ((q ^ (r & 7)) << 4)) = out;
        }
      }
      FenceProxyAsyncShared();
      __syncwarp();
      if (lane == 0) BarArrive(&a_ready[s]);
    }
    // Epilogue: warp w reads TMEM lanes 32 * (w % 4) .. +31, i.e. vertices m0 + 32 * (w % 4) + lane.
    const bool ok = __all_sync(kAllLanes, BarWait(accum, 0, nullptr));
    if (!ok && lane == 0) give_up();
    TcFenceAfter();
    const int quarter = warp & 3;
    const LabelT* labels = static_cast<const LabelT*>(a.labels);
    const bool write = ok && !*abort;
    for (int sub = 0; sub < kSubTiles; ++sub) {
      const int v = m0 + sub * kTensorTileM + quarter * kWarp + lane;
      const uint32_t lane_addr = tmem + (static_cast<uint32_t>(quarter * kWarp) << 16) + sub * bn;
      int cur_slot = -1, own = -1, part = 0;
      auto flush = [&]() {
        const unsigned total = __reduce_add_sync(kAllLanes, static_cast<unsigned>(part));
        if (lane == 0 && write && cur_slot >= 0 && total != 0) {
          atomicAdd(reinterpret_cast<unsigned long long*>(a.intra + cur_slot), static_cast<unsigned long long>(total));
        }
      };
      for (int c0 = 0; c0 < bn; c0 += 16) {
        uint32_t acc[16];
        TmemLoad16(lane_addr + c0, acc);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int col = n0 + c0 + i;
          if (col >= a.columns) break;
          const int slot = col / a.k;
          if (slot != cur_slot) {
            flush();
            cur_slot = slot;
            part = 0;
            own = v < a.n ? static_cast<int>(labels[static_cast<size_t>(slot) * a.label_ld + v]) : -1;
          }
          const int val = static_cast<int>(acc[i]);
          if (write && a.g != nullptr && v < a.n_store) a.g[static_cast<size_t>(col) * a.ld + v] = val;
          if (own == col - slot * a.k) part += val;
        }
      }
      flush();
    }
  }
  TcFenceBefore();
  __syncthreads();
  if (warp == 1) {
    TcFenceAfter();
    TmemDealloc(tmem, a.tmem_cols);
  }
}

template <typename LabelT>
__global__ void __launch_bounds__(256)
    k_build_z(const LabelT* __restrict__ labels, int label_ld, int n, int k, int kz, uint8_t* __restrict__ z,
              int32_t* __restrict__ sizes, int kpad, int64_t* __restrict__ intra, int32_t* __restrict__ bad,
              const Control* stop) {
  if (stop != nullptr && stop->stop) return;
  __shared__ int s_sizes[kMaxK];
  __shared__ int s_bad;
  const int slot = blockIdx.x;
  const int tid = threadIdx.x;
  const LabelT* lab = labels + static_cast<size_t>(slot) * label_ld;
  for (int c = tid; c < k; c += blockDim.x) s_sizes[c] = 0;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  const int words = kz / 4;
  uint32_t* rows = reinterpret_cast<uint32_t*>(z + static_cast<size_t>(slot) * k * kz);
  for (int i = tid; i < words; i += blockDim.x) {
    int l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int u = 4 * i + j;
      l[j] = u < n ? static_cast<int>(lab[u]) : -1;
      if (u < n && (l[j] < 0 || l[j] >= k)) {
        s_bad = 1;
        l[j] = -1;
      }
      if (sizes != nullptr && l[j] >= 0) atomicAdd(&s_sizes[l[j]], 1);
    }
    for (int c = 0; c < k; ++c) {
      rows[static_cast<size_t>(c) * words + i] = static_cast<uint32_t>(l[0] == c) |
                                                 (static_cast<uint32_t>(l[1] == c) << 8) |
                                                 (static_cast<uint32_t>(l[2] == c) << 16) |
                                                 (static_cast<uint32_t>(l[3] == c) << 24);
    }
  }
  __syncthreads();
  if (sizes != nullptr) {
    for (int c = tid; c < k; c += blockDim.x) sizes[static_cast<size_t>(slot) * kpad + c] = s_sizes[c];
  }
  if (tid == 0) {
    if (intra != nullptr) intra[slot] = 0;
    if (bad != nullptr) bad[slot] = s_bad;
  }
}

// f = m + sum_c C(size_c, 2) - intra per labeling (the recount's last step); -1 for a bad label, -2 when the
// contraction's bounded wait gave up.
__global__ void k_tensor_finish(const int32_t* sizes, int kpad, const int64_t* intra, const int32_t* bad,
                                const int32_t* error, int count, int k, long long edges, int64_t* f_out) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  long long pairs = 0;
  for (int c = 0; c < k; ++c) {
    const long long sz = sizes[static_cast<size_t>(slot) * kpad + c];
    pairs += sz * (sz - 1) / 2;
  }
  f_out[slot] = *error ? -2 : bad[slot] ? -1 : edges + pairs - intra[slot];
}

using EncodeTiledFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeTiledFn EncodeTiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess) {
      fn = reinterpret_cast<EncodeTiledFn>(p);
    }
  });
  return fn;
}

size_t TensorSmem(int bn) {
  return 1024 + static_cast<size_t>(kStages) * (kSubTiles * (kATileBytes + kBitsTileBytes) + bn * kTileK) +
         (3 * kStages + 1) * sizeof(uint64_t) + 16;
}

}  // namespace

bool PlanTensorRebuild(TensorRebuild& t, int n, int columns, const char** why) {
  if (n < kTensorTileM) {
    *why = "the tensor-core rebuild needs n >= 128";
    return false;
  }
  if (columns < 1) {
    *why = "no columns";
    return false;
  }
  t.n = n;
  t.words = (n + 31) / 32;
  t.ktiles = (t.words + 3) / 4;
  t.kz = t.ktiles * kTileK;
  t.columns = columns;
  const int blocks = (columns + kTensorMaxN - 1) / kTensorMaxN;
  t.bn = ((columns + blocks - 1) / blocks + 15) / 16 * 16;
  t.n_tiles = (columns + t.bn - 1) / t.bn;
  t.z_rows = t.n_tiles * t.bn;
  t.m_tiles = (n + kTensorTileM * kSubTiles - 1) / (kTensorTileM * kSubTiles);
  t.tmem_cols = 32;
  while (t.tmem_cols < kSubTiles * t.bn) t.tmem_cols *= 2;
  t.smem = TensorSmem(t.bn);
  return true;
}

cudaError_t EncodeTensorRebuild(TensorRebuild& t, const uint32_t* bits, int pitch_words, uint8_t* z) {
  EncodeTiledFn encode = EncodeTiled();
  if (encode == nullptr) return cudaErrorNotSupported;
  t.z = z;
  {
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(t.words), static_cast<cuuint64_t>(t.n)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(pitch_words) * 4};
    const cuuint32_t box[2] = {4, kTensorTileM};
    const cuuint32_t estr[2] = {1, 1};
    if (encode(&t.bits_map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint32_t*>(bits), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      return cudaErrorInvalidValue;
    }
  }
  {
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(t.kz), static_cast<cuuint64_t>(t.z_rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(t.kz)};
    const cuuint32_t box[2] = {kTileK, static_cast<cuuint32_t>(t.bn)};
    const cuuint32_t estr[2] = {1, 1};
    if (encode(&t.z_map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, z, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      return cudaErrorInvalidValue;
    }
  }
  return cudaSuccess;
}

template <typename LabelT>
cudaError_t LaunchBuildZ(const TensorRebuild& t, const LabelT* labels, int label_ld, int count, int k, int32_t* sizes,
                         int kpad, int64_t* intra, int32_t* bad, const Control* ctl, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  k_build_z<LabelT><<<count, 256, 0, st>>>(labels, label_ld, t.n, k, t.kz, t.z, sizes, kpad, intra, bad, ctl);
  return cudaGetLastError();
}

template <typename LabelT>
cudaError_t LaunchTensorRebuild(const TensorRebuild& t, int32_t* g, int ld, int n_store, int count, int k,
                                const LabelT* labels, int label_ld, int64_t* intra, int32_t* error, const Control* ctl,
                                cudaStream_t st) {
  const int columns = count * k;
  if (columns <= 0) return cudaSuccess;
  if (columns > t.z_rows) return cudaErrorInvalidValue;
  const cudaError_t attr = cudaFuncSetAttribute(k_rebuild_tensor<LabelT>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem);
  if (attr != cudaSuccess) return attr;
  TensorArgs a{};
  a.g = g;
  a.ld = ld;
  a.n = t.n;
  a.n_store = n_store;
  a.columns = columns;
  a.k = k;
  a.bn = t.bn;
  a.ktiles = t.ktiles;
  a.tmem_cols = t.tmem_cols;
  a.labels = labels;
  a.label_ld = label_ld;
  a.intra = intra;
  a.error = error;
  a.stop = ctl;
  const dim3 grid(t.m_tiles, (columns + t.bn - 1) / t.bn);
  k_rebuild_tensor<LabelT><<<grid, kThreads, t.smem, st>>>(t.bits_map, t.z_map, a);
  return cudaGetLastError();
}

template cudaError_t LaunchBuildZ<uint8_t>(const TensorRebuild&, const uint8_t*, int, int, int, int32_t*, int, int64_t*,
                                           int32_t*, const Control*, cudaStream_t);
template cudaError_t LaunchTensorRebuild<uint8_t>(const TensorRebuild&, int32_t*, int, int, int, int, const uint8_t*,
                                                  int, int64_t*, int32_t*, const Control*, cudaStream_t);

}  // namespace ccb

using namespace ccb;

extern "C" {

int ccb_evaluate_labelings_tensor(const uint32_t* bits, uint32_t n, uint32_t words_per_row, uint64_t edges, int32_t k,
                                  int32_t count, const int32_t* labels, int64_t* f_out, int32_t* sizes_out,
                                  int32_t* g_out, void* stream) {
  auto report = [](int status, const std::string& message) {
    SetLastError(message);
    return status;
  };
  if (k < 1 || k > CCB_MAX_CLUSTERS) return report(CCB_ERR_INVALID, "k must be in [1, 64]");
  if (count < 0) return report(CCB_ERR_INVALID, "count must be >= 0");
  if (n > (uint32_t)CCB_MAX_VERTICES_WIDE) return report(CCB_ERR_INVALID, "n exceeds 1048576");
  if (count == 0) return report(CCB_OK, "");
  if (bits == nullptr || labels == nullptr || f_out == nullptr) return report(CCB_ERR_INVALID, "null pointer");
  if (words_per_row < (n + 31) / 32) return report(CCB_ERR_INVALID, "words_per_row < ceil(n / 32)");
  if (words_per_row % 4 != 0 || reinterpret_cast<uintptr_t>(bits) % 16 != 0) {
    return report(CCB_ERR_INVALID, "the tensor-core recount needs 16-byte aligned rows (words_per_row % 4 == 0)");
  }
  if ((long long)count * k > (1 << 24)) return report(CCB_ERR_INVALID, "count * k exceeds 16777216");
  TensorRebuild t;
  const char* why = nullptr;
  if (!PlanTensorRebuild(t, (int)n, count * k, &why)) return report(CCB_ERR_INVALID, why);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int kpad = (k + 3) / 4 * 4;
  const size_t z_bytes = (size_t)t.z_rows * t.kz;
  const size_t sizes_bytes = sizes_out ? 0 : (size_t)count * kpad * 4;
  const size_t scratch = z_bytes + (size_t)count * 8 + (size_t)count * 4 + 16 + sizes_bytes;
  uint8_t* buf = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&buf), scratch, st);
  if (e != cudaSuccess) return report(CCB_ERR_DEVICE_MEMORY, cudaGetErrorString(e));
  uint8_t* z = buf;
  int64_t* intra = reinterpret_cast<int64_t*>(buf + z_bytes);  // z_bytes is a multiple of 128
  int32_t* bad = reinterpret_cast<int32_t*>(intra + count);
  int32_t* error = bad + count;
  int32_t* sizes = sizes_out ? sizes_out : error + 4;
  const int sizes_ld = sizes_out ? k : kpad;
  auto fail = [&](cudaError_t err) {
    cudaFreeAsync(buf, st);
    return report(CCB_ERR_CUDA, cudaGetErrorString(err));
  };
  if ((e = cudaMemsetAsync(z + (size_t)count * k * t.kz, 0, z_bytes - (size_t)count * k * t.kz, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(error, 0, 4, st)) != cudaSuccess) {
    return fail(e);
  }
  if ((e = EncodeTensorRebuild(t, bits, (int)words_per_row, z)) != cudaSuccess) return fail(e);
  const int label_ld = (int)n;
  k_build_z<int32_t><<<count, 256, 0, st>>>(labels, label_ld, (int)n, k, t.kz, z, sizes, sizes_ld, intra, bad, nullptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  if ((e = LaunchTensorRebuild<int32_t>(t, g_out, (int)n, (int)n, count, k, labels, label_ld, intra, error, nullptr,
                                        st)) != cudaSuccess) {
    return fail(e);
  }
  k_tensor_finish<<<(count + 127) / 128, 128, 0, st>>>(sizes, sizes_ld, intra, bad, error, count, k, (long long)edges,
                                                       f_out);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  cudaFreeAsync(buf, st);
  return report(CCB_OK, "");
}

}  // extern "C"
