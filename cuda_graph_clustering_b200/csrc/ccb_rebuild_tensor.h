// G = A*Z on the tensor cores (tcgen05, kind::i8, int32 accumulators in TMEM), fed by TMA.
//
// The popcount rebuild (cuda/cc_population_kernels.cuh:44-136 in the reference; k_rebuild / k_rebuild_tiles
// here) counts, for every slot s, cluster c and vertex v, the neighbours of v labelled c:
// G[s][c][v] = sum_u A[v][u] * Z[s*k+c][u] with Z the one-hot labels.  Over the whole population that is
// one dense contraction with M = n (vertices v), N = pop*k (slot-cluster columns), K = n (vertices u) and
// 0/1 operands, exact in int32.  Here:
//   k_build_z       writes Z as uint8 rows [column][kz] (kz = ceil(ceil(n/32)/4) * 128 bytes, zero past n);
//   k_rebuild_tensor one CTA per 256-vertex tile of v (two 128-row accumulators in TMEM) and block of up to
//                   256 columns: TMA brings the two sub-tiles' adjacency words (2 KiB each per 128 u) and the Z
//                   block (128-byte swizzle) into a 3-stage shared-memory pipeline; four warps expand the bits
//                   into int8 rows in the UMMA 128-byte swizzled K-major layout; one thread issues
//                   tcgen05.mma kind::i8 (M 128, N <= 256, K 32) for both sub-tiles against the same Z stage, so
//                   each Z byte crossing from L2 serves 256 rows; the epilogue reads the accumulators
//                   (tcgen05.ld) and writes G and each slot's intra-cluster sum sum_v G[s][label_s(v)][v].
// Every mbarrier wait is bounded (time and spins); one that gives up sets *error = kErrorWaitTimeout, the
// kernel drains its own copies and MMAs, frees its TMEM and returns.  Tensor maps cover this GPU's memory
// only; no load uses cluster multicast.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "ccb_device.cuh"

namespace ccb {

constexpr int kTensorTileM = 128;  // vertices v per accumulator (one TMEM lane each); a CTA holds two
constexpr int kTensorMaxN = 256;   // columns per CTA (one MMA's N)

struct TensorRebuild {
  CUtensorMap bits_map;   // adjacency rows: uint32, box 4 words x 128 rows, no swizzle
  CUtensorMap z_map;      // one-hot Z: uint8 [z_rows][kz], box 128 bytes x bn rows, 128-byte swizzle
  uint8_t* z = nullptr;   // device, z_rows * kz bytes (rows >= the live columns stay zero)
  int n = 0;              // vertices
  int words = 0;          // meaningful words per adjacency row, ceil(n / 32)
  int ktiles = 0;         // K steps of 128 vertices, ceil(words / 4)
  int kz = 0;             // bytes per Z row, ktiles * 128
  int columns = 0;        // columns planned for (count * k)
  int bn = 0;             // columns per CTA, a multiple of 16, <= 256
  int n_tiles = 0;        // column blocks for `columns`
  int z_rows = 0;         // n_tiles * bn
  int m_tiles = 0;        // ceil(n / 256)
  int tmem_cols = 0;      // power of two >= 2 * bn (and >= 32)
  size_t smem = 0;        // dynamic shared memory per CTA
};

// Tile plan for n vertices and `columns` output columns; false (with a reason) when the path does not apply.
bool PlanTensorRebuild(TensorRebuild& t, int n, int columns, const char** why);
// Encodes both tensor maps: `bits` rows of `pitch_words` words (16-byte aligned rows), `z` of z_rows * kz bytes.
cudaError_t EncodeTensorRebuild(TensorRebuild& t, const uint32_t* bits, int pitch_words, uint8_t* z);

// Z rows of `count` labelings (label row s at labels + s * label_ld) for k clusters.  Optional: cluster sizes
// [count][kpad], a bad-label flag per labeling, intra[count] zeroed.  With ctl non-null nothing runs once
// ctl->stop is set (the caller passes it in the iteration's perturb / copy modes, like the other rebuild kernels).
template <typename LabelT>
cudaError_t LaunchBuildZ(const TensorRebuild& t, const LabelT* labels, int label_ld, int count, int k, int32_t* sizes,
                         int kpad, int64_t* intra, int32_t* bad, const Control* ctl, cudaStream_t st);

// G[col][v] (col = s * k + c, row stride ld; g may be null) for v < n_store and col < count * k, plus
// intra[s] += sum_v G[s][label_s(v)][v].  error: device int32, set to kErrorWaitTimeout if a wait gave up.
template <typename LabelT>
cudaError_t LaunchTensorRebuild(const TensorRebuild& t, int32_t* g, int ld, int n_store, int count, int k,
                                const LabelT* labels, int label_ld, int64_t* intra, int32_t* error,
                                const Control* ctl, cudaStream_t st);

}  // namespace ccb
