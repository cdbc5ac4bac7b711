// Packed 16-bit counter vectors shared by the K <= 8 descents (ccb_descent_registers.cuh,
// ccb_descent_stream.cuh): KP = 2, 4 or 8 lanes in one 4-, 8- or 16-byte vector.
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

// L2 eviction priorities for state that streams from global memory (PTX createpolicy + .L2::cache_hint): the
// slots' packed vectors are re-read every move and should stay in L2 (evict_last), while bitset rows are read
// once per move at random and should leave first (evict_first).  Hints only: the values read and written are
// the same as with plain accesses.  The accesses are volatile so that a load is never hoisted out of the move
// loop or merged with the same address's load of another move.
__device__ __forceinline__ uint64_t L2PolicyEvictLast() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t L2PolicyEvictFirst() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint32_t LoadL2Hint(const uint32_t* a, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol) : "memory");
  return v;
}
__device__ __forceinline__ uint2 LoadL2Hint(const uint2* a, uint64_t pol) {
  uint2 v;
  asm volatile("ld.global.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(a), "l"(pol)
               : "memory");
  return v;
}
__device__ __forceinline__ uint4 LoadL2Hint(const uint4* a, uint64_t pol) {
  uint4 v;
  asm volatile("ld.global.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(a), "l"(pol) : "memory");
  return v;
}
__device__ __forceinline__ void StoreL2Hint(uint32_t* a, uint32_t v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.u32 [%0], %1, %2;" :: "l"(a), "r"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void StoreL2Hint(uint2* a, uint2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.u32 [%0], {%1, %2}, %3;" :: "l"(a), "r"(v.x), "r"(v.y), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void StoreL2Hint(uint4* a, uint4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.u32 [%0], {%1, %2, %3, %4}, %5;"
               :: "l"(a), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "l"(pol) : "memory");
}

}  // namespace ccb
