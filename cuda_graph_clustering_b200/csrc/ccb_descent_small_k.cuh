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

}  // namespace ccb
