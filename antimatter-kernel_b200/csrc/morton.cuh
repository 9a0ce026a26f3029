// Morton-key helpers shared by the spatial kernels.
#pragma once
#include <cstdint>

namespace amk {

// Spreads the low 21 bits of v to every third bit.
__device__ __forceinline__ uint64_t spread3_21(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

// 63-bit key with x in bit 0 of each triple, then y, then z.
__device__ __forceinline__ uint64_t morton3_21(uint32_t x, uint32_t y, uint32_t z) {
  return spread3_21(x) | (spread3_21(y) << 1) | (spread3_21(z) << 2);
}

// Total order of doubles as unsigned integers (for atomicMin/Max).
__device__ __forceinline__ unsigned long long double_order_bits(double v) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double double_from_order_bits(unsigned long long b) {
  const unsigned long long r = (b >> 63) ? (b & 0x7fffffffffffffffull) : ~b;
  return __longlong_as_double(static_cast<long long>(r));
}

}  // namespace amk
