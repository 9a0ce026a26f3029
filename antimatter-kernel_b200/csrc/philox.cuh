// Philox4x32-10 (Salmon et al., SC'11) for the device and the host.
//
// Stream layout (the same rule the tests restate independently):
//   key = {seed, tag}
//   cooling noise:      tag 0xC0011, counter {particle id, step lo, step hi, 0}
//                       -> 4 uniforms -> 2 Box-Muller pairs -> 3 normals used
//   annihilation draw:  tag 0xA2211, counter {owner id, partner id, step lo, step hi}
//                       -> word 0 -> uniform in (0, 1)
//   cloud generators:   tag 0x1C100 + generator, counter {particle id, attempt, 0, 0}
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define AMK_HD inline
#else
#define AMK_HD __host__ __device__ __forceinline__
#endif

namespace amk {

constexpr uint32_t kTagCooling = 0xC0011u;
constexpr uint32_t kTagAnnihilation = 0xA2211u;
constexpr uint32_t kTagCloud = 0x1C100u;

struct Philox4 {
  uint32_t w[4];
};

AMK_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

AMK_HD Philox4 philox4x32(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2,
                          uint32_t c3) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = mulhi32(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = mulhi32(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  Philox4 r;
  r.w[0] = c0;
  r.w[1] = c1;
  r.w[2] = c2;
  r.w[3] = c3;
  return r;
}

// Uniform in (0, 1) from one word: (w + 1/2) / 2^32.
AMK_HD double u01(uint32_t w) { return (static_cast<double>(w) + 0.5) * 2.3283064365386963e-10; }

}  // namespace amk
