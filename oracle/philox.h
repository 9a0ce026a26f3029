// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), restated for the
// CPU oracle. TEST INFRASTRUCTURE ONLY.
//
// Stream layout shared with the CUDA library (both restate the same rule):
//   key     = {seed (low 32 bits), tag}
//   cooling : tag 0xC0011u, counter {particle id, step lo, step hi, 0}
//             -> four uniforms -> Box-Muller -> three N(0,1) draws
//   annihilation : tag 0xA2211u, counter {owner id, partner id, step lo, step hi}
//             -> first word -> uniform in (0,1)
#ifndef AMK_ORACLE_PHILOX_H_
#define AMK_ORACLE_PHILOX_H_
#include <cmath>
#include <cstdint>

namespace orc {

constexpr uint32_t kTagCooling = 0xC0011u;
constexpr uint32_t kTagAnnihilation = 0xA2211u;

struct U32x4 {
  uint32_t v[4];
};

inline U32x4 Philox4x32(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2,
                        uint32_t c3) {
  const uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;
  const uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = static_cast<uint64_t>(kM0) * c0;
    const uint64_t p1 = static_cast<uint64_t>(kM1) * c2;
    const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += kW0;
    k1 += kW1;
  }
  return U32x4{{c0, c1, c2, c3}};
}

// Uniform in the open interval (0, 1) from one 32-bit word.
inline double U01(uint32_t w) { return (static_cast<double>(w) + 0.5) * 2.3283064365386963e-10; }

// The cooling stream's three N(0,1) draws for particle `id` at `step`:
// Box-Muller on the four uniforms of one Philox block.
inline void CoolingNormals(uint32_t seed, uint32_t id, uint64_t step, double* out3) {
  const double two_pi = 2.0 * 3.14159265358979323846;
  const U32x4 w = Philox4x32(seed, kTagCooling, id, static_cast<uint32_t>(step),
                             static_cast<uint32_t>(step >> 32), 0u);
  const double u1 = U01(w.v[0]), u2 = U01(w.v[1]);
  const double u3 = U01(w.v[2]), u4 = U01(w.v[3]);
  const double r1 = std::sqrt(-2.0 * std::log(u1));
  const double r2 = std::sqrt(-2.0 * std::log(u3));
  out3[0] = r1 * std::cos(two_pi * u2);
  out3[1] = r1 * std::sin(two_pi * u2);
  out3[2] = r2 * std::cos(two_pi * u4);
}

// The annihilation stream's uniform for the ordered pair owner -> partner.
inline double AnnihilationUniform(uint32_t seed, uint32_t owner, uint32_t partner, uint64_t step) {
  const U32x4 w = Philox4x32(seed, kTagAnnihilation, owner, partner, static_cast<uint32_t>(step),
                             static_cast<uint32_t>(step >> 32));
  return U01(w.v[0]);
}

}  // namespace orc
#endif
