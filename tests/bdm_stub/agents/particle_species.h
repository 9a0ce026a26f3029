// Test stand-in for the reference's species codes (the enum values are the
// ones the reference and the C ABI use).
#pragma once
#include <cstdint>
namespace bdm {
enum class ParticleSpecies : uint8_t {
  kAntiproton = 0,
  kPositron = 1,
  kAntihydrogen = 2,
  kElectron = 3,
  kProton = 4,
  kAntihelium = 5,
};
}  // namespace bdm
