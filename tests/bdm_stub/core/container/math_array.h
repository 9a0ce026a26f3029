// Test stand-in for BioDynaMo's Real3: three doubles, brace-initialised and
// indexed, which is all the adapter uses.
#pragma once
#include <array>
#include "core/real_t.h"
namespace bdm {
struct Real3 {
  std::array<real_t, 3> v;
  Real3() : v{0.0, 0.0, 0.0} {}
  Real3(real_t a, real_t b, real_t c) : v{a, b, c} {}
  real_t& operator[](int i) { return v[i]; }
  const real_t& operator[](int i) const { return v[i]; }
};
}  // namespace bdm
