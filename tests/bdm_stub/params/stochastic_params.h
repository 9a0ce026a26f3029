// Test stand-in for the reference's StochasticParams.
#pragma once
#include "core/real_t.h"
namespace bdm {
struct StochasticParams {
  bool annihilation_enabled = false;
  real_t contact_radius = 1e-9;
  real_t annihilation_probability = 0.1;
};
}  // namespace bdm
