// Test stand-in for the reference's PhysicsParams (the members the adapter reads).
#pragma once
#include "core/real_t.h"
namespace bdm {
struct PhysicsParams {
  int seed = 42;
  real_t dt = 1e-9;
};
}  // namespace bdm
