// Test stand-in for BioDynaMo's Param: the three parameter groups the
// adapter reads, returned by Get<T>().
#pragma once
#include "params/interaction_params.h"
#include "params/physics_params.h"
#include "params/stochastic_params.h"
namespace bdm {
class Param {
 public:
  PhysicsParams physics;
  StochasticParams stochastic;
  template <typename T>
  const T* Get() const;
};
template <>
inline const PhysicsParams* Param::Get<PhysicsParams>() const { return &physics; }
template <>
inline const StochasticParams* Param::Get<StochasticParams>() const { return &stochastic; }
}  // namespace bdm
