// Test stand-in for the reference's energy-method settings.
#pragma once
#include "core/real_t.h"
namespace bdm {
enum class ComputationMethod { kStandard, kBarnesHut, kFastMultipole };
struct EnergyComputationSettings {
  ComputationMethod method = ComputationMethod::kStandard;
  real_t cutoff_radius = 0.0;
  real_t barnes_hut_theta = 0.5;
  real_t fast_multipole_theta = 0.5;
  real_t fast_multipole_order = 4;
};
}  // namespace bdm
