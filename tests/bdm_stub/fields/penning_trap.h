// Test stand-in for the reference's PenningTrapField: the geometry getters
// the adapter reads (d = sqrt(z0^2/2 + rho0^2/4), penning_trap.cc:15-20).
#pragma once
#include <cmath>
#include "core/real_t.h"
namespace bdm {
class PenningTrapField {
 public:
  PenningTrapField(real_t b0, real_t voltage, real_t z0, real_t rho0)
      : b0_(b0), voltage_(voltage), d_(std::sqrt((z0 * z0) / 2.0 + (rho0 * rho0) / 4.0)) {}
  real_t GetB0() const { return b0_; }
  real_t GetTrapVoltage() const { return voltage_; }
  real_t GetCharacteristicDimension() const { return d_; }

 private:
  real_t b0_, voltage_, d_;
};
}  // namespace bdm
