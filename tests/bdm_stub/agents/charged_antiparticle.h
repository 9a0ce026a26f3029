// Test stand-in for the reference's agent type, reduced to the members the
// Coulomb drivers use.
#pragma once
#include "core/container/math_array.h"
namespace bdm {
class Agent {
 public:
  virtual ~Agent() = default;
};
class ChargedAntiparticle : public Agent {
 public:
  Real3 position;
  real_t charge = 0.0;
  bool annihilated = false;
  Real3 coulomb_force;
  const Real3& GetPosition() const { return position; }
  real_t GetCharge() const { return charge; }
  bool IsAnnihilated() const { return annihilated; }
  void SetCoulombForce(const Real3& f) { coulomb_force = f; }
};
inline ChargedAntiparticle* FastCast(Agent* a) { return static_cast<ChargedAntiparticle*>(a); }
}  // namespace bdm
