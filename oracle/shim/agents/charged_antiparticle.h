// Stand-in for the reference's BioDynaMo agent: only the members the solver
// drivers touch (position, charge, annihilation flag, Coulomb-force slot).
#ifndef AMK_SHIM_CHARGED_ANTIPARTICLE_H_
#define AMK_SHIM_CHARGED_ANTIPARTICLE_H_
#include "agents/particle_species.h"
#include "core/container/math_array.h"
namespace bdm {
class Agent {
 public:
  virtual ~Agent() = default;
};
class ChargedAntiparticle : public Agent {
 public:
  Real3 position_{{0.0, 0.0, 0.0}};
  real_t charge_ = 0.0;
  bool annihilated_ = false;
  Real3 coulomb_force_{{0.0, 0.0, 0.0}};
  const Real3& GetPosition() const { return position_; }
  real_t GetCharge() const { return charge_; }
  bool IsAnnihilated() const { return annihilated_; }
  void SetCoulombForce(const Real3& f) { coulomb_force_ = f; }
};
inline ChargedAntiparticle* FastCast(Agent* a) { return static_cast<ChargedAntiparticle*>(a); }
}  // namespace bdm
#endif
