// Stand-in for the reference's BioDynaMo agent (TEST INFRASTRUCTURE ONLY):
// the members the reference's solver drivers and behaviours touch, over
// plain fields. `uid_` is the agent's creation index, which the stand-in
// Random and Environment use to replay the CUDA library's random streams
// and neighbour order.
#ifndef AMK_SHIM_CHARGED_ANTIPARTICLE_H_
#define AMK_SHIM_CHARGED_ANTIPARTICLE_H_
#include <cstdint>
#include "agents/particle_species.h"
#include "core/container/math_array.h"
namespace bdm {
class Agent {
 public:
  virtual ~Agent() = default;
  uint32_t uid_ = 0;
  Real3 position_{{0.0, 0.0, 0.0}};
  bool removed_ = false;
  const Real3& GetPosition() const { return position_; }
  void SetPosition(const Real3& p) { position_ = p; }
  void RemoveFromSimulation() { removed_ = true; }
};
class ChargedAntiparticle : public Agent {
 public:
  ChargedAntiparticle() = default;
  ChargedAntiparticle(const Real3& position, ParticleSpecies species, const Real3& velocity)
      : velocity_(velocity), species_(species) {
    position_ = position;
    const SpeciesProperties props = GetDefaultSpeciesProperties(species);
    mass_ = props.mass;
    charge_ = props.charge;
  }
  Real3 velocity_{{0.0, 0.0, 0.0}};
  real_t mass_ = 0.0;
  real_t charge_ = 0.0;
  ParticleSpecies species_ = ParticleSpecies::kElectron;
  bool annihilated_ = false;
  Real3 coulomb_force_{{0.0, 0.0, 0.0}};
  const Real3& GetVelocity() const { return velocity_; }
  void SetVelocity(const Real3& v) { velocity_ = v; }
  real_t GetMass() const { return mass_; }
  real_t GetCharge() const { return charge_; }
  ParticleSpecies GetSpecies() const { return species_; }
  bool IsAnnihilated() const { return annihilated_; }
  void MarkAnnihilated() { annihilated_ = true; }
  const Real3& GetCoulombForce() const { return coulomb_force_; }
  void SetCoulombForce(const Real3& f) { coulomb_force_ = f; }
};
inline ChargedAntiparticle* FastCast(Agent* a) { return static_cast<ChargedAntiparticle*>(a); }
}  // namespace bdm
#endif
