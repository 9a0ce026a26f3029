// Test stand-in for the reference's agent type, reduced to the members the
// adapter's drivers, behaviours and energy use.
#pragma once
#include <cstdint>
#include "agents/particle_species.h"
#include "core/container/math_array.h"
namespace bdm {
struct AgentUid {
  uint64_t index = 0;
  uint64_t GetIndex() const { return index; }
};
class Agent {
 public:
  virtual ~Agent() = default;
  AgentUid uid;
  bool removed = false;
  AgentUid GetUid() const { return uid; }
  void RemoveFromSimulation() { removed = true; }
};
class ChargedAntiparticle : public Agent {
 public:
  Real3 position;
  Real3 velocity;
  real_t charge = 0.0;
  real_t mass = 0.0;
  ParticleSpecies species = ParticleSpecies::kElectron;
  bool annihilated = false;
  Real3 coulomb_force;
  const Real3& GetPosition() const { return position; }
  void SetPosition(const Real3& p) { position = p; }
  const Real3& GetVelocity() const { return velocity; }
  void SetVelocity(const Real3& v) { velocity = v; }
  real_t GetCharge() const { return charge; }
  real_t GetMass() const { return mass; }
  ParticleSpecies GetSpecies() const { return species; }
  bool IsAnnihilated() const { return annihilated; }
  void MarkAnnihilated() { annihilated = true; }
  const Real3& GetCoulombForce() const { return coulomb_force; }
  void SetCoulombForce(const Real3& f) { coulomb_force = f; }
};
inline ChargedAntiparticle* FastCast(Agent* a) { return static_cast<ChargedAntiparticle*>(a); }
}  // namespace bdm
