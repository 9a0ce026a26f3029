// C entry points over the reference's own per-agent code, compiled in place
// from the reference tree (src/forces/lorentz.cc, src/forces/cooling.cc,
// src/interaction/annihilation.cc, src/interaction/coulomb_interaction.cc)
// against the BioDynaMo stand-ins in oracle/shim. TEST INFRASTRUCTURE ONLY:
// the checker for the CUDA library's push, cooling, annihilation and cutoff
// kernels; nothing in the product links it.
//
// A "world" holds ChargedAntiparticle stand-ins (uid = creation index), one
// LorentzForce and one CyclotronCooling instance per agent (the reference
// attaches one of each to every agent, antimatter-kernel.cc:93-94, so the
// back-stagger flag of LorentzForce is per agent), an AnnihilationInteraction,
// the trap field from the reference's own PenningTrapField, and the
// parameter groups the behaviours read.
//
// One step runs each behaviour over all agents in ascending uid order, phase
// by phase (all Lorentz pushes, then all cooling kicks, then all annihilation
// visits). That is the CUDA library's deterministic order; the reference's
// scheduler runs the three behaviours agent by agent in parallel, so its
// annihilation draws race (the stand-in Random replays the library's Philox
// draw for exactly the pair being considered).

#include <cstdint>
#include <memory>
#include <vector>

#include "agents/charged_antiparticle.h"
#include "core/resource_manager.h"
#include "core/simulation.h"
#include "fields/penning_trap.h"
#include "forces/cooling.h"
#include "forces/lorentz.h"
#include "interaction/annihilation.h"
#include "interaction/coulomb_interaction.h"
#include "params/physics_params.h"
#include "params/stochastic_params.h"

using bdm::ChargedAntiparticle;
using bdm::ParticleSpecies;
using bdm::Real3;

namespace {

struct World {
  bdm::PhysicsParams physics;
  bdm::StochasticParams stochastic;
  bdm::Param param;
  bdm::Random random;
  bdm::ResourceManager rm;
  std::unique_ptr<bdm::Environment> env;
  bdm::Simulation sim;
  std::unique_ptr<bdm::PenningTrapField> field;
  std::vector<std::unique_ptr<ChargedAntiparticle>> agents;
  std::vector<std::unique_ptr<bdm::LorentzForce>> lorentz;
  std::vector<std::unique_ptr<bdm::CyclotronCooling>> cooling;
  bdm::AnnihilationInteraction annihilation;
  uint32_t seed = 0;

  void Activate() {
    bdm::Simulation::Active() = &sim;
    bdm::g_shim_rng.seed = seed;
  }
};

}  // namespace

extern "C" {

// A world of n agents (species codes of particle_species.h) in the trap
// (b0, voltage, z0, rho0) with time step dt, cooling (tau_scale, bath
// temperature), annihilation parameters and the random-stream seed.
void* amkref_world_create(long n, const double* x, const double* y, const double* z, const double* vx,
                          const double* vy, const double* vz, const uint8_t* species, double b0,
                          double voltage, double z0, double rho0, double dt, double cooling_scale,
                          double bath_temp, int annihilation_enabled, double contact_radius,
                          double probability, uint32_t seed) {
  if (n < 0) return nullptr;
  auto* w = new World();
  w->physics.b0 = b0;
  w->physics.trap_voltage = voltage;
  w->physics.z0 = z0;
  w->physics.rho0 = rho0;
  w->physics.dt = dt;
  w->stochastic.annihilation_enabled = annihilation_enabled != 0;
  w->stochastic.contact_radius = contact_radius;
  w->stochastic.annihilation_probability = probability;
  w->param.Set(&w->physics);
  w->param.Set(&w->stochastic);
  w->env = std::make_unique<bdm::Environment>(&w->rm);
  w->sim.param = &w->param;
  w->sim.random = &w->random;
  w->sim.environment = w->env.get();
  w->seed = seed;
  w->Activate();
  w->field = std::make_unique<bdm::PenningTrapField>(
      bdm::PenningTrapField::MakeFromGeometry(b0, voltage, z0, rho0));
  for (long i = 0; i < n; ++i) {
    auto a = std::make_unique<ChargedAntiparticle>(Real3{{x[i], y[i], z[i]}},
                                                   static_cast<ParticleSpecies>(species[i]),
                                                   Real3{{vx[i], vy[i], vz[i]}});
    a->uid_ = static_cast<uint32_t>(i);
    w->rm.agents.push_back(a.get());
    w->agents.push_back(std::move(a));
    w->lorentz.push_back(std::make_unique<bdm::LorentzForce>(w->field.get()));
    w->cooling.push_back(std::make_unique<bdm::CyclotronCooling>(w->field.get(), cooling_scale, bath_temp));
  }
  return w;
}

void amkref_world_destroy(void* h) { delete static_cast<World*>(h); }

// Marks agents annihilated (alive[i] == 0) before a call.
int amkref_world_set_alive(void* h, const uint8_t* alive) {
  auto* w = static_cast<World*>(h);
  for (size_t i = 0; i < w->agents.size(); ++i)
    if (!alive[i]) w->agents[i]->MarkAnnihilated();
  return 0;
}

// Overwrites every agent's Coulomb-force slot.
int amkref_world_set_forces(void* h, const double* fx, const double* fy, const double* fz) {
  auto* w = static_cast<World*>(h);
  for (size_t i = 0; i < w->agents.size(); ++i) w->agents[i]->SetCoulombForce(Real3{{fx[i], fy[i], fz[i]}});
  return 0;
}

// ComputeStandardCoulombForces (coulomb_interaction.cc:23-80) on the world.
int amkref_world_coulomb_standard(void* h, double cutoff_radius) {
  auto* w = static_cast<World*>(h);
  w->Activate();
  bdm::ComputeStandardCoulombForces(&w->rm, cutoff_radius);
  return 0;
}

// One step of the behaviours on `step` (1-based, the random streams' step):
// LorentzForce::Run (lorentz.cc:37-71) on every agent, then
// CyclotronCooling::Run (cooling.cc:24-66), then AnnihilationInteraction::Run
// (annihilation.cc:21-61), each over agents in ascending uid order; a phase
// flag of 0 skips it. Returns the number of agents marked annihilated during
// the call.
long amkref_world_behaviours(void* h, uint64_t step, int lorentz, int cooling, int annihilation) {
  auto* w = static_cast<World*>(h);
  w->Activate();
  bdm::g_shim_rng.step = step;
  long before = 0;
  for (auto& a : w->agents) before += a->IsAnnihilated() ? 1 : 0;
  if (lorentz)
    for (size_t i = 0; i < w->agents.size(); ++i) w->lorentz[i]->Run(w->agents[i].get());
  if (cooling)
    for (size_t i = 0; i < w->agents.size(); ++i) {
      bdm::g_shim_rng.particle = w->agents[i]->uid_;
      bdm::g_shim_rng.gaus_calls = 0;
      w->cooling[i]->Run(w->agents[i].get());
    }
  if (annihilation)
    for (size_t i = 0; i < w->agents.size(); ++i) {
      bdm::g_shim_rng.particle = w->agents[i]->uid_;
      w->annihilation.Run(w->agents[i].get());
    }
  long after = 0;
  for (auto& a : w->agents) after += a->IsAnnihilated() ? 1 : 0;
  return after - before;
}

// The world's state: positions, velocities, alive flags and force slots
// (any output may be NULL).
int amkref_world_get(void* h, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                     uint8_t* alive, double* fx, double* fy, double* fz) {
  auto* w = static_cast<World*>(h);
  for (size_t i = 0; i < w->agents.size(); ++i) {
    const ChargedAntiparticle& a = *w->agents[i];
    if (x) x[i] = a.position_[0];
    if (y) y[i] = a.position_[1];
    if (z) z[i] = a.position_[2];
    if (vx) vx[i] = a.velocity_[0];
    if (vy) vy[i] = a.velocity_[1];
    if (vz) vz[i] = a.velocity_[2];
    if (alive) alive[i] = a.IsAnnihilated() ? 0 : 1;
    if (fx) fx[i] = a.coulomb_force_[0];
    if (fy) fy[i] = a.coulomb_force_[1];
    if (fz) fz[i] = a.coulomb_force_[2];
  }
  return 0;
}

// CyclotronCooling::CoolingTime (cooling.cc:16-22).
double amkref_cooling_time(double charge, double mass, double b_mag) {
  return bdm::CyclotronCooling::CoolingTime(charge, mass, b_mag);
}

// IsAntiparticlePair (annihilation.cc:12-19) on species codes.
int amkref_is_antiparticle_pair(int a, int b) {
  return bdm::IsAntiparticlePair(static_cast<ParticleSpecies>(a), static_cast<ParticleSpecies>(b)) ? 1 : 0;
}

}  // extern "C"
