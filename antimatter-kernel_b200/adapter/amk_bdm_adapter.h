// Drop-in declarations for a BioDynaMo application of the reference: the
// solver classes, behaviours and energy diagnostics of
//   interaction/barnes-hut.h, interaction/fast-multipole.h,
//   interaction/coulomb_interaction.h, forces/lorentz.h, forces/cooling.h,
//   interaction/annihilation.h, analysis/energy_analysis.h
// with the reference's public signatures, implemented by libamk on the GPU
// (amk_bdm_adapter.cc). Put this header in place of those seven and the
// adapter source in place of their .cc files; the reference's agent,
// field, parameter and species headers stay.
//
// The behaviours keep the reference's constructors and per-agent Run(), but
// Run() only queues its agent: BioDynaMo calls Run() agent by agent (in
// parallel), which on a GPU is one launch per particle. AmkRunQueuedBehaviours()
// -- registered as a standalone operation that runs after the agent
// operations of every step -- pushes, cools and annihilates all queued agents
// in one pass of the library's fused kernels and writes them back.
#pragma once

#include <cstddef>
#include <vector>

#include "agents/particle_species.h"
#include "core/behavior/behavior.h"
#include "core/container/math_array.h"
#include "core/real_t.h"
#include "params/interaction_params.h"

namespace bdm {

class Agent;
class ResourceManager;
class PenningTrapField;

// barnes-hut.h:28-74. Build() keeps the sources; the first query evaluates
// the library's tree walk for every source at once (forces per unit charge
// and potentials, each target excluding itself) and later queries for a
// source (self_index = its index) read that result. A query for any other
// point evaluates it as an extra zero-charge source.
class BarnesHutTree {
 public:
  struct Source {
    Real3 position;
    real_t charge = 0.0;
  };
  static constexpr size_t kNoSelf = static_cast<size_t>(-1);

  explicit BarnesHutTree(real_t theta, size_t leaf_capacity = 8);
  void Build(const std::vector<Source>& sources);
  Real3 ComputeForce(const Real3& position, real_t charge, size_t self_index = kNoSelf) const;
  real_t ComputePotential(const Real3& position, size_t self_index = kNoSelf) const;
  size_t NumNodes() const;

 private:
  void Evaluate() const;
  real_t theta_ = 0.5;
  size_t leaf_capacity_ = 8;
  std::vector<Source> sources_;
  mutable bool evaluated_ = false;
  mutable std::vector<double> ex_, ey_, ez_, phi_;  // field per unit charge (N/C), potential (V)
  mutable long nodes_ = 0;
};
void ComputeBarnesHutCoulombForces(ResourceManager* rm, real_t theta);

// fast-multipole.h:46-71.
class FastMultipoleSolver {
 public:
  struct Source {
    Real3 position;
    real_t charge = 0.0;
  };
  FastMultipoleSolver(int order, real_t theta, size_t leaf_capacity = 32);
  void ComputeForces(const std::vector<Source>& sources, std::vector<Real3>* forces) const;
  real_t ComputePotentialEnergy(const std::vector<Source>& sources) const;
  void Compute(const std::vector<Source>& sources, std::vector<Real3>* forces, double* potential_energy = nullptr) const;

 private:
  int order_ = 4;
  real_t theta_ = 0.5;
  size_t leaf_capacity_ = 32;
};
void ComputeFastMultipoleCoulombForces(ResourceManager* rm, int order, real_t theta);

// coulomb_interaction.h:10.
void ComputeStandardCoulombForces(ResourceManager* rm, real_t cutoff_radius);

// lorentz.h:15-35.
class LorentzForce : public Behavior {
  BDM_BEHAVIOR_HEADER(LorentzForce, Behavior, 1);

 public:
  LorentzForce() = default;
  explicit LorentzForce(const PenningTrapField* field);
  ~LorentzForce() override = default;
  void Run(Agent* agent) override;
  const PenningTrapField* GetField() const { return field_; }
  void SetField(const PenningTrapField* field) { field_ = field; }

 private:
  friend void AmkRunQueuedBehaviours();
  const PenningTrapField* field_ = nullptr;
  real_t dt_ = 1e-9;
  bool velocity_staggered_ = false;
};

// cooling.h:16-40.
class CyclotronCooling : public Behavior {
  BDM_BEHAVIOR_HEADER(CyclotronCooling, Behavior, 1);

 public:
  CyclotronCooling() = default;
  explicit CyclotronCooling(const PenningTrapField* field, real_t tau_scale = 1.0, real_t bath_temp_K = 0.0);
  ~CyclotronCooling() override = default;
  void Run(Agent* agent) override;
  static real_t CoolingTime(real_t charge, real_t mass, real_t b_mag);
  const PenningTrapField* GetField() const { return field_; }
  void SetField(const PenningTrapField* field) { field_ = field; }

 private:
  friend void AmkRunQueuedBehaviours();
  const PenningTrapField* field_ = nullptr;
  real_t tau_scale_ = 1.0;
  real_t bath_temp_K_ = 0.0;
};

// annihilation.h:11-20.
bool IsAntiparticlePair(ParticleSpecies a, ParticleSpecies b);
class AnnihilationInteraction : public Behavior {
  BDM_BEHAVIOR_HEADER(AnnihilationInteraction, Behavior, 1);

 public:
  AnnihilationInteraction() = default;
  ~AnnihilationInteraction() override = default;
  void Run(Agent* agent) override;
};

// Runs the queued behaviours of one scheduler step on the GPU: every agent
// queued by LorentzForce::Run gets the Boris push (with its own one-time
// back-stagger), the cyclotron-cooling kick when CyclotronCooling::Run
// queued it too (every queued agent must then carry the same cooling and
// field parameters), then the agents queued by AnnihilationInteraction::Run
// are matched under the library's deterministic rule (the reference visits
// agents in parallel with a shared random stream). Random streams are keyed
// by the agents' uids and the scheduler step being simulated
// (Scheduler::GetSimulatedSteps() + 1). Throws std::runtime_error with the
// library's message on failure.
void AmkRunQueuedBehaviours();

// energy_analysis.h:13-35.
struct EnergyBreakdown {
  real_t kinetic = 0.0;
  real_t trap_potential = 0.0;
  real_t energy_potential = 0.0;
  size_t num_active_particles = 0;
  real_t Total() const { return kinetic + trap_potential + energy_potential; }
};
struct EnergyHistory {
  bool has_previous = false;
  real_t prev_trap_potential = 0.0;
  real_t prev_coulomb_potential = 0.0;
};
EnergyBreakdown ComputeTotalEnergy(ResourceManager* rm, const PenningTrapField& field,
                                   const EnergyComputationSettings& energy, EnergyHistory* history = nullptr);

}  // namespace bdm
