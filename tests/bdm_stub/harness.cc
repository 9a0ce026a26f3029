// Test harness over the BioDynaMo drop-in adapter: builds stand-in agents,
// drives the adapter's reference-shaped drivers, solver classes, behaviours
// and energy the way the reference's application does, and returns the
// results through C entry points for the Python tests.
#include <cmath>
#include <memory>
#include <vector>

#include "agents/charged_antiparticle.h"
#include "amk_bdm_adapter.h"
#include "core/resource_manager.h"
#include "core/simulation.h"
#include "fields/penning_trap.h"

namespace {

struct Agents {
  std::vector<std::unique_ptr<bdm::ChargedAntiparticle>> parts;
  bdm::ResourceManager rm;
  Agents(long n, const double* x, const double* y, const double* z, const double* q) {
    for (long i = 0; i < n; ++i) {
      auto p = std::make_unique<bdm::ChargedAntiparticle>();
      p->position = bdm::Real3(x[i], y[i], z[i]);
      p->charge = q ? q[i] : 0.0;
      p->coulomb_force = bdm::Real3(NAN, NAN, NAN);
      p->uid.index = static_cast<uint64_t>(i);
      rm.agents.push_back(p.get());
      parts.push_back(std::move(p));
    }
  }
};

bdm::Simulation& Sim() {
  static bdm::Simulation sim;
  bdm::Simulation::Active() = &sim;
  return sim;
}

}  // namespace

// method 0 standard (param = cutoff), 1 Barnes-Hut (param = theta), 2 FMM
// (param = theta, order): every agent's Coulomb-force slot (NaN where the
// driver did not write).
extern "C" int harness_run(int method, long n, const double* x, const double* y, const double* z, const double* q,
                           const unsigned char* annihilated, double param, int order, double* fx, double* fy,
                           double* fz) {
  Agents a(n, x, y, z, q);
  for (long i = 0; i < n; ++i) a.parts[i]->annihilated = annihilated[i] != 0;
  try {
    if (method == 0) bdm::ComputeStandardCoulombForces(&a.rm, param);
    if (method == 1) bdm::ComputeBarnesHutCoulombForces(&a.rm, param);
    if (method == 2) bdm::ComputeFastMultipoleCoulombForces(&a.rm, order, param);
  } catch (...) {
    return -1;
  }
  for (long i = 0; i < n; ++i) {
    fx[i] = a.parts[i]->coulomb_force[0];
    fy[i] = a.parts[i]->coulomb_force[1];
    fz[i] = a.parts[i]->coulomb_force[2];
  }
  return 0;
}

// BarnesHutTree: Build over the sources, ComputeForce / ComputePotential for
// every source (self excluded) into f (3n) / phi (n), then for the extra
// point (px, py, pz) with charge pq into f_extra (3) / phi_extra; returns
// NumNodes (or -1).
extern "C" long harness_bh_class(long n, const double* x, const double* y, const double* z, const double* q,
                                 double theta, long leaf, double* f, double* phi, double px, double py, double pz,
                                 double pq, double* f_extra, double* phi_extra) {
  try {
    std::vector<bdm::BarnesHutTree::Source> s(static_cast<size_t>(n));
    for (long i = 0; i < n; ++i) {
      s[i].position = bdm::Real3(x[i], y[i], z[i]);
      s[i].charge = q[i];
    }
    bdm::BarnesHutTree tree(theta, static_cast<size_t>(leaf));
    tree.Build(s);
    for (long i = 0; i < n; ++i) {
      const bdm::Real3 fi = tree.ComputeForce(s[i].position, s[i].charge, static_cast<size_t>(i));
      for (int d = 0; d < 3; ++d) f[3 * i + d] = fi[d];
      phi[i] = tree.ComputePotential(s[i].position, static_cast<size_t>(i));
    }
    const bdm::Real3 e = tree.ComputeForce(bdm::Real3(px, py, pz), pq);
    for (int d = 0; d < 3; ++d) f_extra[d] = e[d];
    *phi_extra = tree.ComputePotential(bdm::Real3(px, py, pz));
    return static_cast<long>(tree.NumNodes());
  } catch (...) {
    return -1;
  }
}

// FastMultipoleSolver::Compute (forces into f, 3n) and
// ComputePotentialEnergy (into *energy).
extern "C" int harness_fmm_class(long n, const double* x, const double* y, const double* z, const double* q,
                                 int order, double theta, double* f, double* energy) {
  try {
    std::vector<bdm::FastMultipoleSolver::Source> s(static_cast<size_t>(n));
    for (long i = 0; i < n; ++i) {
      s[i].position = bdm::Real3(x[i], y[i], z[i]);
      s[i].charge = q[i];
    }
    bdm::FastMultipoleSolver solver(order, theta);
    std::vector<bdm::Real3> out;
    solver.ComputeForces(s, &out);
    for (long i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) f[3 * i + d] = out[i][d];
    *energy = solver.ComputePotentialEnergy(s);
    return 0;
  } catch (...) {
    return -1;
  }
}

// The reference application's step loop on the adapter: per step the
// standard Coulomb driver (cutoff), then LorentzForce, CyclotronCooling and
// AnnihilationInteraction Run() on every agent, then the standalone
// operation AmkRunQueuedBehaviours(). State after `steps` steps is written
// back into x..vz and alive; energies (time-centred, standard method with
// the same cutoff) after the last two steps into energy[0..7] (kinetic,
// trap, coulomb, active for each).
extern "C" int harness_steps(long n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const unsigned char* species, const double* q, const double* m, unsigned char* alive,
                             double b0, double voltage, double z0, double rho0, double dt, double cutoff,
                             double cooling_scale, double bath_temp, int annihilation, double contact_radius,
                             double probability, int seed, int steps, double* energy) {
  try {
    bdm::Simulation& sim = Sim();
    sim.param.physics.dt = dt;
    sim.param.physics.seed = seed;
    sim.param.stochastic.annihilation_enabled = annihilation != 0;
    sim.param.stochastic.contact_radius = contact_radius;
    sim.param.stochastic.annihilation_probability = probability;
    bdm::PenningTrapField field(b0, voltage, z0, rho0);
    Agents a(n, x, y, z, q);
    std::vector<std::unique_ptr<bdm::Behavior>> behaviours;
    std::vector<std::vector<bdm::Behavior*>> per_agent(static_cast<size_t>(n));
    for (long i = 0; i < n; ++i) {
      bdm::ChargedAntiparticle* p = a.parts[i].get();
      p->velocity = bdm::Real3(vx[i], vy[i], vz[i]);
      p->species = static_cast<bdm::ParticleSpecies>(species[i]);
      p->mass = m[i];
      p->coulomb_force = bdm::Real3(0.0, 0.0, 0.0);
      behaviours.push_back(std::make_unique<bdm::LorentzForce>(&field));
      per_agent[i].push_back(behaviours.back().get());
      behaviours.push_back(std::make_unique<bdm::CyclotronCooling>(&field, cooling_scale, bath_temp));
      per_agent[i].push_back(behaviours.back().get());
      if (annihilation) {
        behaviours.push_back(std::make_unique<bdm::AnnihilationInteraction>());
        per_agent[i].push_back(behaviours.back().get());
      }
    }
    bdm::EnergyComputationSettings es;
    es.method = bdm::ComputationMethod::kStandard;
    es.cutoff_radius = cutoff;
    bdm::EnergyHistory history;
    for (int s = 1; s <= steps; ++s) {
      sim.scheduler.simulated_steps = static_cast<uint64_t>(s - 1);  // steps completed before this one
      bdm::ComputeStandardCoulombForces(&a.rm, cutoff);
      for (long i = 0; i < n; ++i)
        if (!a.parts[i]->removed)
          for (bdm::Behavior* b : per_agent[i]) b->Run(a.parts[i].get());
      bdm::AmkRunQueuedBehaviours();
      if (s >= steps - 1) {
        const bdm::EnergyBreakdown e = bdm::ComputeTotalEnergy(&a.rm, field, es, &history);
        double* out = energy + 4 * (s - (steps - 1));
        out[0] = e.kinetic;
        out[1] = e.trap_potential;
        out[2] = e.energy_potential;
        out[3] = static_cast<double>(e.num_active_particles);
      }
    }
    for (long i = 0; i < n; ++i) {
      const bdm::ChargedAntiparticle& p = *a.parts[i];
      x[i] = p.position[0];
      y[i] = p.position[1];
      z[i] = p.position[2];
      vx[i] = p.velocity[0];
      vy[i] = p.velocity[1];
      vz[i] = p.velocity[2];
      alive[i] = p.annihilated ? 0 : 1;
    }
    return 0;
  } catch (...) {
    return -1;
  }
}

// CyclotronCooling::CoolingTime and IsAntiparticlePair through the adapter.
extern "C" double harness_cooling_time(double q, double m, double b) { return bdm::CyclotronCooling::CoolingTime(q, m, b); }
extern "C" int harness_is_pair(int a, int b) {
  return bdm::IsAntiparticlePair(static_cast<bdm::ParticleSpecies>(a), static_cast<bdm::ParticleSpecies>(b)) ? 1 : 0;
}
