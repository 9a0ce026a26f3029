// Drop-in replacement of the reference's solver, behaviour and energy
// sources for a BioDynaMo application (declarations in amk_bdm_adapter.h,
// which replaces the reference's headers of the same classes), computed by
// libamk on the GPU:
//   ComputeStandardCoulombForces / ComputeBarnesHutCoulombForces /
//   ComputeFastMultipoleCoulombForces      (coulomb_interaction.h:10,
//                                           barnes-hut.h:76, fast-multipole.h:73)
//   BarnesHutTree, FastMultipoleSolver     (barnes-hut.h:28-74, fast-multipole.h:46-71)
//   LorentzForce, CyclotronCooling,
//   AnnihilationInteraction                (lorentz.h:15-35, cooling.h:16-40,
//                                           annihilation.h:11-20)
//   ComputeTotalEnergy                     (energy_analysis.h:35)
//
// Build it into the application in place of coulomb_interaction.cc,
// barnes-hut.cc, fast-multipole.cc, lorentz.cc, cooling.cc, annihilation.cc
// and energy_analysis.cc, and link libamk.so:
//   g++ -std=c++17 -I<repo>/include -I<biodynamo includes> -c amk_bdm_adapter.cc
//   ... -L<repo>/antimatter-kernel_b200 -lamk
// and register AmkRunQueuedBehaviours as a standalone operation after the
// agent operations.
//
// Every call gathers the agents it needs (in ResourceManager order, as the
// reference does), hands them to one process-wide libamk context and writes
// the results back. Semantics kept from the reference:
//   * the Coulomb drivers leave annihilated agents untouched; cutoff_radius
//     <= 0 gives every live agent a zero force (coulomb_interaction.cc:33-37);
//     the FMM driver gives neutral agents a zero force and leaves them out of
//     the sources (fast-multipole.cc:682-691);
//   * LorentzForce moves v back by dt/2 on its first push, per agent, and
//     consumes the Coulomb-force slot (lorentz.cc:56-70);
//   * an annihilated agent is removed at its next AnnihilationInteraction
//     visit (annihilation.cc:30-33);
//   * the energy's potentials are time-centred with the caller's history
//     (energy_analysis.cc:126-142).
// The context lives on the CUDA device named by the environment variable
// AMK_DEVICE (default 0) and is created by the first call. Errors, which
// the reference cannot have, are thrown as std::runtime_error with
// amk_last_error()'s message.
#include "amk_bdm_adapter.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "agents/charged_antiparticle.h"
#include "amk.h"
#include "core/param/param.h"
#include "core/resource_manager.h"
#include "core/scheduler.h"
#include "core/simulation.h"
#include "fields/penning_trap.h"
#include "params/physics_params.h"
#include "params/stochastic_params.h"

namespace bdm {
namespace {

amk_ctx* Context() {
  static std::once_flag once;
  static amk_ctx* ctx = nullptr;
  static int rc = AMK_OK;
  std::call_once(once, [] {
    amk_params p;
    amk_params_default(&p);
    const char* dev = std::getenv("AMK_DEVICE");
    rc = amk_create(&p, dev ? std::atoi(dev) : 0, &ctx);
  });
  if (rc != AMK_OK || !ctx) throw std::runtime_error(std::string("libamk context: ") + amk_last_error());
  return ctx;
}

void Check(int rc) {
  if (rc != AMK_OK) throw std::runtime_error(amk_last_error());
}

// The library's trap parameters for a field: z0 = sqrt(2) d with rho0 = 0
// reproduces the field's characteristic dimension d.
void SetTrap(amk_params* p, const PenningTrapField& field) {
  p->b0 = field.GetB0();
  p->trap_voltage = field.GetTrapVoltage();
  p->z0 = std::sqrt(2.0) * field.GetCharacteristicDimension();
  p->rho0 = 0.0;
}

uint32_t StableId(const Agent* a) { return static_cast<uint32_t>(a->GetUid().GetIndex()); }

// Structure-of-arrays copy of agents.
struct Gathered {
  std::vector<ChargedAntiparticle*> agents;
  std::vector<double> x, y, z, vx, vy, vz, q, m, fx, fy, fz;
  std::vector<uint8_t> species;
  std::vector<uint32_t> ids;
  void Add(ChargedAntiparticle* p) {
    const Real3& r = p->GetPosition();
    const Real3& v = p->GetVelocity();
    const Real3& f = p->GetCoulombForce();
    agents.push_back(p);
    x.push_back(r[0]);
    y.push_back(r[1]);
    z.push_back(r[2]);
    vx.push_back(v[0]);
    vy.push_back(v[1]);
    vz.push_back(v[2]);
    q.push_back(p->GetCharge());
    m.push_back(p->GetMass());
    fx.push_back(f[0]);
    fy.push_back(f[1]);
    fz.push_back(f[2]);
    species.push_back(static_cast<uint8_t>(p->GetSpecies()));
    ids.push_back(StableId(p));
  }
  long Size() const { return static_cast<long>(agents.size()); }
  void ZeroForces() {
    fx.assign(agents.size(), 0.0);
    fy.assign(agents.size(), 0.0);
    fz.assign(agents.size(), 0.0);
  }
  void ScatterForces() {
    for (size_t i = 0; i < agents.size(); ++i) agents[i]->SetCoulombForce(Real3{fx[i], fy[i], fz[i]});
  }
  // The gathered agents as the context's particle set (charges and masses
  // as the agents carry them, ids = the agents' uids).
  void Load(amk_ctx* c) {
    const long n = Size();
    Check(amk_set_particles(c, n, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(), species.data()));
    Check(amk_set_charge_mass(c, q.data(), m.data()));
    Check(amk_set_ids(c, ids.data()));
  }
};

template <typename F>
Gathered GatherLive(ResourceManager* rm, F&& keep) {
  Gathered g;
  rm->ForEachAgent([&](Agent* agent) {
    auto* p = FastCast(agent);
    if (p != nullptr && !p->IsAnnihilated() && keep(p)) g.Add(p);
  });
  return g;
}

// Agents queued by the behaviours' Run() since the last flush.
struct Queue {
  std::mutex mu;
  std::vector<std::pair<ChargedAntiparticle*, LorentzForce*>> lorentz;
  std::unordered_map<ChargedAntiparticle*, CyclotronCooling*> cooling;
  std::vector<ChargedAntiparticle*> annihilation;
};
Queue& TheQueue() {
  static Queue q;
  return q;
}

}  // namespace

// ---------------------------------------------------------------- Coulomb drivers
void ComputeStandardCoulombForces(ResourceManager* rm, real_t cutoff_radius) {
  Gathered g = GatherLive(rm, [](ChargedAntiparticle*) { return true; });
  if (g.Size() == 0) return;
  g.ZeroForces();
  if (cutoff_radius > 0.0)
    Check(amk_solve_cutoff(Context(), g.Size(), g.x.data(), g.y.data(), g.z.data(), g.q.data(), cutoff_radius,
                           g.fx.data(), g.fy.data(), g.fz.data()));
  g.ScatterForces();
}

void ComputeBarnesHutCoulombForces(ResourceManager* rm, real_t theta) {
  Gathered g = GatherLive(rm, [](ChargedAntiparticle*) { return true; });
  if (g.Size() == 0) return;
  g.ZeroForces();
  Check(amk_solve_barnes_hut(Context(), g.Size(), g.x.data(), g.y.data(), g.z.data(), g.q.data(), theta, 8,
                             g.fx.data(), g.fy.data(), g.fz.data(), nullptr));
  g.ScatterForces();
}

void ComputeFastMultipoleCoulombForces(ResourceManager* rm, int order, real_t theta) {
  Gathered g = GatherLive(rm, [](ChargedAntiparticle* p) {
    if (p->GetCharge() != 0.0) return true;
    p->SetCoulombForce(Real3{0.0, 0.0, 0.0});
    return false;
  });
  if (g.Size() == 0) return;
  g.ZeroForces();
  Check(amk_solve_fmm(Context(), g.Size(), g.x.data(), g.y.data(), g.z.data(), g.q.data(), order, theta, 32,
                      g.fx.data(), g.fy.data(), g.fz.data(), nullptr));
  g.ScatterForces();
}

// ---------------------------------------------------------------- BarnesHutTree
BarnesHutTree::BarnesHutTree(real_t theta, size_t leaf_capacity) : theta_(theta), leaf_capacity_(leaf_capacity) {}

void BarnesHutTree::Build(const std::vector<Source>& sources) {
  sources_ = sources;
  evaluated_ = false;
  nodes_ = -1;
}

void BarnesHutTree::Evaluate() const {
  const long n = static_cast<long>(sources_.size());
  std::vector<double> x(n), y(n), z(n), q(n);
  for (long i = 0; i < n; ++i) {
    x[i] = sources_[i].position[0];
    y[i] = sources_[i].position[1];
    z[i] = sources_[i].position[2];
    q[i] = sources_[i].charge;
  }
  ex_.assign(n, 0.0);
  ey_.assign(n, 0.0);
  ez_.assign(n, 0.0);
  phi_.assign(n, 0.0);
  if (n > 0)
    Check(amk_solve_barnes_hut(Context(), n, x.data(), y.data(), z.data(), q.data(), theta_,
                               static_cast<long>(leaf_capacity_), ex_.data(), ey_.data(), ez_.data(), phi_.data()));
  for (long i = 0; i < n; ++i) {  // forces on unit charge
    const double inv = q[i] != 0.0 ? 1.0 / q[i] : 0.0;
    ex_[i] *= inv;
    ey_[i] *= inv;
    ez_[i] *= inv;
  }
  evaluated_ = true;
}

namespace {
// The walk for a point that is not one of the sources: the sources plus the
// point (unit charge) as one more source. The point's own charge never
// enters its force or potential (a node holding the target is never
// accepted for theta < 1.15), but it may change where the tree splits.
void ExtraPoint(const std::vector<BarnesHutTree::Source>& s, const Real3& pos, real_t theta, size_t leaf,
                double* f3, double* phi) {
  const long n = static_cast<long>(s.size()) + 1;
  std::vector<double> x(n), y(n), z(n), q(n), fx(n), fy(n), fz(n), ph(n);
  for (long i = 0; i + 1 < n; ++i) {
    x[i] = s[i].position[0];
    y[i] = s[i].position[1];
    z[i] = s[i].position[2];
    q[i] = s[i].charge;
  }
  x[n - 1] = pos[0];
  y[n - 1] = pos[1];
  z[n - 1] = pos[2];
  q[n - 1] = 1.0;
  Check(amk_solve_barnes_hut(Context(), n, x.data(), y.data(), z.data(), q.data(), theta, static_cast<long>(leaf),
                             fx.data(), fy.data(), fz.data(), ph.data()));
  f3[0] = fx[n - 1];
  f3[1] = fy[n - 1];
  f3[2] = fz[n - 1];
  *phi = ph[n - 1];
}

bool IsSource(const std::vector<BarnesHutTree::Source>& s, size_t i, const Real3& pos) {
  return i < s.size() && s[i].position[0] == pos[0] && s[i].position[1] == pos[1] && s[i].position[2] == pos[2];
}
}  // namespace

Real3 BarnesHutTree::ComputeForce(const Real3& position, real_t charge, size_t self_index) const {
  if (IsSource(sources_, self_index, position) && sources_[self_index].charge != 0.0) {
    if (!evaluated_) Evaluate();
    return Real3{charge * ex_[self_index], charge * ey_[self_index], charge * ez_[self_index]};
  }
  double f[3], phi;
  ExtraPoint(sources_, position, theta_, leaf_capacity_, f, &phi);
  return Real3{charge * f[0], charge * f[1], charge * f[2]};
}

real_t BarnesHutTree::ComputePotential(const Real3& position, size_t self_index) const {
  if (IsSource(sources_, self_index, position)) {
    if (!evaluated_) Evaluate();
    return phi_[self_index];
  }
  double f[3], phi;
  ExtraPoint(sources_, position, theta_, leaf_capacity_, f, &phi);
  return phi;
}

size_t BarnesHutTree::NumNodes() const {
  if (nodes_ < 0) {
    const long n = static_cast<long>(sources_.size());
    std::vector<double> x(n), y(n), z(n), q(n);
    for (long i = 0; i < n; ++i) {
      x[i] = sources_[i].position[0];
      y[i] = sources_[i].position[1];
      z[i] = sources_[i].position[2];
      q[i] = sources_[i].charge;
    }
    const long cap = 4 * n + 64;
    std::vector<double> f(12 * static_cast<size_t>(cap));
    std::vector<long> g(11 * static_cast<size_t>(cap));
    const long nn = amk_bh_tree_dump(Context(), n, x.data(), y.data(), z.data(), q.data(),
                                     static_cast<long>(leaf_capacity_), cap, f.data(), g.data());
    if (nn < 0) Check(static_cast<int>(nn));
    nodes_ = nn;
  }
  return static_cast<size_t>(nodes_);
}

// ---------------------------------------------------------------- FastMultipoleSolver
FastMultipoleSolver::FastMultipoleSolver(int order, real_t theta, size_t leaf_capacity)
    : order_(order), theta_(theta), leaf_capacity_(leaf_capacity) {}

void FastMultipoleSolver::Compute(const std::vector<Source>& sources, std::vector<Real3>* forces,
                                  double* potential_energy) const {
  const long n = static_cast<long>(sources.size());
  if (forces) forces->assign(sources.size(), Real3{0.0, 0.0, 0.0});
  if (potential_energy) *potential_energy = 0.0;
  if (n == 0) return;
  std::vector<double> x(n), y(n), z(n), q(n), fx(n), fy(n), fz(n);
  for (long i = 0; i < n; ++i) {
    x[i] = sources[i].position[0];
    y[i] = sources[i].position[1];
    z[i] = sources[i].position[2];
    q[i] = sources[i].charge;
  }
  double e = 0.0;
  Check(amk_solve_fmm(Context(), n, x.data(), y.data(), z.data(), q.data(), order_, theta_,
                      static_cast<long>(leaf_capacity_), fx.data(), fy.data(), fz.data(),
                      potential_energy ? &e : nullptr));
  if (forces)
    for (long i = 0; i < n; ++i) (*forces)[i] = Real3{fx[i], fy[i], fz[i]};
  if (potential_energy) *potential_energy = e;
}

void FastMultipoleSolver::ComputeForces(const std::vector<Source>& sources, std::vector<Real3>* forces) const {
  Compute(sources, forces, nullptr);
}

real_t FastMultipoleSolver::ComputePotentialEnergy(const std::vector<Source>& sources) const {
  double e = 0.0;
  Compute(sources, nullptr, &e);
  return e;
}

// ---------------------------------------------------------------- behaviours
LorentzForce::LorentzForce(const PenningTrapField* field)
    : field_(field), dt_(Simulation::GetActive()->GetParam()->Get<PhysicsParams>()->dt) {}

void LorentzForce::Run(Agent* agent) {
  auto* particle = static_cast<ChargedAntiparticle*>(agent);
  if (particle == nullptr || field_ == nullptr) return;
  if (particle->IsAnnihilated()) return;
  if (particle->GetMass() <= 0.0 || dt_ <= 0.0) return;  // lorentz.cc:45-46
  Queue& q = TheQueue();
  std::lock_guard<std::mutex> lock(q.mu);
  q.lorentz.emplace_back(particle, this);
}

CyclotronCooling::CyclotronCooling(const PenningTrapField* field, real_t tau_scale, real_t bath_temp_K)
    : field_(field), tau_scale_(tau_scale), bath_temp_K_(bath_temp_K) {}

real_t CyclotronCooling::CoolingTime(real_t charge, real_t mass, real_t b_mag) {
  return amk_cooling_time(charge, mass, b_mag);
}

void CyclotronCooling::Run(Agent* agent) {
  auto* particle = static_cast<ChargedAntiparticle*>(agent);
  if (particle == nullptr || field_ == nullptr) return;
  if (particle->IsAnnihilated()) return;
  Queue& q = TheQueue();
  std::lock_guard<std::mutex> lock(q.mu);
  q.cooling[particle] = this;
}

bool IsAntiparticlePair(ParticleSpecies a, ParticleSpecies b) {
  auto either = [&](ParticleSpecies u, ParticleSpecies v) { return (a == u && b == v) || (a == v && b == u); };
  return either(ParticleSpecies::kAntiproton, ParticleSpecies::kProton) ||
         either(ParticleSpecies::kPositron, ParticleSpecies::kElectron);
}

void AnnihilationInteraction::Run(Agent* agent) {
  auto* particle = FastCast(agent);
  if (particle == nullptr) return;
  const auto* sp = Simulation::GetActive()->GetParam()->Get<StochasticParams>();
  if (!sp->annihilation_enabled) return;
  if (particle->IsAnnihilated()) {  // annihilation.cc:30-33
    particle->RemoveFromSimulation();
    return;
  }
  if (sp->contact_radius <= 0.0) return;
  Queue& q = TheQueue();
  std::lock_guard<std::mutex> lock(q.mu);
  q.annihilation.push_back(particle);
}

void AmkRunQueuedBehaviours() {
  Queue& q = TheQueue();
  std::vector<std::pair<ChargedAntiparticle*, LorentzForce*>> lorentz;
  std::unordered_map<ChargedAntiparticle*, CyclotronCooling*> cooling;
  std::vector<ChargedAntiparticle*> annihilation;
  {
    std::lock_guard<std::mutex> lock(q.mu);
    lorentz.swap(q.lorentz);
    cooling.swap(q.cooling);
    annihilation.swap(q.annihilation);
  }
  // the random streams' step index: the scheduler step being simulated
  // (GetSimulatedSteps counts the steps completed before it)
  const long step = static_cast<long>(Simulation::GetActive()->GetScheduler()->GetSimulatedSteps()) + 1;
  const auto* physics = Simulation::GetActive()->GetParam()->Get<PhysicsParams>();
  auto by_uid = [](const ChargedAntiparticle* a, const ChargedAntiparticle* b) { return StableId(a) < StableId(b); };
  amk_ctx* ctx = Context();
  if (!lorentz.empty()) {
    std::sort(lorentz.begin(), lorentz.end(), [&](const auto& a, const auto& b) { return by_uid(a.first, b.first); });
    const LorentzForce* l0 = lorentz.front().second;
    const CyclotronCooling* c0 = cooling.empty() ? nullptr : cooling.begin()->second;
    for (const auto& e : lorentz) {
      if (e.second->field_ != l0->field_ || e.second->dt_ != l0->dt_)
        throw std::runtime_error("AmkRunQueuedBehaviours: queued LorentzForce behaviours differ in field or dt");
      if (c0) {
        auto it = cooling.find(e.first);
        if (it == cooling.end() || it->second->tau_scale_ != c0->tau_scale_ ||
            it->second->bath_temp_K_ != c0->bath_temp_K_)
          throw std::runtime_error("AmkRunQueuedBehaviours: every pushed agent must carry the same cooling");
      }
    }
    amk_params p;
    amk_params_default(&p);
    SetTrap(&p, *l0->field_);
    p.dt = l0->dt_;
    p.seed = physics->seed;
    p.cooling_enabled = c0 ? 1 : 0;
    p.cooling_scale = c0 ? c0->tau_scale_ : 0.0;
    p.bath_temperature = c0 ? c0->bath_temp_K_ : 0.0;
    p.annihilation_enabled = 0;
    p.coulomb_forces_enabled = 0;
    // agents still at v(0) take the one-time back-stagger, the rest do not
    // (the groups are fixed before either is pushed: a pushed agent's flag
    // flips, and it must not join the second group of the same step)
    std::vector<char> was_staggered;
    for (const auto& e : lorentz) was_staggered.push_back(e.second->velocity_staggered_ ? 1 : 0);
    for (int staggered = 0; staggered < 2; ++staggered) {
      Gathered g;
      std::vector<LorentzForce*> owners;
      for (size_t k = 0; k < lorentz.size(); ++k)
        if (was_staggered[k] == staggered) {
          const auto& e = lorentz[k];
          g.Add(e.first);
          owners.push_back(e.second);
        }
      if (g.Size() == 0) continue;
      Check(amk_set_params(ctx, &p));
      g.Load(ctx);
      Check(amk_set_forces(ctx, g.fx.data(), g.fy.data(), g.fz.data()));
      Check(amk_set_step_state(ctx, step - 1, staggered));
      Check(amk_push(ctx));
      Check(amk_get_particles(ctx, g.x.data(), g.y.data(), g.z.data(), g.vx.data(), g.vy.data(), g.vz.data(),
                              nullptr));
      for (long i = 0; i < g.Size(); ++i) {
        ChargedAntiparticle* a = g.agents[i];
        a->SetPosition(Real3{g.x[i], g.y[i], g.z[i]});
        a->SetVelocity(Real3{g.vx[i], g.vy[i], g.vz[i]});
        a->SetCoulombForce(Real3{0.0, 0.0, 0.0});  // consumed (lorentz.cc:70)
        owners[i]->velocity_staggered_ = true;
      }
    }
  }
  if (!annihilation.empty()) {
    std::sort(annihilation.begin(), annihilation.end(), by_uid);
    const auto* sp = Simulation::GetActive()->GetParam()->Get<StochasticParams>();
    Gathered g;
    for (ChargedAntiparticle* a : annihilation)
      if (!a->IsAnnihilated()) g.Add(a);
    if (g.Size() > 0) {
      amk_params p;
      amk_params_default(&p);
      p.seed = physics->seed;
      p.annihilation_enabled = 1;
      p.contact_radius = sp->contact_radius;
      p.annihilation_probability = sp->annihilation_probability;
      p.coulomb_forces_enabled = 0;
      Check(amk_set_params(ctx, &p));
      g.Load(ctx);
      Check(amk_set_step_state(ctx, step, 1));
      long marked = 0;
      Check(amk_annihilate(ctx, &marked));
      std::vector<uint8_t> alive(static_cast<size_t>(g.Size()));
      Check(amk_get_particles(ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, alive.data()));
      for (long i = 0; i < g.Size(); ++i)
        if (!alive[i]) g.agents[i]->MarkAnnihilated();
    }
  }
}

// ---------------------------------------------------------------- energy
EnergyBreakdown ComputeTotalEnergy(ResourceManager* rm, const PenningTrapField& field,
                                   const EnergyComputationSettings& energy, EnergyHistory* history) {
  EnergyBreakdown result;
  Gathered g = GatherLive(rm, [](ChargedAntiparticle*) { return true; });
  result.num_active_particles = static_cast<size_t>(g.Size());
  if (g.Size() > 0) {
    amk_params p;
    amk_params_default(&p);
    SetTrap(&p, field);
    switch (energy.method) {
      case ComputationMethod::kFastMultipole: p.energy_method = AMK_METHOD_FAST_MULTIPOLE; break;
      case ComputationMethod::kBarnesHut: p.energy_method = AMK_METHOD_BARNES_HUT; break;
      default: p.energy_method = AMK_METHOD_STANDARD; break;
    }
    p.cutoff_radius = energy.cutoff_radius;
    p.barnes_hut_theta = energy.barnes_hut_theta;
    p.fast_multipole_theta = energy.fast_multipole_theta;
    p.fast_multipole_order = energy.fast_multipole_order;
    amk_ctx* ctx = Context();
    Check(amk_set_params(ctx, &p));
    g.Load(ctx);
    amk_energy_out e;
    Check(amk_energy(ctx, 0, &e));
    result.kinetic = e.kinetic;
    result.trap_potential = e.trap_potential;
    result.energy_potential = e.coulomb_potential;
  }
  if (history != nullptr) {  // energy_analysis.cc:126-142
    const real_t raw_trap = result.trap_potential, raw_coulomb = result.energy_potential;
    if (history->has_previous) {
      result.trap_potential = 0.5 * (history->prev_trap_potential + raw_trap);
      result.energy_potential = 0.5 * (history->prev_coulomb_potential + raw_coulomb);
    }
    history->prev_trap_potential = raw_trap;
    history->prev_coulomb_potential = raw_coulomb;
    history->has_previous = true;
  }
  return result;
}

}  // namespace bdm
