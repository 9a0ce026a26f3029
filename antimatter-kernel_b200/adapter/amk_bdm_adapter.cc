// Drop-in replacement of the reference's three Coulomb drivers for a
// BioDynaMo application: the same free functions with the same signatures
// (interaction/coulomb_interaction.h:10, interaction/barnes-hut.h:76,
// interaction/fast-multipole.h:73), computed by libamk on the GPU.
//
// Build it into the application in place of coulomb_interaction.cc,
// barnes-hut.cc and fast-multipole.cc, and link libamk.so:
//   g++ -std=c++17 -I<repo>/include -I<biodynamo includes> -c amk_bdm_adapter.cc
//   ... -L<repo>/antimatter-kernel_b200 -lamk
//
// Each call gathers the non-annihilated agents (in ResourceManager order,
// as the reference does), hands positions and charges to one process-wide
// libamk context and writes each agent's Coulomb-force slot, which the
// LorentzForce behaviour consumes. Semantics kept from the reference:
//   * annihilated agents are left untouched;
//   * cutoff_radius <= 0 gives every live agent a zero force
//     (coulomb_interaction.cc:33-37);
//   * the FMM driver gives neutral agents a zero force and leaves them out
//     of the sources (fast-multipole.cc:682-691).
// The context lives on the CUDA device named by the environment variable
// AMK_DEVICE (default 0) and is created by the first call. Errors, which
// the reference cannot have, are thrown as std::runtime_error with
// amk_last_error()'s message.
#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "agents/charged_antiparticle.h"
#include "amk.h"
#include "core/resource_manager.h"

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

// Structure-of-arrays copy of the live agents.
struct Gathered {
  std::vector<ChargedAntiparticle*> agents;
  std::vector<double> x, y, z, q, fx, fy, fz;
  void Add(ChargedAntiparticle* p) {
    const Real3& r = p->GetPosition();
    agents.push_back(p);
    x.push_back(r[0]);
    y.push_back(r[1]);
    z.push_back(r[2]);
    q.push_back(p->GetCharge());
  }
  long Size() const { return static_cast<long>(agents.size()); }
  void Resize() {
    fx.assign(agents.size(), 0.0);
    fy.assign(agents.size(), 0.0);
    fz.assign(agents.size(), 0.0);
  }
  void Scatter() {
    for (size_t i = 0; i < agents.size(); ++i) agents[i]->SetCoulombForce(Real3{fx[i], fy[i], fz[i]});
  }
};

}  // namespace

void ComputeStandardCoulombForces(ResourceManager* rm, real_t cutoff_radius) {
  Gathered g;
  rm->ForEachAgent([&](Agent* agent) {
    auto* p = FastCast(agent);
    if (p != nullptr && !p->IsAnnihilated()) g.Add(p);
  });
  if (g.Size() == 0) return;
  g.Resize();
  if (cutoff_radius > 0.0)
    Check(amk_solve_cutoff(Context(), g.Size(), g.x.data(), g.y.data(), g.z.data(), g.q.data(), cutoff_radius,
                           g.fx.data(), g.fy.data(), g.fz.data()));
  g.Scatter();
}

void ComputeBarnesHutCoulombForces(ResourceManager* rm, real_t theta) {
  Gathered g;
  rm->ForEachAgent([&](Agent* agent) {
    auto* p = FastCast(agent);
    if (p != nullptr && !p->IsAnnihilated()) g.Add(p);
  });
  if (g.Size() == 0) return;
  g.Resize();
  Check(amk_solve_barnes_hut(Context(), g.Size(), g.x.data(), g.y.data(), g.z.data(), g.q.data(), theta, 8,
                             g.fx.data(), g.fy.data(), g.fz.data(), nullptr));
  g.Scatter();
}

void ComputeFastMultipoleCoulombForces(ResourceManager* rm, int order, real_t theta) {
  Gathered g;
  rm->ForEachAgent([&](Agent* agent) {
    auto* p = FastCast(agent);
    if (p == nullptr || p->IsAnnihilated()) return;
    if (p->GetCharge() == 0.0)
      p->SetCoulombForce(Real3{0.0, 0.0, 0.0});
    else
      g.Add(p);
  });
  if (g.Size() == 0) return;
  g.Resize();
  Check(amk_solve_fmm(Context(), g.Size(), g.x.data(), g.y.data(), g.z.data(), g.q.data(), order, theta, 32,
                      g.fx.data(), g.fy.data(), g.fz.data(), nullptr));
  g.Scatter();
}

}  // namespace bdm
