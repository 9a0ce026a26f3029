// Test harness: builds agents, calls one of the adapter's reference-shaped
// drivers and returns every agent's Coulomb-force slot (NaN stays in the
// slots the driver did not write).
#include <cmath>
#include <vector>

#include "agents/charged_antiparticle.h"
#include "core/resource_manager.h"

namespace bdm {
void ComputeStandardCoulombForces(ResourceManager* rm, real_t cutoff_radius);
void ComputeBarnesHutCoulombForces(ResourceManager* rm, real_t theta);
void ComputeFastMultipoleCoulombForces(ResourceManager* rm, int order, real_t theta);
}  // namespace bdm

extern "C" int harness_run(int method, long n, const double* x, const double* y, const double* z, const double* q,
                           const unsigned char* annihilated, double param, int order, double* fx, double* fy,
                           double* fz) {
  std::vector<bdm::ChargedAntiparticle> parts(static_cast<size_t>(n));
  bdm::ResourceManager rm;
  for (long i = 0; i < n; ++i) {
    parts[i].position = bdm::Real3(x[i], y[i], z[i]);
    parts[i].charge = q[i];
    parts[i].annihilated = annihilated[i] != 0;
    parts[i].coulomb_force = bdm::Real3(NAN, NAN, NAN);
    rm.agents.push_back(&parts[i]);
  }
  try {
    if (method == 0) bdm::ComputeStandardCoulombForces(&rm, param);
    if (method == 1) bdm::ComputeBarnesHutCoulombForces(&rm, param);
    if (method == 2) bdm::ComputeFastMultipoleCoulombForces(&rm, order, param);
  } catch (...) {
    return -1;
  }
  for (long i = 0; i < n; ++i) {
    fx[i] = parts[i].coulomb_force[0];
    fy[i] = parts[i].coulomb_force[1];
    fz[i] = parts[i].coulomb_force[2];
  }
  return 0;
}
