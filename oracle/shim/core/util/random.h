// Stand-in for BioDynaMo's Random (TEST INFRASTRUCTURE ONLY). BioDynaMo's
// ROOT generator is not available, so the stand-in replays the CUDA
// library's Philox streams (oracle/philox.h) for the draw the reference's
// code is making: Gaus for the current particle and step (the k-th call
// returns mean + sigma * z_k of that particle's three cooling normals),
// Uniform for the current (owner, partner, step) annihilation candidate.
// The harness sets the context before each Run; the neighbour stand-in sets
// the partner before each neighbour visit.
#ifndef AMK_SHIM_RANDOM_H_
#define AMK_SHIM_RANDOM_H_
#include <cstdint>
#include "philox.h"
namespace bdm {
struct ShimRngContext {
  uint32_t seed = 0;
  uint32_t particle = 0;
  uint32_t partner = 0;
  uint64_t step = 0;
  int gaus_calls = 0;
};
inline ShimRngContext g_shim_rng;
class Random {
 public:
  double Gaus(double mean, double sigma) {
    double z[3];
    orc::CoolingNormals(g_shim_rng.seed, g_shim_rng.particle, g_shim_rng.step, z);
    const int k = g_shim_rng.gaus_calls++ % 3;
    return mean + sigma * z[k];
  }
  double Uniform(double min, double max) {
    const double u = orc::AnnihilationUniform(g_shim_rng.seed, g_shim_rng.particle, g_shim_rng.partner,
                                              g_shim_rng.step);
    return min + (max - min) * u;
  }
};
}  // namespace bdm
#endif
