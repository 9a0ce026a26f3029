// Stand-in for BioDynaMo's ResourceManager: a flat list of agents visited in
// insertion order, enough for the reference's Compute*CoulombForces drivers.
#ifndef AMK_SHIM_RESOURCE_MANAGER_H_
#define AMK_SHIM_RESOURCE_MANAGER_H_
#include <vector>
#include "agents/charged_antiparticle.h"
namespace bdm {
class ResourceManager {
 public:
  std::vector<Agent*> agents;
  template <typename F>
  void ForEachAgent(F&& f) {
    for (Agent* a : agents) f(a);
  }
};
}  // namespace bdm
#endif
