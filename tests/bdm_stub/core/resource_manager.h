// Test stand-in for BioDynaMo's ResourceManager: agents visited in
// insertion order.
#pragma once
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
