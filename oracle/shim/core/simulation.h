// Stand-in for BioDynaMo's Simulation (TEST INFRASTRUCTURE ONLY): the
// active simulation hands out the parameter groups, the random stream
// stand-in and the neighbour-search stand-in of the harness's world.
#ifndef AMK_SHIM_SIMULATION_H_
#define AMK_SHIM_SIMULATION_H_
#include "core/environment/environment.h"
#include "core/param/param.h"
#include "core/util/random.h"
namespace bdm {
class Simulation {
 public:
  Param* param = nullptr;
  Random* random = nullptr;
  Environment* environment = nullptr;
  static Simulation*& Active() {
    static Simulation* active = nullptr;
    return active;
  }
  static Simulation* GetActive() { return Active(); }
  const Param* GetParam() const { return param; }
  Random* GetRandom() { return random; }
  Environment* GetEnvironment() { return environment; }
};
}  // namespace bdm
#endif
