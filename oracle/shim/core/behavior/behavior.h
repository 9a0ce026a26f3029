// Stand-in for BioDynaMo's Behavior base class (TEST INFRASTRUCTURE ONLY):
// a virtual Run(Agent*) and an empty class-header macro.
#ifndef AMK_SHIM_BEHAVIOR_H_
#define AMK_SHIM_BEHAVIOR_H_
#include "agents/charged_antiparticle.h"
#define BDM_BEHAVIOR_HEADER(type, base, version) \
 public:                                         \
  static const char* BehaviorName() { return #type; }
namespace bdm {
class Behavior {
 public:
  virtual ~Behavior() = default;
  virtual void Run(Agent* agent) = 0;
};
}  // namespace bdm
#endif
