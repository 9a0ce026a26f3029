// Test stand-in for BioDynaMo's Behavior base class.
#pragma once
#define BDM_BEHAVIOR_HEADER(type, base, version) \
 public:                                         \
  static const char* BehaviorName() { return #type; }
namespace bdm {
class Agent;
class Behavior {
 public:
  virtual ~Behavior() = default;
  virtual void Run(Agent* agent) = 0;
};
}  // namespace bdm
