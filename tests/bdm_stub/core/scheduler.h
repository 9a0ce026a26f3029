// Test stand-in for BioDynaMo's Scheduler: the number of completed steps
// (Scheduler::GetSimulatedSteps), set by the test harness before each step.
#pragma once
#include <cstdint>
namespace bdm {
class Scheduler {
 public:
  uint64_t simulated_steps = 0;
  uint64_t GetSimulatedSteps() const { return simulated_steps; }
};
}  // namespace bdm
