// Test stand-in for BioDynaMo's Simulation: the active simulation's Param
// and Scheduler.
#pragma once
#include "core/param/param.h"
#include "core/scheduler.h"
namespace bdm {
class Simulation {
 public:
  Param param;
  static Simulation*& Active() {
    static Simulation* s = nullptr;
    return s;
  }
  static Simulation* GetActive() { return Active(); }
  Scheduler scheduler;
  const Param* GetParam() const { return &param; }
  Scheduler* GetScheduler() { return &scheduler; }
};
}  // namespace bdm
