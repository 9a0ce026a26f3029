// Test stand-in for BioDynaMo's Simulation: the active simulation's Param.
#pragma once
#include "core/param/param.h"
namespace bdm {
class Simulation {
 public:
  Param param;
  static Simulation*& Active() {
    static Simulation* s = nullptr;
    return s;
  }
  static Simulation* GetActive() { return Active(); }
  const Param* GetParam() const { return &param; }
};
}  // namespace bdm
