// Stand-in for BioDynaMo's Environment (TEST INFRASTRUCTURE ONLY): a
// brute-force neighbour search over the resource manager's agents in
// ascending id order, visiting every other agent (removed ones excluded)
// with |x_j - x_i|^2 < squared_radius. Before each visit it records the
// neighbour's id as the current random-stream partner.
#ifndef AMK_SHIM_ENVIRONMENT_H_
#define AMK_SHIM_ENVIRONMENT_H_
#include "core/resource_manager.h"
#include "core/util/random.h"
namespace bdm {
class Environment {
 public:
  explicit Environment(ResourceManager* rm = nullptr) : rm_(rm) {}
  void Update() {}
  template <typename F>
  void ForEachNeighbor(F& f, const Agent& query, real_t squared_radius) {
    const Real3& xi = query.GetPosition();
    for (Agent* a : rm_->agents) {
      if (a == &query || a->removed_) continue;
      const Real3& xj = a->GetPosition();
      const real_t dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
      const real_t d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < squared_radius) {
        g_shim_rng.partner = a->uid_;
        f(a, d2);
      }
    }
  }

 private:
  ResourceManager* rm_;
};
}  // namespace bdm
#endif
