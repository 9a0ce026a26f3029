// Stand-in for BioDynaMo's Math helpers (TEST INFRASTRUCTURE ONLY).
#ifndef AMK_SHIM_MATH_H_
#define AMK_SHIM_MATH_H_
#include "core/container/math_array.h"
namespace bdm {
struct Math {
  static Real3 CrossProduct(const Real3& a, const Real3& b) {
    return Real3{{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}};
  }
};
}  // namespace bdm
#endif
