// Stand-in for BioDynaMo's ParamGroup (TEST INFRASTRUCTURE ONLY).
#ifndef AMK_SHIM_PARAM_GROUP_H_
#define AMK_SHIM_PARAM_GROUP_H_
#include "core/container/math_array.h"
#include "core/real_t.h"
#define BDM_PARAM_GROUP_HEADER(type, version) \
 public:                                      \
  type() = default
namespace bdm {
struct ParamGroup {
  virtual ~ParamGroup() = default;
};
}  // namespace bdm
#endif
