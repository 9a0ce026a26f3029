// Stand-in for BioDynaMo's Param (TEST INFRASTRUCTURE ONLY): parameter
// groups registered by type, returned by Get<T>().
#ifndef AMK_SHIM_PARAM_H_
#define AMK_SHIM_PARAM_H_
#include <map>
#include <stdexcept>
#include <typeindex>
#include "core/param/param_group.h"
namespace bdm {
class Param {
 public:
  template <typename T>
  void Set(T* group) {
    groups_[std::type_index(typeid(T))] = group;
  }
  template <typename T>
  const T* Get() const {
    auto it = groups_.find(std::type_index(typeid(T)));
    if (it == groups_.end()) throw std::logic_error("parameter group not registered");
    return static_cast<const T*>(it->second);
  }

 private:
  std::map<std::type_index, ParamGroup*> groups_;
};
}  // namespace bdm
#endif
