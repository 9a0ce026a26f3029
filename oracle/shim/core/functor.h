// Stand-in for BioDynaMo's L2F lambda-to-functor helper (TEST
// INFRASTRUCTURE ONLY): the functor simply forwards to the lambda.
#ifndef AMK_SHIM_FUNCTOR_H_
#define AMK_SHIM_FUNCTOR_H_
#include <utility>
#include "core/real_t.h"
namespace bdm {
class Agent;
template <typename L>
struct LambdaFunctor {
  L lambda;
  void operator()(Agent* a, real_t squared_distance) { lambda(a, squared_distance); }
};
template <typename L>
LambdaFunctor<L> L2F(L&& l) {
  return LambdaFunctor<L>{std::forward<L>(l)};
}
}  // namespace bdm
#endif
