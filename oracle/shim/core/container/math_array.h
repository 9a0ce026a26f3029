// Stand-in for BioDynaMo's MathArray/Real3: a 3-vector of doubles with the
// operators the reference solvers use (+, -, scalar *, dot product via *).
#ifndef AMK_SHIM_MATH_ARRAY_H_
#define AMK_SHIM_MATH_ARRAY_H_
#include <cstddef>
#include "core/real_t.h"
namespace bdm {
template <typename T, std::size_t N>
struct MathArray {
  T data_[N];
  T& operator[](std::size_t i) { return data_[i]; }
  const T& operator[](std::size_t i) const { return data_[i]; }
  MathArray operator+(const MathArray& o) const {
    MathArray r;
    for (std::size_t i = 0; i < N; ++i) r.data_[i] = data_[i] + o.data_[i];
    return r;
  }
  MathArray operator-(const MathArray& o) const {
    MathArray r;
    for (std::size_t i = 0; i < N; ++i) r.data_[i] = data_[i] - o.data_[i];
    return r;
  }
  MathArray operator*(T s) const {
    MathArray r;
    for (std::size_t i = 0; i < N; ++i) r.data_[i] = data_[i] * s;
    return r;
  }
  T operator*(const MathArray& o) const {
    T s = 0;
    for (std::size_t i = 0; i < N; ++i) s += data_[i] * o.data_[i];
    return s;
  }
};
using Real3 = MathArray<real_t, 3>;
}  // namespace bdm
#endif
