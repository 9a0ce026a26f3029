// Minimal stand-in for BioDynaMo's core/real_t.h so that the reference's
// solver sources compile unmodified for the CPU oracle. BioDynaMo's default
// build uses double precision.
#ifndef AMK_SHIM_REAL_T_H_
#define AMK_SHIM_REAL_T_H_
namespace bdm {
using real_t = double;
}
#endif
