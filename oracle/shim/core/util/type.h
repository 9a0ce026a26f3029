// Stand-in for BioDynaMo's core/util/type.h (only real_t is needed).
#ifndef AMK_SHIM_TYPE_H_
#define AMK_SHIM_TYPE_H_
#include "core/real_t.h"
#endif
