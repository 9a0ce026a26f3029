// Test stand-in for BioDynaMo's real_t (double in BioDynaMo's default build).
#pragma once
namespace bdm {
using real_t = double;
}
