// Test-harness stand-in for boost::math::isfinite.
#pragma once
#include <cmath>
namespace boost {
namespace math {
template <class T>
bool isfinite(T x) { return std::isfinite(x); }
}  // namespace math
}  // namespace boost
