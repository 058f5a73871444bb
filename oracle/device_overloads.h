// Force-included into the host build of the reference (oracle/_ref) only.
// Device code resolves unqualified cos / sin / sqrt / acos / atan2 / fabs on
// a float argument to CUDA's float overloads in the global namespace; under
// g++ the same calls would pick the double ::cos etc. from math.h.  Bringing
// the std float overloads into the global namespace makes the host build
// resolve them as the device build does.
#pragma once
#include <cmath>
using std::acos;
using std::atan2;
using std::cos;
using std::exp;
using std::fabs;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
