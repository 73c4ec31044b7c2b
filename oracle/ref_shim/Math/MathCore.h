// Shim of BaseProject Math/MathCore.h: EPSILON and PI for Real = double (the
// values the CPU restatement and the GPU library fix: 1e-6 and pi rounded to
// double), maximum / minimum.
#ifndef TSR_SHIM_MATHCORE_H
#define TSR_SHIM_MATHCORE_H
#include "Platform/DataTypes.h"

namespace Math {
const Real EPSILON = 1e-6;
const Real PI = 3.14159265358979323846;
template <class T> inline T maximum(const T &a, const T &b) { return a > b ? a : b; }
template <class T> inline T minimum(const T &a, const T &b) { return a < b ? a : b; }
}  // namespace Math
using Math::EPSILON;
#endif
