// Shim of BaseProject Math/Vector4.h (included, not used, by the hot path).
#ifndef TSR_SHIM_VECTOR4_H
#define TSR_SHIM_VECTOR4_H
#include "Math/Vector3.h"
namespace Math {
class Vector4 {
public:
    Vector4() : x(0.0), y(0.0), z(0.0), w(0.0) {}
    Vector4(Real x_, Real y_, Real z_, Real w_) : x(x_), y(y_), z(z_), w(w_) {}
    Real x, y, z, w;
};
}  // namespace Math
#endif
