// Shim of BaseProject Math/Vector3.h: componentwise FP64 vector arithmetic
// (x, y and z each rounded separately, in that order), as the CPU restatement
// assumes.
#ifndef TSR_SHIM_VECTOR3_H
#define TSR_SHIM_VECTOR3_H
#include "Platform/DataTypes.h"

namespace Math {
class Vector3 {
public:
    Vector3() : x(0.0), y(0.0), z(0.0) {}
    Vector3(Real x_, Real y_, Real z_) : x(x_), y(y_), z(z_) {}
    void set(Real x_, Real y_, Real z_) { x = x_; y = y_; z = z_; }
    Vector3 operator+(const Vector3 &o) const { return Vector3(x + o.x, y + o.y, z + o.z); }
    Vector3 operator-(const Vector3 &o) const { return Vector3(x - o.x, y - o.y, z - o.z); }
    Vector3 operator-() const { return Vector3(-x, -y, -z); }
    Vector3 operator*(Real s) const { return Vector3(x * s, y * s, z * s); }
    Vector3 operator/(Real s) const { return Vector3(x / s, y / s, z / s); }
    Vector3 &operator+=(const Vector3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
    Vector3 &operator-=(const Vector3 &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    Vector3 &operator*=(Real s) { x *= s; y *= s; z *= s; return *this; }
    Vector3 &operator/=(Real s) { x /= s; y /= s; z /= s; return *this; }
    bool operator==(const Vector3 &o) const { return x == o.x && y == o.y && z == o.z; }
    bool operator!=(const Vector3 &o) const { return !(*this == o); }
    Real dotProduct(const Vector3 &o) const { return x * o.x + y * o.y + z * o.z; }
    Vector3 crossProduct(const Vector3 &o) const {
        return Vector3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
    }
    Real getLengthSquared() const { return x * x + y * y + z * z; }
    Real getLength() const { return sqrt(getLengthSquared()); }
    void normalize() {
        const Real l = getLength();
        if (l > 0.0) { x /= l; y /= l; z /= l; }
    }
    Vector3 minimum(const Vector3 &o) const {
        return Vector3(x < o.x ? x : o.x, y < o.y ? y : o.y, z < o.z ? z : o.z);
    }
    Vector3 maximum(const Vector3 &o) const {
        return Vector3(x > o.x ? x : o.x, y > o.y ? y : o.y, z > o.z ? z : o.z);
    }
    Real x, y, z;
};
inline Vector3 operator*(Real s, const Vector3 &v) { return Vector3(v.x * s, v.y * s, v.z * s); }
}  // namespace Math
#endif
