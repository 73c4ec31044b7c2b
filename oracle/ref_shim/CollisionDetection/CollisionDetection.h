// Shim of BaseProject CollisionDetection/CollisionDetection.h: the AABB
// predicates the reference's hot path calls, with the semantics of the CPU
// restatement (oracle/tsr_geom.h), which they call.
#ifndef TSR_SHIM_COLLISIONDETECTION_H
#define TSR_SHIM_COLLISIONDETECTION_H
#include "Math/Vector3.h"
#include "../../tsr_geom.h"

namespace CollisionDetection {
class ObliqueCircularCone;   // ObliqueCircularCone.h

inline tsrg::V3 shim_v3(const Math::Vector3 &v) { return tsrg::V3{v.x, v.y, v.z}; }

inline bool intersectAABBWithSphere(const Math::Vector3 &mn, const Math::Vector3 &mx, const Math::Vector3 &c,
                                    const Real r) {
    return tsrg::aabb_sphere(shim_v3(mn), shim_v3(mx), shim_v3(c), r);
}

inline bool intersectAABBWithLineSegment(Real &entryT, Real &exitT, const Math::Vector3 &s, const Math::Vector3 &e,
                                         const Math::Vector3 &mn, const Math::Vector3 &mx) {
    return tsrg::segment_aabb(entryT, exitT, shim_v3(s), shim_v3(e), shim_v3(mn), shim_v3(mx));
}

inline Real getDistanceToAABB(const Math::Vector3 &p, const Math::Vector3 &mn, const Math::Vector3 &mx) {
    const Real dx = p.x < mn.x ? mn.x - p.x : (p.x > mx.x ? p.x - mx.x : 0.0);
    const Real dy = p.y < mn.y ? mn.y - p.y : (p.y > mx.y ? p.y - mx.y : 0.0);
    const Real dz = p.z < mn.z ? mn.z - p.z : (p.z > mx.z ? p.z - mx.z : 0.0);
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Plane through `p` with normal `n`: signed distance dot(x - p, n).
class Plane {
public:
    Plane(const Math::Vector3 &p, const Math::Vector3 &n, bool /*normalized*/) : mP(p), mN(n) {}
    Real getDistanceToPlane(const Math::Vector3 &x) const { return (x - mP).dotProduct(mN); }
private:
    Math::Vector3 mP, mN;
};
}  // namespace CollisionDetection
#endif
