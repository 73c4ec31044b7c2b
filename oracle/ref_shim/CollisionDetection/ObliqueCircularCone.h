// Shim of BaseProject CollisionDetection/ObliqueCircularCone.h with the
// semantics the CPU restatement assumes (oracle/tsr_geom.h, tsrg::Cone): apex,
// end-disc centre and normal, end radius; discs parallel to the end disc; a
// cut length measured back from the end (REAL_MAX keeps the whole cone).  The
// separating-axis test is the restatement's conservative box test (the
// reference's leaf sums do not depend on which conservative test is used,
// because addKernel re-tests every leaf centre exactly).
#ifndef TSR_SHIM_OBLIQUECIRCULARCONE_H
#define TSR_SHIM_OBLIQUECIRCULARCONE_H
#include "CollisionDetection/CollisionDetection.h"

namespace CollisionDetection {
class ObliqueCircularCone {
public:
    ObliqueCircularCone(const Math::Vector3 &apex, const Math::Vector3 &endOutsideNormal,
                        const Math::Vector3 &endCenter, const Real endRadius, const Real length)
        : mApex(apex), mApexToEnd(endCenter - apex) {
        tsrg::cone_init(mCone, shim_v3(apex), shim_v3(endOutsideNormal), shim_v3(endCenter), endRadius, length);
    }
    virtual ~ObliqueCircularCone() {}
    bool isDegenerated() const { return tsrg::cone_degenerated(mCone); }
    Real getLength() const { return mCone.length; }
    Real getTCompleteCone(const Math::Vector3 &x) const { return tsrg::cone_t_complete(mCone, shim_v3(x)); }
    Real getTCutCone(const Real tComplete) const { return tsrg::cone_t_cut(mCone, tComplete); }
    const Math::Vector3 &getApexToEnd() const { return mApexToEnd; }
    const Math::Vector3 &getApex() const { return mApex; }
    Real getEndRadius() const { return mCone.radius; }
    bool haveSeparatingAxis(const Math::Vector3 &boxMin, const Math::Vector3 &boxExtent) const {
        return tsrg::cone_box_separated(mCone, shim_v3(boxMin), boxExtent.x);
    }
private:
    Math::Vector3 mApex, mApexToEnd;
    tsrg::Cone mCone;
};
}  // namespace CollisionDetection
#endif
