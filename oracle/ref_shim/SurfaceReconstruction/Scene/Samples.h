// Shadow of the reference's Scene/Samples.h for the reference build: the
// sample arrays and the getters the hot-path sources call, with the
// reference's definitions -- getMaxSamplingDistance = scale * h_SVO
// (Samples.h:409-412), the AABB of the sample spheres of radius
// getMaxSamplingDistance + EPSILON (Samples.cpp:110-119,290-298,442-449), link
// l = sample l / K, slot l % K (Samples.h:343-346,418-437), in-place reorder
// (Samples.cpp:825-835), and the signed distance to the sample's tangent plane
// (Samples.cpp:451-455, BaseProject Plane: dot(x - p, n)).
#ifndef TSR_SHIM_SAMPLES_H
#define TSR_SHIM_SAMPLES_H
#include <stdexcept>
#include <vector>
#include "Math/MathCore.h"
#include "Math/Vector3.h"
#include "Platform/Storage/Path.h"
#include "Platform/Utilities/Array.h"

namespace SurfaceReconstruction {
class Samples {
public:
    uint32 getCount() const { return (uint32)mPositions.size(); }
    const Math::Vector3 &getPositionWS(const uint32 i) const { return mPositions[i]; }
    const Math::Vector3 &getNormalWS(const uint32 i) const { return mNormals[i]; }
    const Real getScale(const uint32 i) const { return mScales[i]; }
    Real getConfidence(const uint32 i) const { return mConfidences[i]; }
    Real getMaxSamplingDistance(const uint32 i) const { return getScale(i) * mMaxRelativeSamplingDistance; }
    uint32 getMaxCamerasPerSample() const { return mMaxCamsPerSample; }
    uint32 getMaxParentLinkCount() const {
        const uint64 count = (uint64)getCount() * getMaxCamerasPerSample();
        if (count >= (uint64)((uint32)-1)) throw std::runtime_error("too many camera to sample links");
        return (uint32)count;
    }
    uint32 getSampleIdx(const uint32 link) const { return link / getMaxCamerasPerSample(); }
    uint32 getCameraIdx(const uint32 link) const {
        return getCameraIdx(link % getMaxCamerasPerSample(), getSampleIdx(link));
    }
    uint32 getCameraIdx(const uint32 slot, const uint32 sampleIdx) const {
        if (slot >= mMaxCamsPerSample || sampleIdx >= getCount()) return (uint32)-1;
        return mParentCameras[(uint64)sampleIdx * mMaxCamsPerSample + slot];
    }
    Real getDistanceToPlane(const Math::Vector3 &pWS, const uint32 i) const {
        return (pWS - mPositions[i]).dotProduct(mNormals[i]);
    }
    const Math::Vector3 *getAABBWS() const { return mAABBWS; }
    void computeAABB() {
        mAABBWS[0].set(REAL_MAX, REAL_MAX, REAL_MAX);
        mAABBWS[1].set(-REAL_MAX, -REAL_MAX, -REAL_MAX);
        for (uint32 i = 0; i < getCount(); ++i) {
            const Math::Vector3 &p = mPositions[i];
            const Real r = getMaxSamplingDistance(i) + Math::EPSILON;
            mAABBWS[0] = mAABBWS[0].minimum(Math::Vector3(p.x - r, p.y - r, p.z - r));
            mAABBWS[1] = mAABBWS[1].maximum(Math::Vector3(p.x + r, p.y + r, p.z + r));
        }
    }
    void reorder(const uint32 *targetIndices) {
        Utilities::Array<Math::Vector3>::reorder(mNormals, targetIndices);
        Utilities::Array<Math::Vector3>::reorder(mPositions, targetIndices);
        Utilities::Array<Real>::reorder(mConfidences, targetIndices);
        Utilities::Array<Real>::reorder(mScales, targetIndices);
        Utilities::Array<uint32>::reorder(mParentCameras, targetIndices, mMaxCamsPerSample);
        mTargets.assign(targetIndices, targetIndices + getCount());
    }
    void erase(const std::vector<uint32> &, const uint32) { throw std::runtime_error("erase is not shimmed"); }

    static const uint32 INVALID_INDEX = (uint32)-1;

    std::vector<Math::Vector3> mPositions, mNormals;
    std::vector<Real> mScales, mConfidences;
    std::vector<uint32> mParentCameras, mTargets;
    uint32 mMaxCamsPerSample = 1;
    Real mMaxRelativeSamplingDistance = 2.0;
    Math::Vector3 mAABBWS[2];
};
}  // namespace SurfaceReconstruction
#endif
