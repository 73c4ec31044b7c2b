// Shadow of the reference's Scene/Camera/Cameras.h: camera centres only, with
// the reference's validity rule (index below the camera count,
// Cameras.h:173-176) and INVALID_ID (Cameras.cpp:29).
#ifndef TSR_SHIM_CAMERAS_H
#define TSR_SHIM_CAMERAS_H
#include <vector>
#include "Math/Vector3.h"
#include "Platform/Storage/Path.h"

namespace SurfaceReconstruction {
class Cameras {
public:
    bool isValid(const uint32 cameraIdx) const { return cameraIdx < (uint32)mPositions.size(); }
    Math::Vector3 getPositionWS(const uint32 cameraIdx) const { return mPositions[cameraIdx]; }
    uint32 getCount() const { return (uint32)mPositions.size(); }
    std::vector<Math::Vector3> mPositions;
    static const uint32 INVALID_ID = (uint32)-1;
};
}  // namespace SurfaceReconstruction
#endif
