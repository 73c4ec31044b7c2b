// Shadow of the reference's Geometry/FlexibleMesh.h for the reference build:
// it records the vertices and triangles DualMarchingCells adds.  The
// post-processing its constructor runs (deleteIsolatedGeometry, fillHoles,
// computeNormalsWeightedByAngles) does nothing here, so the recorded mesh is
// the raw extraction (extractMesh).
#ifndef TSR_SHIM_FLEXIBLEMESH_H
#define TSR_SHIM_FLEXIBLEMESH_H
#include <vector>
#include "Math/Vector3.h"

namespace SurfaceReconstruction {
struct EdgeConflict {
    uint32 mEdgeIdx;
    std::vector<uint32> mTriangles;
};

class FlexibleMesh {
public:
    void reserve(uint32 v, uint32 /*e*/, uint32 i) {
        mPositions.reserve(v);
        mScales.reserve(v);
        mIndices.reserve(i);
    }
    void addVertex(const Math::Vector3 &, const Math::Vector3 &, const Math::Vector3 &position, const Real scale) {
        mPositions.push_back(position);
        mScales.push_back(scale);
    }
    void addTriangle(const uint32 t[3]) { mIndices.insert(mIndices.end(), t, t + 3); }
    uint32 getVertexCount() const { return (uint32)mPositions.size(); }
    uint32 getIndexCount() const { return (uint32)mIndices.size(); }
    void clear() { mPositions.clear(); mScales.clear(); mIndices.clear(); }
    void deleteIsolatedGeometry(uint32) {}
    void fillHoles() {}
    void computeNormalsWeightedByAngles() {}
    const std::vector<EdgeConflict> &getEdgeConflicts() const { return mConflicts; }

    std::vector<Math::Vector3> mPositions;
    std::vector<Real> mScales;
    std::vector<uint32> mIndices;
    std::vector<EdgeConflict> mConflicts;
};
}  // namespace SurfaceReconstruction
#endif
