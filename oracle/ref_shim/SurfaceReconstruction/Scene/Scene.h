// Shadow of the reference's Scene/Scene.h for the reference build (test
// infrastructure): only the singleton accessors the hot-path sources call
// (Scene.h of the reference pulls in cameras, images, FSSF and rendering).
#ifndef TSR_SHIM_SCENE_H
#define TSR_SHIM_SCENE_H
#include "Platform/DataTypes.h"
#include "Platform/Storage/Path.h"

namespace SurfaceReconstruction {
class Cameras;
class Samples;
class Tree;

class Scene {
public:
    static Scene &getSingleton();
    Samples &getSamples();
    const Samples &getSamples() const;
    const Cameras &getCameras() const;
    const Tree *getTree() const;
    uint32 getMinIsleSize() const;
};
}  // namespace SurfaceReconstruction
#endif
