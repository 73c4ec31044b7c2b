// Shim of BaseProject Graphics/Color.h: an RGBA value (the DMC vertex colour).
#ifndef TSR_SHIM_COLOR_H
#define TSR_SHIM_COLOR_H
#include "Platform/DataTypes.h"
namespace Graphics {
class Color {
public:
    Color(float r, float g, float b, float a) : mR(r), mG(g), mB(b), mA(a) {}
    float getRed() const { return mR; }
    float getGreen() const { return mG; }
    float getBlue() const { return mB; }
    float getAlpha() const { return mA; }
private:
    float mR, mG, mB, mA;
};
}  // namespace Graphics
#endif
