// Shim of BaseProject Math/MathHelper.h (see MathCore.h).
#ifndef TSR_SHIM_MATHHELPER_H
#define TSR_SHIM_MATHHELPER_H
#include <vector>
#include "Math/MathCore.h"
#include "Math/Vector3.h"
#endif
