// Shim of BaseProject Platform/Utilities/HelperFunctions.h (included, not used,
// by the hot path).
#ifndef TSR_SHIM_HELPERFUNCTIONS_H
#define TSR_SHIM_HELPERFUNCTIONS_H
#include "Platform/DataTypes.h"
#endif
