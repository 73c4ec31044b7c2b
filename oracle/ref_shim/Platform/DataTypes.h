// Shim of BaseProject Platform/DataTypes.h for the reference build: fixed-width
// integer names and Real = double (the FP64 oracle's precision).
#ifndef TSR_SHIM_DATATYPES_H
#define TSR_SHIM_DATATYPES_H
#include <cassert>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <iostream>

typedef int8_t int8;
typedef uint8_t uint8;
typedef int16_t int16;
typedef uint16_t uint16;
typedef int32_t int32;
typedef uint32_t uint32;
typedef int64_t int64;
typedef uint64_t uint64;
typedef double Real;

#define REAL_MAX DBL_MAX
#define ceilr ceil
#define floorr floor
#define log2r log2
#define sqrtr sqrt
#define fabsr fabs
#define powr pow
#define expr exp
#define cosr cos
#define sinr sin
#define acosr acos

#endif
