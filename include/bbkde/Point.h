// Compatibility name of the reference header include/Point.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_POINT_H
#define BBKDE_COMPAT_POINT_H
#include "bbkde.hpp"
#endif
