// Compatibility name of the reference header include/DecoratedPoint.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_DECORATEDPOINT_H
#define BBKDE_COMPAT_DECORATEDPOINT_H
#include "bbkde.hpp"
#endif
