// Compatibility name of the reference header include/KernelDensity.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KERNELDENSITY_H
#define BBKDE_COMPAT_KERNELDENSITY_H
#include "bbkde.hpp"
#endif
