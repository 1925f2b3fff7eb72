// Compatibility name of the reference header include/Attributes/PointWeights.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_ATTRIBUTES_POINTWEIGHTS_H
#define BBKDE_COMPAT_ATTRIBUTES_POINTWEIGHTS_H
#include "../bbkde.hpp"
#endif
