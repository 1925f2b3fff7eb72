// Compatibility name of the reference header include/Attributes/AdaKdeAttributes.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_ATTRIBUTES_ADAKDEATTRIBUTES_H
#define BBKDE_COMPAT_ATTRIBUTES_ADAKDEATTRIBUTES_H
#include "../bbkde.hpp"
#endif
