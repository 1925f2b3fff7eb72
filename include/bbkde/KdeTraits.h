// Compatibility name of the reference header include/KdeTraits.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KDETRAITS_H
#define BBKDE_COMPAT_KDETRAITS_H
#include "bbkde.hpp"
#endif
