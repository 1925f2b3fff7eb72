// Compatibility name of the reference header include/Kdtree.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KDTREE_H
#define BBKDE_COMPAT_KDTREE_H
#include "bbkde.hpp"
#endif
