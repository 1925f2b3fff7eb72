// Compatibility name of the reference header include/CudaDirectKde.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_CUDADIRECTKDE_H
#define BBKDE_COMPAT_CUDADIRECTKDE_H
#include "bbkde.hpp"
#endif
