// Compatibility name of the reference header include/Kernels/EpanechnikovProductKernel2d.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KERNELS_EPANECHNIKOVPRODUCTKERNEL2D_H
#define BBKDE_COMPAT_KERNELS_EPANECHNIKOVPRODUCTKERNEL2D_H
#include "../bbkde.hpp"
#endif
