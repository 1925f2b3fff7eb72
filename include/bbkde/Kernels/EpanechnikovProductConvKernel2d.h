// Compatibility name of the reference header include/Kernels/EpanechnikovProductConvKernel2d.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KERNELS_EPANECHNIKOVPRODUCTCONVKERNEL2D_H
#define BBKDE_COMPAT_KERNELS_EPANECHNIKOVPRODUCTCONVKERNEL2D_H
#include "../bbkde.hpp"
#endif
