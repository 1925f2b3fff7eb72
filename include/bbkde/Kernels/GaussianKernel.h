// Compatibility name of the reference header include/Kernels/GaussianKernel.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KERNELS_GAUSSIANKERNEL_H
#define BBKDE_COMPAT_KERNELS_GAUSSIANKERNEL_H
#include "../bbkde.hpp"
#endif
