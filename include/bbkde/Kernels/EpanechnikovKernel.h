// Compatibility name of the reference header include/Kernels/EpanechnikovKernel.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KERNELS_EPANECHNIKOVKERNEL_H
#define BBKDE_COMPAT_KERNELS_EPANECHNIKOVKERNEL_H
#include "../bbkde.hpp"
#endif
