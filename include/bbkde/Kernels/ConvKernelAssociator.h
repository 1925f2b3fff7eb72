// Compatibility name of the reference header include/Kernels/ConvKernelAssociator.h: everything lives in
// bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_KERNELS_CONVKERNELASSOCIATOR_H
#define BBKDE_COMPAT_KERNELS_CONVKERNELASSOCIATOR_H
#include "../bbkde.hpp"
#endif
