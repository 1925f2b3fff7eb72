// Compatibility name of the reference header include/MarginalDensityAssociator.h:
// everything lives in bbkde.hpp (the C++ drop-in over libbbkde.so).
#ifndef BBKDE_COMPAT_MARGINALDENSITYASSOCIATOR_H
#define BBKDE_COMPAT_MARGINALDENSITYASSOCIATOR_H
#include "bbkde.hpp"
#endif
