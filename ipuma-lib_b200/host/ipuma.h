// Umbrella header of the drop-in API (src/ipuma.h).
#ifndef IPUMA_H
#define IPUMA_H
#include "ipu_batch_affine.h"
#endif
