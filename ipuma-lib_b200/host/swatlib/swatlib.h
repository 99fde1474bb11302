// Umbrella header of the swatlib helpers (src/swatlib/swatlib.h).
#ifndef IPUMA_B200_SWATLIB_H
#define IPUMA_B200_SWATLIB_H
#include "encoding.h"
#include "fasta.h"
#include "matrix.h"
#include "similarity.h"
#include "timing.hpp"
#include "vector.hpp"
#endif
