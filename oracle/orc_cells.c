/* orc_cells.c -- instantiates the per-cell oracle kernels in float32 and
 * float64.  TEST INFRASTRUCTURE ONLY (see umag_oracle.h). */
#include "umag_oracle.h"
#include <math.h>
#include <stddef.h>

#define REAL float
#define SFX f32
#include "orc_cells.inc"
#undef REAL
#undef SFX

#define REAL double
#define SFX f64
#include "orc_cells.inc"
#undef REAL
#undef SFX
