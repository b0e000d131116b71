/* orc_sim.c -- instantiates the engine restatement in float32 and float64.
 * TEST INFRASTRUCTURE ONLY (see umag_oracle.h). */
#include "umag_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* engine/run.go:14-43 defaults, engine/torque.go:27 GammaLL */
void orc_solver_defaults(orc_solver* s) {
    memset(s, 0, sizeof(*s));
    s->dt = 1e-15;
    s->max_err = 1e-5;
    s->rel_err = 1e-4;
    s->min_slope = 1e8;
    s->headroom = 0.8;
    s->gamma_ll = 1.7595e11;
    s->solver = 5;
}

#define REAL float
#define SFX f32
#include "orc_sim.inc"
#undef REAL
#undef SFX

#define REAL double
#define SFX f64
#include "orc_sim.inc"
#undef REAL
#undef SFX
