/*
 * CPU oracle for the RayGauss ray caster — TEST INFRASTRUCTURE ONLY (never on the product path).
 * Instantiates rg_oracle_impl.h in FP32 (_f32: literal restatement of the reference's FP32
 * arithmetic) and FP64 (_f64: the same algorithm in double, the accuracy yardstick).
 * Built by oracle/Makefile into oracle/liboracle.so; loaded only by tests/, smoke() and the
 * cpu_baseline leg of bench.py through oracle/oracle.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* 1: gather ray candidates through the grid prefilter (orc_grid.h); 0: scan every Gaussian.  Both
 * give the same candidate lists; the switch lets the tests check that. */
static int orc_grid_enabled = 1;
void orc_set_grid(int on) { orc_grid_enabled = on ? 1 : 0; }

#define REAL float
#define SFX _f32
#include "rg_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX _f64
#include "rg_oracle_impl.h"
#undef REAL
#undef SFX

int orc_num_threads(void) {
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
