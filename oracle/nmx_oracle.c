/*
 * CPU oracle for the dense-factorization path -- TEST INFRASTRUCTURE ONLY.
 *
 * Built into oracle/liboracle.so and loaded by tests/, the smoke check and
 * the benchmark's CPU baseline as the checker.  The shipped library
 * (numax_b200/libnmxla.so) never links or calls it.
 *
 * The restated algorithms live in nmx_oracle_impl.h, instantiated here for
 * float64 and float32.  Constants are numax's:
 *   NMX_PIVOT_FLOOR  numax/linalg/common.mojo:27  (_PIVOT_FLOOR = 1e-30)
 *   NMX_MIN_SPLIT    numax/linalg/panel.mojo:434  (_MIN_SPLIT = 4)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <omp.h>

#define NMX_PIVOT_FLOOR 1e-30
#define NMX_MIN_SPLIT 4
#define NMX_BATCH_MAX_N 128

#define T double
#define FN(name) name##_f64
#include "nmx_oracle_impl.h"
#undef T
#undef FN

#define T float
#define FN(name) name##_f32
#include "nmx_oracle_impl.h"
#undef T
#undef FN

int orc_max_threads(void) { return omp_get_max_threads(); }
