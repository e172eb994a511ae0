/*
 * CPU ORACLE -- test infrastructure, not the product: the checker the GPU path is
 * compared against. Only tests/, the smoke check and bench.py's cpu_baseline leg load
 * it. Built by oracle/build.py into oracle/liboracle.so (g++ -O2 -ffp-contract=off
 * -fopenmp), both precisions in one library.
 */
#include <math.h>

typedef struct orc_geo {
  int ndim;
  int n[3];   /* logical extents, ghosts included */
  int ext[3]; /* padded extents */
  int s[3];   /* strides */
  int lo[3], hi[3];
  int dir;    /* Dirichlet faces, bit 2 * axis + side */
  int R;
} orc_geo;

#define REAL float
#define SFX _f32
#define FMAF fmaf
#include "oracle_impl.h"
#undef REAL
#undef SFX
#undef FMAF

#define REAL double
#define SFX _f64
#define FMAF fma
#include "oracle_impl.h"
