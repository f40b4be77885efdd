/*
 * CPU oracle for the BGK3D_HIT hot path (TEST INFRASTRUCTURE ONLY).
 *
 * Restates, in plain C, the reference's Taylor-Green init (SRC/init.F90),
 * single-rank periodic halo fill (SRC/bcond.comm.step3.F90), fused
 * stream-collide (SRC/col_MC.F90) and diagnostics (SRC/diagno.F90,
 * SRC/dissipation.F90). Three storage forms are compiled from one body
 * (bgk_oracle_impl.h):
 *   _f64  double storage, double arithmetic  (reference DOUBLE_P build)
 *   _f32  float storage, float arithmetic    (reference default build)
 *   _f16  binary16 storage of scale*(f - w), float arithmetic (no reference
 *         counterpart; the reference stops on HALF_P, SRC/precision.F90:40-43);
 *         its collision is the fused-multiply-add form defined in
 *         fast16_cell, shared operation for operation with the CUDA kernels
 *
 * Parity unpinned: the reference has no tests or golden vectors, and its
 * Fortran/MPI build cannot be compiled here. Only tests/, the smoke check and
 * the benchmark's CPU-baseline leg may load this library.
 *
 * Build with -ffp-contract=off and without fast-math so that every operation
 * rounds as written (see oracle/Makefile).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SUF _f64
#define STOR double
#define REAL double
#define SIN sin
#define COS cos
#define SQRT sqrt
#define ENC(L, x) (x)
#define DEC(L, s) (s)
#include "bgk_oracle_impl.h"
#undef SUF
#undef STOR
#undef REAL
#undef SIN
#undef COS
#undef SQRT
#undef ENC
#undef DEC

#define SUF _f32
#define STOR float
#define REAL float
#define SIN sinf
#define COS cosf
#define SQRT sqrtf
#define ENC(L, x) (x)
#define DEC(L, s) (s)
#include "bgk_oracle_impl.h"
#undef SUF
#undef STOR
#undef REAL
#undef SIN
#undef COS
#undef SQRT
#undef ENC
#undef DEC

#define FAST16
#define SUF _f16
#define STOR _Float16
#define REAL float
#define SIN sinf
#define COS cosf
#define SQRT sqrtf
#define ENC(L, x) ((_Float16)((x) * (L)->scale))
#define DEC(L, s) ((float)(s) * (L)->inv_scale)
#include "bgk_oracle_impl.h"
#undef FAST16
#undef SUF
#undef STOR
#undef REAL
#undef SIN
#undef COS
#undef SQRT
#undef ENC
#undef DEC

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* Timed CPU baseline: `steps` iterations of the reference loop body
   (boundaries + col_MC, SRC/bgk3d_HIT.F90:131,140) in double precision on an
   already-initialised lattice, in the row-vectorised form (bit-identical to
   orc_step_f64). Returns elapsed seconds. */
double orc_time_steps_f64(orc_lat_f64 *L, double svisc, int steps) {
    double t0 = now_s();
    for (int s = 0; s < steps; ++s) orc_step_rows_f64(L, svisc);
    return now_s() - t0;
}
