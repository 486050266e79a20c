/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle for the label-indexed anisotropic
 * elastic staggered-grid FDTD of Jerome-Graves/pulse-echo-azimuthal-simulation
 * (sim/core/fdtd.py, forward_fused_labels :1618-1816). It is the checker for
 * the CUDA product path and the timed CPU port in bench.py; the product
 * package never loads it. Parity of this restatement is pinned by
 * tests/test_oracle_pins.py against (a) the reference's own kernel sources
 * compiled for the host (oracle/_ref, recipe oracle/build_ref.py) bit for bit,
 * and (b) golden traces of the reference's NumPy array path
 * (tests/golden/make_golden.py).
 *
 * Build: see oracle/build_oracle.py (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int nz, ny, nx;
    int n_mat;
    int nc;
    double coeffs[4];
    double inv_h, dt, dt_h;      /* already-rounded scalars, cast to REAL inside */
    int record;                  /* 0 pressure, 1 vx, 2 vy, 3 vz */
    int damped_record;           /* 1: pressure from end-of-step damped stress */
    int fma_mode;                /* 0 separate rounding, 1 product FMA placement */
    int nt;
    int n_threads;
    int n_src;
    int n_rec_groups;
    const int32_t *mats;         /* (nz, ny, nx) material index */
    const void *ctab;            /* (n_mat, 36) REAL */
    const void *rho;             /* (n_mat,) REAL */
    const float *damp;           /* (nz, ny, nx) combined damping or NULL */
    const int64_t *src_idx;      /* (n_src,) flat C-order cell index */
    const void *src_w;           /* (n_src,) REAL */
    const void *wavelet;         /* (nt,) REAL */
    const int64_t *rec_off;      /* (n_rec_groups + 1,) CSR offsets */
    const int64_t *rec_idx;      /* flat cell index per entry */
    const void *rec_w;           /* REAL weight per entry */
} OracleProblem;

#define REAL float
#define SUFFIX _f32
#define FMA_FN fmaf
#include "fdtd_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef FMA_FN

#define REAL double
#define SUFFIX _f64
#define FMA_FN fma
#include "fdtd_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef FMA_FN

int oracle_abi_version(void) { return 1; }
int oracle_problem_size(void) { return (int)sizeof(OracleProblem); }
