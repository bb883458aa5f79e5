/*
 * phix_oracle.c -- CPU oracle for PhiX's explicit finite-difference time step.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference algorithm
 * used to check the sm_100a kernels.  The product never links or calls it.
 * Build: oracle/Makefile -> oracle/liboracle.so (gcc -O2 -ffp-contract=off), and
 * oracle/liboracle_omp.so (the same source with OpenMP on every per-cell loop:
 * the timed CPU baseline on all host cores; identical bits).
 *
 * Pinning: tests/test_oracle_pin.py checks this restatement, in fma_mode 0,
 * bit for bit against the reference's own CPU path compiled from its sources
 * (oracle/_ref, recipe in oracle/Makefile) and against the golden vectors in
 * tests/golden/ that the same recipe produced; fma_mode 1 is compared with
 * the reference's GPU build on a B200.
 *
 * Exported functions come in two precisions: *_f64 (double, the reference's
 * arithmetic) and *_f32 (float, the arithmetic of the FP32 kernels).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { OR_BC_NONE = 0, OR_BC_PERIODIC = 1, OR_BC_NOFLUX = 2, OR_BC_FIXED = 3 };
enum { OR_PW_IDENT = 0, OR_PW_AC = 1, OR_PW_DW = 2, OR_PW_CHAC_C = 3, OR_PW_CHAC_E = 4, OR_PW_MUL = 5 };
enum { OR_PHYS_AC = 0, OR_PHYS_CH = 1, OR_PHYS_CHAC = 2 };
enum { OR_EULER = 0, OR_RK4 = 1 };

/* Grid descriptor; same field order and sizes as phix_grid_t in
 * include/phix_b200.h plus the oracle-only fma_mode in the padding slot. */
typedef struct {
    int32_t dim;
    int32_t n[3];
    int32_t ghost;
    int32_t bc_type[6]; /* [2*axis + side], side 0 = low, 1 = high */
    int32_t fma_mode;   /* 0: no contraction, 1: contracted multiply-add */
    double d[3];
    double bc_val[6];
} or_grid_t;

#define REAL double
#define SFX _f64
#define FMA fma
#include "oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

#define REAL float
#define SFX _f32
#define FMA fmaf
#include "oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

int or_abi_version(void) { return 1; }

#ifdef OR_OMP
#include <omp.h>
/* Host threads the OpenMP build runs its loops on. */
int or_threads(void) { return omp_get_max_threads(); }
#else
int or_threads(void) { return 1; }
#endif
