/* Shim that lets the reference's OpenCL C kernel (tcoh.cl) compile as plain
 * C, so that the reference itself can run on the host cores as a checker and
 * as the timed CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY: used by oracle/Makefile to build oracle/_ref/,
 * never by the product.
 *
 * Two builds. Generic: the OpenCL build constants that ocl.c:222-229 passes
 * with -D become run-time globals (set by ref_runner.c before each run),
 * except NPAIRS, which tcoh.cl tests with #if and is therefore given on the
 * compiler command line (one library per value). Specialised
 * (TCOH_REF_SPECIALISED, oracle/build_ref_variants.py): every constant is
 * given with -D on the command line, exactly as ocl.c builds the kernel for
 * one configuration, so that the compiler sees constant trip counts and
 * fixed-size private arrays, as the OpenCL JIT does. <tgmath.h> keeps log, sqrt, hypot, fabs,
 * fmin, fmax and copysign in single precision on float arguments, as in
 * OpenCL C; the compiler is run without floating-point contraction.
 */
#ifndef TCOH_REF_SHIM_H
#define TCOH_REF_SHIM_H

#include <math.h>
#include <stddef.h>
#include <tgmath.h>

typedef unsigned char uchar;
typedef struct {
    float x, y;
} float2;

extern int ref_N, ref_WA, ref_WR, ref_W, ref_SHP_TEST, ref_EMI, ref_BIAS,
    ref_MIN_LOOKS, ref_KS_MAX, ref_PAIRS_ALL;
extern float ref_AD_NORM, ref_AD_SIGMA, ref_AD_CRIT, ref_TLOG_CRIT;
extern __thread int ref_gid[2];

#ifndef TCOH_REF_SPECIALISED
#define N          ref_N
#define WA         ref_WA
#define WR         ref_WR
#define W          ref_W
#define SHP_TEST   ref_SHP_TEST
#define EMI        ref_EMI
#define BIAS       ref_BIAS
#define MIN_LOOKS  ref_MIN_LOOKS
#define KS_MAX     ref_KS_MAX
#define AD_NORM    ref_AD_NORM
#define AD_SIGMA   ref_AD_SIGMA
#define AD_CRIT    ref_AD_CRIT
#define TLOG_CRIT  ref_TLOG_CRIT
#define PAIRS_ALL  ref_PAIRS_ALL
#endif

#define __kernel
#define __global
#define rsqrt(x) (1.0f / sqrtf(x))
#define get_global_id(d) ref_gid[d]

#endif
