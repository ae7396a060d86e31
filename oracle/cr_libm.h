/*
 * cr_libm.h -- correctly rounded exp, expm1 and log1p for the oracles.
 * TEST INFRASTRUCTURE.
 *
 * Each function evaluates in 113-bit quad precision (libquadmath) and rounds
 * once to double, which is the correctly rounded result except for
 * arguments whose value lies within about 2^-110 of a rounding midpoint
 * (none is known; e^x is never a midpoint for x != 0).
 *
 * The C library's exp, expm1 and log1p are accurate to about half an ulp
 * but not correctly rounded, and libraries differ in which last bits they
 * return.  A "strict_cr" oracle -- the reference's sources, or the C
 * restatement, built with these functions in place of the C library's --
 * is what a correctly rounded C library would compute, and what the CUDA
 * parity build (cg_crmath.h) is compared with bit for bit.
 *
 * Included with -include: renames the three calls in the including file.
 */
#ifndef CG_CR_LIBM_H
#define CG_CR_LIBM_H
#include <math.h>
#include <quadmath.h>

static inline double cg_cr_exp(double x) { return (double)expq((__float128)x); }
static inline double cg_cr_expm1(double x) { return (double)expm1q((__float128)x); }
static inline double cg_cr_log1p(double x) { return (double)log1pq((__float128)x); }

#ifndef CG_CR_LIBM_NO_RENAME
#define exp cg_cr_exp
#define expm1 cg_cr_expm1
#define log1p cg_cr_log1p
#endif
#endif
