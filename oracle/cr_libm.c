/*
 * cr_libm.c -- exp, expm1 and log1p with external linkage, correctly rounded
 * (cr_libm.h).  TEST INFRASTRUCTURE.  Linked into an oracle executable, these
 * definitions take the place of the C library's for every call in the
 * program: the reference's sources stay unmodified and run as they would on
 * a correctly rounded C library.
 */
#define CG_CR_LIBM_NO_RENAME
#include "cr_libm.h"

double exp(double x) { return cg_cr_exp(x); }
double expm1(double x) { return cg_cr_expm1(x); }
double log1p(double x) { return cg_cr_log1p(x); }
