/*
 * Declarations-only stand-in for <fftw3.h> (FFTW 3 public API names).
 *
 * TEST INFRASTRUCTURE, not product code.  The reference's BSSN header
 * (components/bssn/bssn.h) includes utils/Fourier.h, which includes
 * <fftw3.h>; FFTW is not installed in this image.  The evolution path that
 * the oracle driver exercises never executes an FFT (the Fourier helper is
 * only used under USE_GENERALIZED_NEWTON, components/bssn/bssn.cc:203), so
 * declarations are enough for the reference's sources to compile.  No symbol
 * declared here is defined anywhere; a link error would mean an FFT call was
 * reached, which the oracle build must not allow.
 */
#ifndef CG_ORACLE_FFTW3_STUB_H
#define CG_ORACLE_FFTW3_STUB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef long double fftwl_complex[2];
typedef struct fftw_plan_s *fftw_plan;
typedef struct fftwl_plan_s *fftwl_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out,
                               unsigned flags);

void *fftwl_malloc(size_t n);
void fftwl_free(void *p);
void fftwl_execute(const fftwl_plan p);
void fftwl_destroy_plan(fftwl_plan p);
void fftwl_execute_dft_r2c(const fftwl_plan p, long double *in,
                           fftwl_complex *out);
void fftwl_execute_dft_c2r(const fftwl_plan p, fftwl_complex *in,
                           long double *out);
fftwl_plan fftwl_plan_dft_r2c_3d(int n0, int n1, int n2, long double *in,
                                 fftwl_complex *out, unsigned flags);
fftwl_plan fftwl_plan_dft_c2r_3d(int n0, int n1, int n2, fftwl_complex *in,
                                 long double *out, unsigned flags);
fftwl_plan fftwl_plan_dft_r2c_1d(int n, long double *in, fftwl_complex *out,
                                 unsigned flags);
fftwl_plan fftwl_plan_dft_c2r_1d(int n, fftwl_complex *in, long double *out,
                                 unsigned flags);

#ifdef __cplusplus
}
#endif

#endif
