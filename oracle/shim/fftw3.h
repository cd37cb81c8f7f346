/*
 * fftw3.h -- compatibility shim (TEST INFRASTRUCTURE ONLY).
 *
 * Declares the single-precision FFTW3 API names that FWI-EDU calls.  The
 * transforms are implemented in shim.c by this project's own double-precision
 * FFT (radix-2 plus Bluestein for other lengths), with FFTW's conventions:
 * forward sign -1, backward sign +1, no normalisation, r2c of n real samples
 * gives n/2+1 complex bins, c2r reads n/2+1 bins and ignores the imaginary
 * parts of the DC and Nyquist bins.
 */
#ifndef FWI_SHIM_FFTW3_H
#define FWI_SHIM_FFTW3_H

#include <stddef.h>

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

typedef float fftwf_complex[2];
typedef struct fwi_shim_fftwf_plan_s *fftwf_plan;

#ifdef __cplusplus
extern "C" {
#endif
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int n);
void fftwf_cleanup_threads(void);
#ifdef __cplusplus
}
#endif

#endif
