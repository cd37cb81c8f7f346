/* fwi_setup.h -- host-side per-model set-up of the B200 engine (internal). */
#ifndef FWI_SETUP_H
#define FWI_SETUP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Coefficient fields of one padded model window, in the device layout:
 * Nx columns of ld floats (ld = Nz rounded up to a multiple of 4), z fastest,
 * rows Nz..ld-1 zero.  ck = coef3*K (the reference multiplies coef3 by K first). */
typedef struct {
    int nz, nxx, pml, Nz, Nx, ld;
    float *c1, *c2, *ck, *irx, *irz, *ir; /* Nx*ld each, 64-byte aligned */
    float *K;                              /* Nx*ld, bulk modulus of the beta-scaled model */
    float invdx, invdz, invdxdx, invdzdz, invdtdt;
} fwi_coefs;

/* vpm, rhom: the window [nxx][nz] of the model.  Returns 0 or -1 (allocation). */
int fwi_setup_coefs(const float *vpm, const float *rhom, int nz, int nxx, int pml, float dx, float dz,
                    float dt, float fpeak, fwi_coefs *out);
void fwi_free_coefs(fwi_coefs *c);

/* checkpoint interval and count of checkpoint.c:47 and :66-75 */
int fwi_ck_interval(int nt);
int fwi_ck_count(int nt);

/* forward source term 1.0*src*K*dt*dt*invdx*invdz formed in double (propagation.c:558) */
double fwi_src_term_f64(float src, float K, float dt, float invdx, float invdz);
/* replay source / adjoint injection scale src*K*dt*dt*invdx*invdz in float (propagation.c:662, :681) */
float fwi_src_term_f32(float src, float K, float dt, float invdx, float invdz);
/* model operations of the FWI loop, acoustic2d_fwi.c:428-465, on [nx][nz] arrays:
 * trial:  vp = 1/(slow + perturb), water layer, clip, Gardner rho (310 vp^0.25), water, clip
 * update: slow += steplen*perturb, vp = 1/slow, water, clip, Gardner, water, clip, slow = 1/vp */
void fwi_model_trial(const float *slow, const float *perturb, float *vp, float *rho, int nx, int nz, int waterdepth,
                     float vp_water, float rho_water, float vpmin, float vpmax, float rhomin, float rhomax, int gardner);
void fwi_model_update(float *slow, float *vp, float *rho, const float *perturb, float steplen, int nx, int nz,
                      int waterdepth, float vp_water, float rho_water, float vpmin, float vpmax, float rhomin,
                      float rhomax, int gardner);
/* cosine taper coefficients 0.5(1+cos(pi*i/L)), i = 0..L (common.c:826-831) */
void fwi_taper_coefs(int L, float *out);

/* The residual filters and trace interpolation as matrices (column-major, float), so that the
 * device applies them to all traces of all shots as one GEMM each.
 * fwi_filter_operator: apply_traces_lowpass (filter 0, common.c:584-687) or apply_traces_bandpass
 *   (filter 1, :689-794) of length-n traces: FFT, the cosine-tapered window on the non-negative
 *   frequencies, inverse FFT, / n -- a circular convolution, C[i + j n] = h[(i - j) mod n].
 * fwi_interp_operator: interpolate_traces (:482-582) from ns to nt samples by r: M[i + j nt],
 *   rows i >= (ns - 1) r + 1 zero. */
void fwi_filter_window(int filter, int n, float fpass, float fcut, float dt, float *win);
void fwi_filter_operator(int filter, int n, float fpass, float fcut, float dt, float *C);
void fwi_interp_operator(int ns, int r, int nt, float *M);

/* The same filters and the interpolation as circular convolutions applied by FFT on the device.
 * fwi_filter_kernel: h[0..n) of apply_traces_lowpass/bandpass, the length-n circular kernel
 *   y[i] = sum_j h[(i - j) mod n] x[j] (FP64);
 * fwi_interp_kernel: g[0..N), N = (ns - 1) r + 1, of interpolate_traces: y[i] = sum_j g[(i - j r) mod N] x[j];
 * fwi_conv_size: M = the power of two >= 2n - 1, so that an M-point circular convolution of the
 *   zero-padded signal with the wrapped kernel equals the n-point one on [0, n);
 * fwi_conv_spectrum: G = FFT_M(wrapped h) / M, M complex floats as (re, im) pairs (FP64 FFT);
 * fwi_fft_twiddles: exp(-2 pi i k / M), k < M / 2, as (re, im) float pairs. */
void fwi_filter_kernel(int filter, int n, float fpass, float fcut, float dt, double *h);
void fwi_interp_kernel(int ns, int r, double *g);
int fwi_conv_size(int n);
void fwi_conv_spectrum(const double *h, int n, int M, float *G);
void fwi_fft_twiddles(int M, float *tw);
/* the same two tables in FP64 (for transforms that run in FP64) */
void fwi_conv_spectrum_f64(const double *h, int n, int M, double *G);
void fwi_fft_twiddles_f64(int M, double *tw);
/* fwi_bluestein_tables: the tables of an N-point DFT computed as an M-point convolution
 * (Bluestein; M = fwi_conv_size(N)): the chirp b_m = exp(i pi m^2 / N), m < N, then the spectra
 * FFT_M(b wrapped) / M and FFT_M(conj(b) wrapped) / M (b is even in m, so b_{-m} = b_m sits at
 * M - m), as (re, im) pairs: N + 2M complex values, FP64 (f64 != 0) or FP32. */
void fwi_bluestein_tables(int N, int M, int f64, void *out);

/* lowpass2d (filter 0, common.c:1042-1162) / bandpass2d (filter 1, :1164-1284) window over the
 * full Nx x Nz wavenumber plane of the padded field, W[ix * Nz + iz], from the reference's float
 * expressions (generate_frequency, common.c:333-361); the filter applies it between the 2-D DFTs
 * of the padded field (Bluestein transforms on the device, fwi_bluestein_tables). */
void fwi_wavenumber_window(int filter, int Nx, int Nz, float dx, float dz, float kpass, float kcut, float *W);

#ifdef __cplusplus
}
#endif
#endif
