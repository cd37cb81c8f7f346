/*
 * fwi_setup.c -- host-side per-model set-up of the B200 engine.
 *
 * Builds the coefficient fields the device stencil streams: pad the model window
 * (pad_model2d, common.c:110-176), build the MEAL damping D and scale Beta
 * (mealCoefs2d, propagation.c:192-354), fold them into the model and the time
 * coefficients (propagation.c:513-529), then K, 1/rho and its derivatives
 * (acoustic_iso2d_rgfd_parameter, propagation.c:103-171, with the two-point edge
 * derivative of calculate_gradient2d, common.c:416-479).
 *
 * This runs once per (model window, peak frequency) and stays on the host on
 * purpose: the reference evaluates these fields with the C library's expf, logf
 * and powf and rounds double expressions to float at fixed points, and keeping
 * the same operation order here with the same libm gives identical coefficient
 * bits, which is what lets the device stencil reproduce the reference exactly.
 * The file is compiled with -O2 -fno-fast-math -ffp-contract=off.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fwi_setup.h"

#define AT(a, ix, iz, n1) (a)[(size_t)(ix) * (size_t)(n1) + (size_t)(iz)]

static float *falloc(size_t n)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, (n ? n : 1) * sizeof(float))) return NULL;
    memset(p, 0, (n ? n : 1) * sizeof(float));
    return (float *)p;
}

int fwi_ck_interval(int nt)
{
    float r = roundf(sqrtf(2.0f * (nt - 1)));
    return (int)(r > 3.0f ? r : 3.0f);
}

int fwi_ck_count(int nt)
{
    int d = fwi_ck_interval(nt), n = 0;
    for (int it = 0; it < nt; it++) n += (it % d == 0 || (it + 1) % d == 0);
    return n;
}

double fwi_src_term_f64(float src, float K, float dt, float invdx, float invdz)
{
    return 1.0 * src * K * dt * dt * invdx * invdz;
}

float fwi_src_term_f32(float src, float K, float dt, float invdx, float invdz)
{
    return src * K * dt * dt * invdx * invdz;
}

void fwi_taper_coefs(int L, float *out)
{
    for (int i = 0; i <= L; i++) {
        float x = (float)3.141592653589793 * i / L;
        out[i] = 0.5f * (1.0f + cosf(x));
    }
}

/* the absorbing-layer weight of layer l of n: 2^(d^alpha) - 1, d = l/n (propagation.c:173-190) */
static float layer_weight(float alpha, int l, int n)
{
    float d = (0.1f * l) / (0.1f * n);
    return expf(logf(2.0f) * powf(d, alpha)) - 1.0f;
}

void fwi_free_coefs(fwi_coefs *c)
{
    free(c->c1); free(c->c2); free(c->ck); free(c->irx); free(c->irz); free(c->ir); free(c->K);
    memset(c, 0, sizeof(*c));
}

int fwi_setup_coefs(const float *vpm, const float *rhom, int nz, int nxx, int pml, float dx, float dz,
                    float dt, float fpeak, fwi_coefs *o)
{
    memset(o, 0, sizeof(*o));
    const int Nz = nz + 2 * pml, Nx = nxx + 2 * pml, nl = pml;
    const size_t n = (size_t)Nz * Nx;
    o->nz = nz; o->nxx = nxx; o->pml = pml; o->Nz = Nz; o->Nx = Nx;
    o->ld = (Nz + 3) & ~3;
    o->invdx = 1.0f / dx;
    o->invdz = 1.0f / dz;
    o->invdxdx = 1.0f / (dx * dx);
    o->invdzdz = 1.0f / (dz * dz);
    o->invdtdt = 1.0f / (dt * dt);

    float *vp = falloc(n), *rho = falloc(n), *Dx = falloc(n), *Dz = falloc(n), *Bx = falloc(n), *Bz = falloc(n);
    float *K = falloc(n), *ir = falloc(n), *irx = falloc(n), *irz = falloc(n);
    size_t nl_out = (size_t)o->ld * Nx;
    o->c1 = falloc(nl_out); o->c2 = falloc(nl_out); o->ck = falloc(nl_out);
    o->irx = falloc(nl_out); o->irz = falloc(nl_out); o->ir = falloc(nl_out); o->K = falloc(nl_out);
    if (!vp || !rho || !Dx || !Dz || !Bx || !Bz || !K || !ir || !irx || !irz || !o->c1 || !o->c2 || !o->ck ||
        !o->irx || !o->irz || !o->ir || !o->K) {
        free(vp); free(rho); free(Dx); free(Dz); free(Bx); free(Bz); free(K); free(ir); free(irx); free(irz);
        fwi_free_coefs(o);
        return -1;
    }

    /* edge-replicating pad: interior, then top, bottom, left, right */
    for (int ix = 0; ix < nxx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            AT(vp, ix + nl, iz + nl, Nz) = AT(vpm, ix, iz, nz);
            AT(rho, ix + nl, iz + nl, Nz) = AT(rhom, ix, iz, nz);
        }
    for (int ix = 0; ix < Nx; ix++) {
        for (int iz = 0; iz < nl; iz++) {
            AT(vp, ix, iz, Nz) = AT(vp, ix, nl, Nz);
            AT(rho, ix, iz, Nz) = AT(rho, ix, nl, Nz);
        }
        for (int iz = nz + nl; iz < Nz; iz++) {
            AT(vp, ix, iz, Nz) = AT(vp, ix, nz + nl - 1, Nz);
            AT(rho, ix, iz, Nz) = AT(rho, ix, nz + nl - 1, Nz);
        }
    }
    for (int ix = 0; ix < nl; ix++)
        for (int iz = 0; iz < Nz; iz++) {
            AT(vp, ix, iz, Nz) = AT(vp, nl, iz, Nz);
            AT(rho, ix, iz, Nz) = AT(rho, nl, iz, Nz);
        }
    for (int ix = nxx + nl; ix < Nx; ix++)
        for (int iz = 0; iz < Nz; iz++) {
            AT(vp, ix, iz, Nz) = AT(vp, nxx + nl - 1, iz, Nz);
            AT(rho, ix, iz, Nz) = AT(rho, nxx + nl - 1, iz, Nz);
        }

    /* MEAL: per-side damping and scale; both default to 0 and 1 outside the layers */
    for (size_t i = 0; i < n; i++) { Bx[i] = 1.0f; Bz[i] = 1.0f; }
    const float pd = 2.0f, alpha = 2.5f, ppw_fd = 10.0f;
    const float Rcoef = powf(10.0f, -1.0f * ((log10f(nl) - 1.0f) / (log10f(2.0f))) - 3.0f - 0.5f * pd);
    const float logR = logf(Rcoef), s3 = sqrtf(3.0f);
    const float thick_x = nl * dx, thick_z = nl * dz;
    for (int ix = 0; ix < Nx; ix++)
        for (int l = 1; l <= nl; l++) {
            float w = layer_weight(alpha, l, nl);
            int zs[2] = {nl - l, Nz - nl - 1 + l}; /* top then bottom: the bottom write wins on overlap */
            for (int k = 0; k < 2; k++) {
                int iz = zs[k];
                float v = AT(vp, ix, iz, Nz);
                float d0 = -1.0f * (1.0f + pd) * v * logR / (2.0f * thick_z);
                float ppw = (v / s3) / (dz * fpeak);
                float beta = 2.0f * ppw / ppw_fd;
                AT(Dz, ix, iz, Nz) = d0 * w;
                AT(Bz, ix, iz, Nz) = 1.0f + (beta - 1.0f) * w;
            }
        }
    for (int l = 1; l <= nl; l++) {
        float w = layer_weight(alpha, l, nl);
        for (int iz = 0; iz < Nz; iz++) {
            int xs[2] = {nl - l, Nx - nl - 1 + l}; /* left then right */
            for (int k = 0; k < 2; k++) {
                int ix = xs[k];
                float v = AT(vp, ix, iz, Nz);
                float d0 = -1.0f * (1.0f + pd) * v * logR / (2.0f * thick_x);
                float ppw = (v / s3) / (dx * fpeak);
                float beta = 2.0f * ppw / ppw_fd;
                AT(Dx, ix, iz, Nz) = d0 * w;
                AT(Bx, ix, iz, Nz) = 1.0f + (beta - 1.0f) * w;
            }
        }
    }

    /* combine, fold into the model, time coefficients formed in double and rounded to float.
     * Away from the layers Dx = Dz = 0 and Bx = Bz = 1 exactly, so D = 0, Beta = 1 and the
     * expressions reduce exactly to coef1 = 2, coef2 = -1, coef3 = dt*dt: no libm call needed there. */
    const float dtdt = dt * dt;
    const int ld = o->ld;
    for (int ix = 0; ix < Nx; ix++) {
        int xband = ix < nl || ix >= Nx - nl;
        for (int iz = 0; iz < Nz; iz++) {
            size_t i = (size_t)ix * Nz + iz;
            float c1, c2, c3;
            if (xband || iz < nl || iz >= Nz - nl) {
                float D = sqrtf(powf(Dx[i], 2.0f) + powf(Dz[i], 2.0f));
                float B = sqrtf(powf(Bx[i] - 1.0f, 2.0f) + powf(Bz[i] - 1.0f, 2.0f)) + 1.0f;
                D /= B;
                vp[i] /= B;
                rho[i] *= B;
                c1 = (float)((2.0 - dt * dt * D * D) / (1.0 + dt * D));
                c2 = (float)(-1.0 * (1.0 - dt * D) / (1.0 + dt * D));
                c3 = (float)((dt * dt) / (1.0 + dt * D));
            } else {
                c1 = 2.0f;
                c2 = -1.0f;
                c3 = (float)((double)dtdt / 1.0);
            }
            AT(o->c1, ix, iz, ld) = c1;
            AT(o->c2, ix, iz, ld) = c2;
            Dx[i] = c3; /* Dx is free from here on: keep coef3 until K is known */
        }
    }

    /* K, 1/rho and d(1/rho)/dx, d(1/rho)/dz: two-point at the edges, 12-point optimised inside */
    for (size_t i = 0; i < n; i++) {
        K[i] = rho[i] * vp[i] * vp[i];
        ir[i] = 1.0f / rho[i];
    }
    for (int ix = 0; ix < Nx; ix++)
        for (int iz = 0; iz < Nz; iz++) {
            size_t i = (size_t)ix * Nz + iz;
            if (ix == 0) irx[i] = (ir[i + Nz] - ir[i]) / dx;
            else if (ix == Nx - 1) irx[i] = (ir[i] - ir[i - Nz]) / dx;
            else irx[i] = (ir[i + Nz] - ir[i - Nz]) / (2.0f * dx);
            if (iz == 0) irz[i] = (ir[i + 1] - ir[i]) / dz;
            else if (iz == Nz - 1) irz[i] = (ir[i] - ir[i - 1]) / dz;
            else irz[i] = (ir[i + 1] - ir[i - 1]) / (2.0f * dz);
        }
    const float G1 = 0.91067892f, G2 = -0.34187892f, G3 = 0.13833962f;
    const float G4 = -0.04880710f, G5 = 0.01302148f, G6 = -0.00199047f;
    for (int ix = 6; ix < Nx - 6; ix++)
        for (int iz = 6; iz < Nz - 6; iz++) {
            size_t i = (size_t)ix * Nz + iz;
            const float *r = ir + i;
            irx[i] = (G1 * (r[Nz] - r[-Nz]) + G2 * (r[2 * Nz] - r[-2 * Nz]) + G3 * (r[3 * Nz] - r[-3 * Nz]) +
                      G4 * (r[4 * Nz] - r[-4 * Nz]) + G5 * (r[5 * Nz] - r[-5 * Nz]) + G6 * (r[6 * Nz] - r[-6 * Nz])) *
                     o->invdx;
            irz[i] = (G1 * (r[1] - r[-1]) + G2 * (r[2] - r[-2]) + G3 * (r[3] - r[-3]) + G4 * (r[4] - r[-4]) +
                      G5 * (r[5] - r[-5]) + G6 * (r[6] - r[-6])) *
                     o->invdz;
        }
    for (int ix = 0; ix < Nx; ix++)
        for (int iz = 0; iz < Nz; iz++) {
            size_t i = (size_t)ix * Nz + iz;
            AT(o->ck, ix, iz, ld) = Dx[i] * K[i];
            AT(o->ir, ix, iz, ld) = ir[i];
            AT(o->irx, ix, iz, ld) = irx[i];
            AT(o->irz, ix, iz, ld) = irz[i];
            AT(o->K, ix, iz, ld) = K[i];
        }
    free(vp); free(rho); free(Dx); free(Dz); free(Bx); free(Bz); free(K); free(ir); free(irx); free(irz);
    return 0;
}

/* set_waterlayer_value, clip_model, v2slow/slow2v, vp2density (common.c:218-330, 898-924) */
static void water_layer(float *m, float v, int wd, int nx, int nz)
{
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < wd; iz++) m[(size_t)ix * nz + iz] = v;
}
static void clip(float *m, size_t n, float lo, float hi)
{
    for (size_t i = 0; i < n; i++) {
        if (m[i] > hi) m[i] = hi;
        else if (m[i] < lo) m[i] = lo;
    }
}
static void reciprocal(const float *a, float *b, size_t n)
{
    for (size_t i = 0; i < n; i++) b[i] = a[i] != 0.0f ? 1.0f / a[i] : 0.0f;
}
static void gardner(const float *vp, float *rho, size_t n)
{
    for (size_t i = 0; i < n; i++) rho[i] = 310.0f * powf(vp[i], 0.25f);
}

void fwi_model_trial(const float *slow, const float *perturb, float *vp, float *rho, int nx, int nz, int waterdepth,
                     float vp_water, float rho_water, float vpmin, float vpmax, float rhomin, float rhomax, int g)
{
    size_t n = (size_t)nx * nz;
    for (size_t i = 0; i < n; i++) vp[i] = slow[i] + perturb[i];
    reciprocal(vp, vp, n);
    water_layer(vp, vp_water, waterdepth, nx, nz);
    clip(vp, n, vpmin, vpmax);
    if (g == 1) {
        gardner(vp, rho, n);
        water_layer(rho, rho_water, waterdepth, nx, nz);
        clip(rho, n, rhomin, rhomax);
    }
}

void fwi_model_update(float *slow, float *vp, float *rho, const float *perturb, float steplen, int nx, int nz,
                      int waterdepth, float vp_water, float rho_water, float vpmin, float vpmax, float rhomin,
                      float rhomax, int g)
{
    size_t n = (size_t)nx * nz;
    for (size_t i = 0; i < n; i++) slow[i] = slow[i] + steplen * perturb[i];
    reciprocal(slow, vp, n);
    water_layer(vp, vp_water, waterdepth, nx, nz);
    clip(vp, n, vpmin, vpmax);
    if (g == 1) {
        gardner(vp, rho, n);
        water_layer(rho, rho_water, waterdepth, nx, nz);
        clip(rho, n, rhomin, rhomax);
    }
    reciprocal(vp, slow, n);
}

/* ------------------------------------------------------------ residual filters, interpolation */
/* The window values come from the reference's own float expressions (apply_traces_lowpass and
 * apply_traces_bandpass; the bandpass forms its cosine argument in double because PI is a double
 * constant there).  Only entries 0..n/2 are used (the non-negative frequencies of an r2c FFT). */
void fwi_filter_window(int filter, int n, float fpass, float fcut, float dt, float *win)
{
    const float df = 1.0f / (n * dt);
    for (int it = 0; it < n; it++) {
        const float f = it * df;
        if (filter == 0) {
            const float taperLen = fcut - fpass;
            if (f < fpass) win[it] = 1.0f;
            else if (f >= fpass && f <= fcut)
                win[it] = 0.5f * (1.0f + cosf((float)3.141592653589793 * (f - fpass) / taperLen));
            else win[it] = 0.0f;
        } else {
            const float lo = fpass, hi = fcut - fpass;
            if (f < fpass) win[it] = 0.5f * (1.0f + cosf(3.141592653589793 * (fpass - f) / lo));
            else if (f >= fpass && f <= fcut) win[it] = 0.5f * (1.0f + cosf(3.141592653589793 * (f - fpass) / hi));
            else win[it] = 0.0f;
        }
    }
}

/* h[m] = (1/n) sum_k W(k) cos(2 pi k m / n) with W(k) = win[min(k, n - k)] (the real window seen
 * by a real signal's full spectrum), in double; k m mod n is stepped incrementally */
static void circular_kernel(const float *win, int n, double *h)
{
    double *cs = (double *)malloc(sizeof(double) * (size_t)n);
    for (int m = 0; m < n; m++) cs[m] = cos(2.0 * 3.141592653589793 * m / n);
    for (int m = 0; m < n; m++) {
        double a = 0.0;
        int idx = 0;
        for (int k = 0; k < n; k++) {
            a += (double)win[k <= n / 2 ? k : n - k] * cs[idx];
            idx += m;
            if (idx >= n) idx -= n;
        }
        h[m] = a / n;
    }
    free(cs);
}

void fwi_filter_operator(int filter, int n, float fpass, float fcut, float dt, float *C)
{
    float *win = (float *)malloc(sizeof(float) * (size_t)n);
    double *h = (double *)malloc(sizeof(double) * (size_t)n);
    fwi_filter_window(filter, n, fpass, fcut, dt, win);
    circular_kernel(win, n, h);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) C[(size_t)j * n + i] = (float)h[(i - j + n) % n];
    free(win);
    free(h);
}

/* ------------------------------------------------------------ FFT convolution spectra */
/* in-place radix-2 FFT of n = 2^k complex doubles (sign -1: forward, +1: inverse, unscaled) */
static void fft_pow2(double *re, double *im, int n, int sign)
{
    for (int i = 1, j = 0; i < n; i++) { /* bit reversal */
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const double ang = sign * 2.0 * 3.141592653589793 / len;
        for (int k = 0; k < len / 2; k++) {
            const double wr = cos(ang * k), wi = sin(ang * k);
            for (int i = k; i < n; i += len) {
                const int j = i + len / 2;
                const double xr = re[j] * wr - im[j] * wi, xi = re[j] * wi + im[j] * wr;
                re[j] = re[i] - xr; im[j] = im[i] - xi;
                re[i] += xr; im[i] += xi;
            }
        }
    }
}

int fwi_conv_size(int n)
{
    int M = 2;
    while (M < 2 * n - 1) M <<= 1;
    return M;
}

void fwi_conv_spectrum(const double *h, int n, int M, float *G)
{
    double *re = (double *)calloc((size_t)M, sizeof(double)), *im = (double *)calloc((size_t)M, sizeof(double));
    for (int m = 0; m < n; m++) re[m] = h[m];
    for (int m = 1; m < n; m++) re[M - m] = h[n - m];
    fft_pow2(re, im, M, -1);
    for (int k = 0; k < M; k++) {
        G[2 * k] = (float)(re[k] / M);
        G[2 * k + 1] = (float)(im[k] / M);
    }
    free(re);
    free(im);
}

void fwi_conv_spectrum_f64(const double *h, int n, int M, double *G)
{
    double *re = (double *)calloc((size_t)M, sizeof(double)), *im = (double *)calloc((size_t)M, sizeof(double));
    for (int m = 0; m < n; m++) re[m] = h[m];
    for (int m = 1; m < n; m++) re[M - m] = h[n - m];
    fft_pow2(re, im, M, -1);
    for (int k = 0; k < M; k++) {
        G[2 * k] = re[k] / M;
        G[2 * k + 1] = im[k] / M;
    }
    free(re);
    free(im);
}

void fwi_bluestein_tables(int N, int M, int f64, void *out)
{
    double *br = (double *)malloc(sizeof(double) * (size_t)N), *bi = (double *)malloc(sizeof(double) * (size_t)N);
    for (int m = 0; m < N; m++) {
        /* m^2 mod 2N keeps the angle small (the chirp has period 2N in m^2) */
        const long long q = ((long long)m * m) % (2LL * N);
        const double a = 3.141592653589793 * (double)q / N;
        br[m] = cos(a);
        bi[m] = sin(a);
    }
    double *re = (double *)calloc((size_t)M, sizeof(double)), *im = (double *)calloc((size_t)M, sizeof(double));
    double *spec = (double *)malloc(sizeof(double) * 4 * (size_t)M);
    for (int c = 0; c < 2; c++) {  /* c = 0: b, c = 1: conj(b) */
        memset(re, 0, sizeof(double) * (size_t)M);
        memset(im, 0, sizeof(double) * (size_t)M);
        const double sg = c ? -1.0 : 1.0;
        for (int m = 0; m < N; m++) {
            re[m] = br[m];
            im[m] = sg * bi[m];
            if (m > 0) {
                re[M - m] = br[m];
                im[M - m] = sg * bi[m];
            }
        }
        fft_pow2(re, im, M, -1);
        for (int k = 0; k < M; k++) {
            spec[(size_t)c * 2 * M + 2 * k] = re[k] / M;
            spec[(size_t)c * 2 * M + 2 * k + 1] = im[k] / M;
        }
    }
    const size_t n2 = 2 * (size_t)N;
    if (f64) {
        double *o = (double *)out;
        for (int m = 0; m < N; m++) o[2 * m] = br[m], o[2 * m + 1] = bi[m];
        memcpy(o + n2, spec, sizeof(double) * 4 * (size_t)M);
    } else {
        float *o = (float *)out;
        for (int m = 0; m < N; m++) o[2 * m] = (float)br[m], o[2 * m + 1] = (float)bi[m];
        for (size_t i = 0; i < 4 * (size_t)M; i++) o[n2 + i] = (float)spec[i];
    }
    free(br);
    free(bi);
    free(re);
    free(im);
    free(spec);
}

void fwi_fft_twiddles_f64(int M, double *tw)
{
    for (int k = 0; k < M / 2; k++) {
        const double a = 2.0 * 3.141592653589793 * k / M;
        tw[2 * k] = cos(a);
        tw[2 * k + 1] = -sin(a);
    }
}

void fwi_fft_twiddles(int M, float *tw)
{
    for (int k = 0; k < M / 2; k++) {
        const double a = 2.0 * 3.141592653589793 * k / M;
        tw[2 * k] = (float)cos(a);
        tw[2 * k + 1] = (float)-sin(a);
    }
}

void fwi_filter_kernel(int filter, int n, float fpass, float fcut, float dt, double *h)
{
    float *win = (float *)malloc(sizeof(float) * (size_t)n);
    fwi_filter_window(filter, n, fpass, fcut, dt, win);
    circular_kernel(win, n, h);
    free(win);
}

void fwi_interp_kernel(int ns, int r, double *g)
{
    const int N = (ns - 1) * r + 1, nkeep = N / (2 * r);
    float *win = (float *)calloc((size_t)N, sizeof(float));
    for (int k = 0; k < nkeep; k++) win[k] = (float)r;
    for (int k = N - nkeep + 1; k < N; k++) win[k] = (float)r;
    double *cs = (double *)malloc(sizeof(double) * (size_t)N);
    for (int m = 0; m < N; m++) cs[m] = cos(2.0 * 3.141592653589793 * m / N);
    for (int m = 0; m < N; m++) {
        double a = 0.0;
        int idx = 0;
        for (int k = 0; k < N; k++) {
            a += (double)win[k] * cs[idx];
            idx += m;
            if (idx >= N) idx -= N;
        }
        g[m] = a / N;
    }
    free(win);
    free(cs);
}

/* zero-stuffing by r, a rectangular window of height r on |k| < N / (2r) of the length-N
 * spectrum (N = (ns - 1) r + 1), inverse FFT, real part / N:  y[i] = sum_j x[j] g[(i - j r) mod N] */
void fwi_interp_operator(int ns, int r, int nt, float *M)
{
    const int N = (ns - 1) * r + 1, nkeep = N / (2 * r);
    float *win = (float *)calloc((size_t)N, sizeof(float));
    for (int k = 0; k < nkeep; k++) win[k] = (float)r;
    for (int k = N - nkeep + 1; k < N; k++) win[k] = (float)r;
    /* win is symmetric (win[k] = win[N - k]), so g is the cosine sum of the full window */
    double *g = (double *)malloc(sizeof(double) * (size_t)N), *cs = (double *)malloc(sizeof(double) * (size_t)N);
    for (int m = 0; m < N; m++) cs[m] = cos(2.0 * 3.141592653589793 * m / N);
    for (int m = 0; m < N; m++) {
        double a = 0.0;
        int idx = 0;
        for (int k = 0; k < N; k++) {
            a += (double)win[k] * cs[idx];
            idx += m;
            if (idx >= N) idx -= N;
        }
        g[m] = a / N;
    }
    for (int j = 0; j < ns; j++)
        for (int i = 0; i < nt; i++)
            M[(size_t)j * nt + i] = i < N ? (float)g[(((long long)i - (long long)j * r) % N + N) % N] : 0.0f;
    free(win);
    free(g);
    free(cs);
}

/* ------------------------------------------------------------ 2-D wavenumber filters */
/* generate_frequency (common.c:333-361): angular frequencies of an n-point FFT, float */
static void angular_frequency(float *f, float d, int n)
{
    const float df = 2.0f * (float)3.141592653589793 / (n * d);
    const int nf = n / 2 + 1;
    f[0] = 0.0f;
    for (int it = 1; it < nf; it++) {
        f[it] = it * df;
        if (n - it >= nf) f[n - it] = -f[it];
    }
}

void fwi_wavenumber_window(int filter, int Nx, int Nz, float dx, float dz, float kpass, float kcut, float *W)
{
    float *kx = (float *)malloc(sizeof(float) * (size_t)Nx), *kz = (float *)malloc(sizeof(float) * (size_t)Nz);
    angular_frequency(kx, dx, Nx);
    angular_frequency(kz, dz, Nz);
    const float pi = (float)3.141592653589793;
    for (int ix = 0; ix < Nx; ix++)
        for (int iz = 0; iz < Nz; iz++) {
            /* the reference evaluates iz <= Nz/2 and lets c2r mirror the rest; |KX|, |KZ| of the
             * mirrored entries are the same floats, so evaluating every entry is identical */
            const float KX = kx[ix] / (2.0f * pi), KZ = kz[iz] / (2.0f * pi);
            const float k = sqrtf(KX * KX + KZ * KZ);
            float w;
            if (filter == 0) {
                const float taperLen = kcut - kpass;
                if (k < kpass) w = 1.0f;
                else if (k >= kpass && k <= kcut) w = 0.5f * (1.0f + cosf(pi * (k - kpass) / taperLen));
                else w = 0.0f;
            } else {
                const float lo = kpass, hi = kcut - kpass;
                if (k < kpass) w = 0.5f * (1.0f + cosf(pi * (kpass - k) / lo));
                else if (k >= kpass && k <= kcut) w = 0.5f * (1.0f + cosf(pi * (k - kpass) / hi));
                else w = 0.0f;
            }
            W[(size_t)ix * Nz + iz] = w;
        }
    free(kx);
    free(kz);
}

