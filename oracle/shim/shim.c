/*
 * shim.c -- compatibility shim (TEST INFRASTRUCTURE ONLY).
 *
 * Implements, in this project's own code, the CWP/SU and FFTW3 entry points
 * that the FWI-EDU C sources call, so that those sources compile unmodified
 * into the oracle (oracle/_ref).  Semantics follow the public documentation of
 * both libraries; nothing here is shipped in the product library.
 */
#include <stdarg.h>
#include <stdint.h>
#include <complex.h>
#include "su.h"
#include "par.h"
#include "segy.h"
#include "fftw3.h"

/* ------------------------------------------------------------------ alloc */
void *alloc1(size_t n1, size_t size)
{
    void *p = malloc(n1 * size ? n1 * size : 1);
    return p;
}
void **alloc2(size_t n1, size_t n2, size_t size)
{
    void **p = (void **)malloc((n2 ? n2 : 1) * sizeof(void *));
    if (!p) return NULL;
    char *blk = (char *)malloc(n1 * n2 * size ? n1 * n2 * size : 1);
    if (!blk) { free(p); return NULL; }
    for (size_t i2 = 0; i2 < n2; i2++) p[i2] = blk + i2 * n1 * size;
    if (n2 == 0) p[0] = blk;
    return p;
}
void ***alloc3(size_t n1, size_t n2, size_t n3, size_t size)
{
    void ***p = (void ***)malloc((n3 ? n3 : 1) * sizeof(void **));
    if (!p) return NULL;
    void **rows = (void **)malloc((n2 * n3 ? n2 * n3 : 1) * sizeof(void *));
    char *blk = (char *)malloc(n1 * n2 * n3 * size ? n1 * n2 * n3 * size : 1);
    if (!rows || !blk) { free(p); free(rows); free(blk); return NULL; }
    for (size_t i3 = 0; i3 < n3; i3++) {
        p[i3] = rows + i3 * n2;
        for (size_t i2 = 0; i2 < n2; i2++) p[i3][i2] = blk + (i3 * n2 + i2) * n1 * size;
    }
    return p;
}
void free1(void *p) { free(p); }
void free2(void **p) { if (p) { free(p[0]); free(p); } }
void free3(void ***p) { if (p) { free(p[0][0]); free(p[0]); free(p); } }

float *alloc1float(size_t n1) { return (float *)alloc1(n1, sizeof(float)); }
float **alloc2float(size_t n1, size_t n2) { return (float **)alloc2(n1, n2, sizeof(float)); }
float ***alloc3float(size_t n1, size_t n2, size_t n3) { return (float ***)alloc3(n1, n2, n3, sizeof(float)); }
double *alloc1double(size_t n1) { return (double *)alloc1(n1, sizeof(double)); }
double **alloc2double(size_t n1, size_t n2) { return (double **)alloc2(n1, n2, sizeof(double)); }
int *alloc1int(size_t n1) { return (int *)alloc1(n1, sizeof(int)); }
int *ealloc1int(size_t n1)
{
    int *p = alloc1int(n1);
    if (!p) err("ealloc1int: out of memory");
    return p;
}
float *ealloc1float(size_t n1)
{
    float *p = alloc1float(n1);
    if (!p) err("ealloc1float: out of memory");
    return p;
}
void free1float(float *p) { free1(p); }
void free2float(float **p) { free2((void **)p); }
void free3float(float ***p) { free3((void ***)p); }
void free1double(double *p) { free1(p); }
void free2double(double **p) { free2((void **)p); }
void free1int(int *p) { free1(p); }

/* ------------------------------------------------------------ err / warn */
static void (*g_err_hook)(const char *msg) = NULL;
void fwi_shim_set_err_hook(void (*hook)(const char *msg)) { g_err_hook = hook; }

void err(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    fflush(stdout);
    fprintf(stderr, "%s\n", buf);
    if (g_err_hook) g_err_hook(buf);
    exit(1);
}
void warn(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fprintf(stderr, "\n");
}

FILE *efopen(const char *file, const char *mode)
{
    FILE *fp = fopen(file, mode);
    if (!fp) err("efopen: cannot open %s", file);
    return fp;
}
int efclose(FILE *stream)
{
    int r = fclose(stream);
    if (r) err("efclose: fclose failed");
    return r;
}

float sasum(int n, float *sx, int incx)
{
    float s = 0.0f;
    for (int i = 0; i < n; i++) s += fabsf(sx[i * incx]);
    return s;
}
int CWP_Exit(void) { return 0; }

/* ---------------------------------------------------------------- getpar */
int xargc = 0;
char **xargv = NULL;
extern char *sdoc[] __attribute__((weak));

void initargs(int argc, char **argv)
{
    xargc = argc;
    xargv = argv;
}
void requestdoc(int flag)
{
    if (flag == 0 && xargc <= 1 && sdoc) {
        for (int i = 0; sdoc[i]; i++) fprintf(stderr, "%s\n", sdoc[i]);
        exit(1);
    }
}
/* the last "name=value" on the command line wins */
static const char *find_par(const char *name)
{
    size_t ln = strlen(name);
    for (int i = xargc - 1; i >= 1; i--) {
        const char *a = xargv[i];
        if (strncmp(a, name, ln) == 0 && a[ln] == '=') return a + ln + 1;
    }
    return NULL;
}
int countparval(const char *name)
{
    const char *v = find_par(name);
    if (!v) return 0;
    int n = 1;
    for (const char *c = v; *c; c++)
        if (*c == ',') n++;
    return n;
}
int getparint(const char *name, int *p)
{
    const char *v = find_par(name);
    if (!v) return 0;
    int n = 0;
    const char *c = v;
    while (1) {
        p[n++] = (int)strtol(c, NULL, 10);
        c = strchr(c, ',');
        if (!c) break;
        c++;
    }
    return n;
}
int getparfloat(const char *name, float *p)
{
    const char *v = find_par(name);
    if (!v) return 0;
    int n = 0;
    const char *c = v;
    while (1) {
        p[n++] = (float)strtod(c, NULL);
        c = strchr(c, ',');
        if (!c) break;
        c++;
    }
    return n;
}
int getpardouble(const char *name, double *p)
{
    const char *v = find_par(name);
    if (!v) return 0;
    int n = 0;
    const char *c = v;
    while (1) {
        p[n++] = strtod(c, NULL);
        c = strchr(c, ',');
        if (!c) break;
        c++;
    }
    return n;
}
int getparstring(const char *name, char **p)
{
    const char *v = find_par(name);
    if (!v) return 0;
    *p = (char *)v;
    return 1;
}

/* ------------------------------------------------------------- SU traces */
void fputtr(FILE *fp, segy *tp)
{
    if (fwrite(tp, 1, HDRBYTES, fp) != HDRBYTES) err("fputtr: header write failed");
    size_t ns = tp->ns;
    if (fwrite(tp->data, sizeof(float), ns, fp) != ns) err("fputtr: data write failed");
}
int fgettr(FILE *fp, segy *tp)
{
    size_t r = fread(tp, 1, HDRBYTES, fp);
    if (r == 0) return 0;
    if (r != HDRBYTES) err("fgettr: short header");
    size_t ns = tp->ns;
    if (fread(tp->data, sizeof(float), ns, fp) != ns) err("fgettr: short trace");
    return (int)ns;
}
int fvgettr(FILE *fp, segy *tp) { return fgettr(fp, tp); }

/* ------------------------------------------------------------------- FFT */
/* The transforms work in double precision and round to float at the plan's arrays.  Built with
 * -DSHIM_FFT_FLOAT they work in float instead, as a single-precision FFT library does: the
 * oracle uses that build to measure how much the reference's results depend on the rounding
 * of the FFT library it is linked with. */
#ifdef SHIM_FFT_FLOAT
typedef float complex fftc_t;
#else
typedef double complex fftc_t;
#endif

/* in-place complex FFT of length n; sign -1 forward, +1 backward */
static void fft_pow2(fftc_t *a, int n, int sign)
{
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { fftc_t t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (int len = 2; len <= n; len <<= 1) {
        double ang = sign * 2.0 * PI / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < len / 2; k++) {
                fftc_t w = cos(ang * k) + I * sin(ang * k);
                fftc_t u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
        }
    }
}
static void fft_any(fftc_t *a, int n, int sign)
{
    if (n <= 1) return;
    if ((n & (n - 1)) == 0) { fft_pow2(a, n, sign); return; }
    /* Bluestein: chirp-z transform through a power-of-two convolution */
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    fftc_t *w = malloc(sizeof(fftc_t) * n);
    fftc_t *A = calloc(m, sizeof(fftc_t));
    fftc_t *B = calloc(m, sizeof(fftc_t));
    for (int k = 0; k < n; k++) {
        /* k*k mod 2n keeps the chirp argument small */
        long long kk = ((long long)k * k) % (2LL * n);
        double ang = sign * PI * (double)kk / n;
        w[k] = cos(ang) + I * sin(ang);
    }
    for (int k = 0; k < n; k++) A[k] = a[k] * w[k];
    B[0] = conj(w[0]);
    for (int k = 1; k < n; k++) B[k] = B[m - k] = conj(w[k]);
    fft_pow2(A, m, -1);
    fft_pow2(B, m, -1);
    for (int i = 0; i < m; i++) A[i] *= B[i];
    fft_pow2(A, m, +1);
    for (int k = 0; k < n; k++) a[k] = A[k] / m * w[k];
    free(w); free(A); free(B);
}

enum { K_C2C = 0, K_R2C = 1, K_C2R = 2, K_R2C_2D = 3, K_C2R_2D = 4 };
struct fwi_shim_fftwf_plan_s {
    int kind, n0, n1, sign;
    void *in, *out;
};

void *fftwf_malloc(size_t n) { return malloc(n ? n : 1); }
void fftwf_free(void *p) { free(p); }
static fftwf_plan mkplan(int kind, int n0, int n1, int sign, void *in, void *out)
{
    fftwf_plan p = (fftwf_plan)malloc(sizeof(*p));
    p->kind = kind; p->n0 = n0; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
    return p;
}
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags)
{ (void)flags; return mkplan(K_C2C, n, 1, sign, in, out); }
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags)
{ (void)flags; return mkplan(K_R2C, n, 1, -1, in, out); }
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags)
{ (void)flags; return mkplan(K_C2R, n, 1, +1, in, out); }
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned flags)
{ (void)flags; return mkplan(K_R2C_2D, n0, n1, -1, in, out); }
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned flags)
{ (void)flags; return mkplan(K_C2R_2D, n0, n1, +1, in, out); }
void fftwf_destroy_plan(fftwf_plan p) { free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int n) { (void)n; }
void fftwf_cleanup_threads(void) {}

/* full 2-D complex transform (row-major n0 x n1) */
static void fft2(fftc_t *a, int n0, int n1, int sign)
{
    fftc_t *col = malloc(sizeof(fftc_t) * n0);
    for (int i = 0; i < n0; i++) fft_any(a + (size_t)i * n1, n1, sign);
    for (int j = 0; j < n1; j++) {
        for (int i = 0; i < n0; i++) col[i] = a[(size_t)i * n1 + j];
        fft_any(col, n0, sign);
        for (int i = 0; i < n0; i++) a[(size_t)i * n1 + j] = col[i];
    }
    free(col);
}

void fftwf_execute(const fftwf_plan p)
{
    int n = p->n0;
    if (p->kind == K_C2C) {
        float (*in)[2] = p->in, (*out)[2] = p->out;
        fftc_t *a = malloc(sizeof(fftc_t) * (n ? n : 1));
        for (int i = 0; i < n; i++) a[i] = in[i][0] + I * in[i][1];
        fft_any(a, n, p->sign);
        for (int i = 0; i < n; i++) { out[i][0] = (float)creal(a[i]); out[i][1] = (float)cimag(a[i]); }
        free(a);
    } else if (p->kind == K_R2C) {
        float *in = p->in;
        float (*out)[2] = p->out;
        fftc_t *a = malloc(sizeof(fftc_t) * (n ? n : 1));
        for (int i = 0; i < n; i++) a[i] = in[i];
        fft_any(a, n, -1);
        for (int i = 0; i <= n / 2; i++) { out[i][0] = (float)creal(a[i]); out[i][1] = (float)cimag(a[i]); }
        free(a);
    } else if (p->kind == K_C2R) {
        float (*in)[2] = p->in;
        float *out = p->out;
        fftc_t *a = malloc(sizeof(fftc_t) * (n ? n : 1));
        for (int i = 0; i <= n / 2; i++) a[i] = in[i][0] + I * in[i][1];
        a[0] = creal(a[0]);
        if (n % 2 == 0) a[n / 2] = creal(a[n / 2]);
        for (int i = n / 2 + 1; i < n; i++) a[i] = conj(a[n - i]);
        fft_any(a, n, +1);
        for (int i = 0; i < n; i++) out[i] = (float)creal(a[i]);
        free(a);
    } else if (p->kind == K_R2C_2D) {
        int n0 = p->n0, n1 = p->n1, h = n1 / 2 + 1;
        float *in = p->in;
        float (*out)[2] = p->out;
        fftc_t *a = malloc(sizeof(fftc_t) * (size_t)n0 * n1);
        for (size_t i = 0; i < (size_t)n0 * n1; i++) a[i] = in[i];
        fft2(a, n0, n1, -1);
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < h; j++) {
                out[(size_t)i * h + j][0] = (float)creal(a[(size_t)i * n1 + j]);
                out[(size_t)i * h + j][1] = (float)cimag(a[(size_t)i * n1 + j]);
            }
        free(a);
    } else if (p->kind == K_C2R_2D) {
        int n0 = p->n0, n1 = p->n1, h = n1 / 2 + 1;
        float (*in)[2] = p->in;
        float *out = p->out;
        fftc_t *a = malloc(sizeof(fftc_t) * (size_t)n0 * n1);
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < h; j++)
                a[(size_t)i * n1 + j] = in[(size_t)i * h + j][0] + I * in[(size_t)i * h + j][1];
        /* Hermitian completion: X[i][j] = conj(X[(n0-i)%n0][n1-j]) */
        for (int i = 0; i < n0; i++)
            for (int j = h; j < n1; j++)
                a[(size_t)i * n1 + j] = conj(a[(size_t)((n0 - i) % n0) * n1 + (n1 - j)]);
        fft2(a, n0, n1, +1);
        for (size_t i = 0; i < (size_t)n0 * n1; i++) out[i] = (float)creal(a[i]);
        free(a);
    }
}
