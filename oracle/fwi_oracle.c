/*
 * fwi_oracle.c -- CPU restatement of the FWI-EDU 2-D acoustic engine.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg call it; the product library never links it.
 *
 * Every function below restates one piece of the reference C implementation
 * (FWILab2dCLangV1.2.6, cited by file:line) in this project's own code.  With
 * ORACLE_REAL=float it keeps the reference's exact expression order and its
 * float/double promotions, so a strict IEEE build (-O2 -fno-fast-math
 * -ffp-contract=off) reproduces the reference bit for bit; the tests pin that
 * against vectors produced by the reference itself (tests/golden).  With
 * ORACLE_REAL=double every quantity is carried in double: the FP64 build of the
 * same algorithm that the precision statements are measured against.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <stdio.h>
#include "fwi_oracle.h"

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;

#define ORC_IS_DOUBLE_double 1
#define ORC_CAT(a, b) a##b
#define ORC_XCAT(a, b) ORC_CAT(a, b)
#if ORC_XCAT(ORC_IS_DOUBLE_, ORACLE_REAL)
#define ORC_F64 1
#define RSQRT sqrt
#define REXP exp
#define RLOG log
#define RPOW pow
#define RLOG10 log10
#define RCOS cos
#define RROUND round
#else
#define ORC_F64 0
#define RSQRT sqrtf
#define REXP expf
#define RLOG logf
#define RPOW powf
#define RLOG10 log10f
#define RCOS cosf
#define RROUND roundf
#endif

#define ORC_PI (3.141592653589793)
#define MST 5 /* imaging / pseudo-Hessian interval, propagation.h:21 */
#define IDX(ix, iz, n1) ((size_t)(ix) * (size_t)(n1) + (size_t)(iz))

int orc_real_size(void) { return (int)sizeof(real); }

/* ------------------------------------------------------------------ setup */

/* pad_model2d, common.c:110-176: centre copy then edge replication top, bottom, left, right */
static void pad_model(const float *mod, int nz, int nx, real *modp, int nl)
{
    int Nz = nz + 2 * nl, Nx = nx + 2 * nl;
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) modp[IDX(ix + nl, iz + nl, Nz)] = (real)mod[IDX(ix, iz, nz)];
    for (int ix = 0; ix < Nx; ix++)
        for (int iz = 0; iz < nl; iz++) modp[IDX(ix, iz, Nz)] = modp[IDX(ix, nl, Nz)];
    for (int ix = 0; ix < Nx; ix++)
        for (int iz = nz + nl; iz < Nz; iz++) modp[IDX(ix, iz, Nz)] = modp[IDX(ix, nz + nl - 1, Nz)];
    for (int ix = 0; ix < nl; ix++)
        for (int iz = 0; iz < Nz; iz++) modp[IDX(ix, iz, Nz)] = modp[IDX(nl, iz, Nz)];
    for (int ix = nx + nl; ix < Nx; ix++)
        for (int iz = 0; iz < Nz; iz++) modp[IDX(ix, iz, Nz)] = modp[IDX(nx + nl - 1, iz, Nz)];
}

/* absorbWeight, propagation.c:173-190 */
static real absorb_weight(real alpha, int l, int nlayer)
{
    real d = ((real)0.1 * l) / ((real)0.1 * nlayer);
    return REXP(RLOG((real)2.0) * RPOW(d, alpha)) - (real)1.0;
}

/* mealCoefs2d, propagation.c:192-354 (vs == NULL branch, as the engine calls it at :511) */
static void meal_coefs(real *D, real *Beta, const real *vp, real fpeak, real alpha,
                       real dz, real dx, int NZ, int NX, int nlayer)
{
    size_t n = (size_t)NZ * NX;
    real pd = 2;
    real Rcoef = RPOW((real)10.0, (real)-1.0 * ((RLOG10((real)nlayer) - (real)1.0) / (RLOG10((real)2.0))) -
                                      (real)3.0 - (real)0.5 * pd);
    real PPWfd = (real)10.0;
    real thicknessx = nlayer * dx, thicknessz = nlayer * dz;
    real *Vs = malloc(n * sizeof(real)), *Dx = malloc(n * sizeof(real)), *Dz = malloc(n * sizeof(real));
    real *Bx = malloc(n * sizeof(real)), *Bz = malloc(n * sizeof(real));
    if (alpha == (real)-1.0) alpha = (real)2.5;
    for (size_t i = 0; i < n; i++) Vs[i] = vp[i] / RSQRT((real)3.0);
    for (size_t i = 0; i < n; i++) {
        D[i] = 0; Dx[i] = 0; Dz[i] = 0;
        Beta[i] = 1; Bx[i] = 1; Bz[i] = 1;
    }
    for (int ix = 0; ix < NX; ix++) {
        for (int l = 1; l <= nlayer; l++) {
            real weight = absorb_weight(alpha, l, nlayer);
            int iz = nlayer - l; /* top */
            real d0z = (real)-1.0 * ((real)1.0 + pd) * vp[IDX(ix, iz, NZ)] * RLOG(Rcoef) / ((real)2.0 * thicknessz);
            real PPWfcs = Vs[IDX(ix, iz, NZ)] / (dz * fpeak);
            real betaz = (real)2.0 * PPWfcs / PPWfd;
            Dz[IDX(ix, iz, NZ)] = d0z * weight;
            Bz[IDX(ix, iz, NZ)] = (real)1.0 + (betaz - (real)1.0) * weight;
            iz = NZ - nlayer - 1 + l; /* bottom */
            d0z = (real)-1.0 * ((real)1.0 + pd) * vp[IDX(ix, iz, NZ)] * RLOG(Rcoef) / ((real)2.0 * thicknessz);
            PPWfcs = Vs[IDX(ix, iz, NZ)] / (dz * fpeak);
            betaz = (real)2.0 * PPWfcs / PPWfd;
            Dz[IDX(ix, iz, NZ)] = d0z * weight;
            Bz[IDX(ix, iz, NZ)] = (real)1.0 + (betaz - (real)1.0) * weight;
        }
    }
    for (int l = 1; l <= nlayer; l++) {
        real weight = absorb_weight(alpha, l, nlayer);
        for (int iz = 0; iz < NZ; iz++) {
            int ix = nlayer - l; /* left */
            real d0x = (real)-1.0 * ((real)1.0 + pd) * vp[IDX(ix, iz, NZ)] * RLOG(Rcoef) / ((real)2.0 * thicknessx);
            real PPWfcs = Vs[IDX(ix, iz, NZ)] / (dx * fpeak);
            real betax = (real)2.0 * PPWfcs / PPWfd;
            Dx[IDX(ix, iz, NZ)] = d0x * weight;
            Bx[IDX(ix, iz, NZ)] = (real)1.0 + (betax - (real)1.0) * weight;
            ix = NX - nlayer - 1 + l; /* right */
            d0x = (real)-1.0 * ((real)1.0 + pd) * vp[IDX(ix, iz, NZ)] * RLOG(Rcoef) / ((real)2.0 * thicknessx);
            PPWfcs = Vs[IDX(ix, iz, NZ)] / (dx * fpeak);
            betax = (real)2.0 * PPWfcs / PPWfd;
            Dx[IDX(ix, iz, NZ)] = d0x * weight;
            Bx[IDX(ix, iz, NZ)] = (real)1.0 + (betax - (real)1.0) * weight;
        }
    }
    for (size_t i = 0; i < n; i++) {
        D[i] = RSQRT(RPOW(Dx[i], (real)2.0) + RPOW(Dz[i], (real)2.0));
        Beta[i] = RSQRT(RPOW(Bx[i] - (real)1.0, (real)2.0) + RPOW(Bz[i] - (real)1.0, (real)2.0)) + (real)1.0;
    }
    free(Vs); free(Dx); free(Dz); free(Bx); free(Bz);
}

/* calculate_gradient2d, common.c:416-479 (one-sided at the edges, central inside) */
static void gradient2d(const real *f, int nx, int nz, real dx, real dz, real *dfdx, real *dfdz)
{
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            if (ix == 0) dfdx[IDX(ix, iz, nz)] = (f[IDX(ix + 1, iz, nz)] - f[IDX(ix, iz, nz)]) / dx;
            else if (ix == nx - 1) dfdx[IDX(ix, iz, nz)] = (f[IDX(ix, iz, nz)] - f[IDX(ix - 1, iz, nz)]) / dx;
            else dfdx[IDX(ix, iz, nz)] = (f[IDX(ix + 1, iz, nz)] - f[IDX(ix - 1, iz, nz)]) / ((real)2.0 * dx);
        }
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            if (iz == 0) dfdz[IDX(ix, iz, nz)] = (f[IDX(ix, iz + 1, nz)] - f[IDX(ix, iz, nz)]) / dz;
            else if (iz == nz - 1) dfdz[IDX(ix, iz, nz)] = (f[IDX(ix, iz, nz)] - f[IDX(ix, iz - 1, nz)]) / dz;
            else dfdz[IDX(ix, iz, nz)] = (f[IDX(ix, iz + 1, nz)] - f[IDX(ix, iz - 1, nz)]) / ((real)2.0 * dz);
        }
}

/* acoustic_iso2d_rgfd_parameter, propagation.c:103-171 */
static void rgfd_parameter(const real *vp, const real *rho, int nx, int nz, real dx, real dz,
                           real *K, real *invrho, real *invrhox, real *invrhoz)
{
    const real C1 = (real)0.91067892f, C2 = (real)-0.34187892f, C3 = (real)0.13833962f;
    const real C4 = (real)-0.04880710f, C5 = (real)0.01302148f, C6 = (real)-0.00199047f;
    real invdx = (real)1.0 / dx, invdz = (real)1.0 / dz;
    for (size_t i = 0; i < (size_t)nx * nz; i++) {
        K[i] = rho[i] * vp[i] * vp[i];
        invrho[i] = (real)1.0 / rho[i];
    }
    gradient2d(invrho, nx, nz, dx, dz, invrhox, invrhoz);
#define IR(a, b) invrho[IDX(a, b, nz)]
    for (int ix = 6; ix < nx - 6; ix++)
        for (int iz = 6; iz < nz - 6; iz++) {
            invrhox[IDX(ix, iz, nz)] = (C1 * (IR(ix + 1, iz) - IR(ix - 1, iz)) + C2 * (IR(ix + 2, iz) - IR(ix - 2, iz)) +
                                        C3 * (IR(ix + 3, iz) - IR(ix - 3, iz)) + C4 * (IR(ix + 4, iz) - IR(ix - 4, iz)) +
                                        C5 * (IR(ix + 5, iz) - IR(ix - 5, iz)) + C6 * (IR(ix + 6, iz) - IR(ix - 6, iz))) *
                                       invdx;
            invrhoz[IDX(ix, iz, nz)] = (C1 * (IR(ix, iz + 1) - IR(ix, iz - 1)) + C2 * (IR(ix, iz + 2) - IR(ix, iz - 2)) +
                                        C3 * (IR(ix, iz + 3) - IR(ix, iz - 3)) + C4 * (IR(ix, iz + 4) - IR(ix, iz - 4)) +
                                        C5 * (IR(ix, iz + 5) - IR(ix, iz - 5)) + C6 * (IR(ix, iz + 6) - IR(ix, iz - 6))) *
                                       invdz;
        }
#undef IR
}

typedef struct {
    int nz, nxx, Nz, Nx, pml, fs;
    int ixStart, ixEnd, izStart, izEnd;
    float dt; /* the caller's float step, promoted where the reference promotes it */
    real invdx, invdz, invdxdx, invdzdz, invdtdt;
    real *coef1, *coef2, *coef3, *K, *invrho, *invrhox, *invrhoz;
} Grid;

/* engine set-up, propagation.c:443-537: pad, MEAL, D/Beta folding, coef1..3 in double, rgfd */
static void grid_build(Grid *g, const float *vpm, const float *rhom, int nz, int nxx, int pml,
                       float dx, float dz, float dt, float fpeak, int fs)
{
    g->nz = nz; g->nxx = nxx; g->pml = pml; g->fs = fs;
    g->Nz = nz + 2 * pml; g->Nx = nxx + 2 * pml;
    g->dt = dt;
    g->invdx = (real)1.0 / (real)dx;
    g->invdz = (real)1.0 / (real)dz;
    g->invdxdx = (real)1.0 / ((real)dx * (real)dx);
    g->invdzdz = (real)1.0 / ((real)dz * (real)dz);
    g->invdtdt = (real)1.0 / ((real)dt * (real)dt);
    size_t n = (size_t)g->Nz * g->Nx;
    real *vp = malloc(n * sizeof(real)), *rho = malloc(n * sizeof(real));
    real *D = malloc(n * sizeof(real)), *Beta = malloc(n * sizeof(real));
    g->coef1 = malloc(n * sizeof(real)); g->coef2 = malloc(n * sizeof(real)); g->coef3 = malloc(n * sizeof(real));
    g->K = malloc(n * sizeof(real)); g->invrho = malloc(n * sizeof(real));
    g->invrhox = malloc(n * sizeof(real)); g->invrhoz = malloc(n * sizeof(real));
    pad_model(vpm, nz, nxx, vp, pml);
    pad_model(rhom, nz, nxx, rho, pml);
    meal_coefs(D, Beta, vp, (real)fpeak, (real)2.5, (real)dz, (real)dx, g->Nz, g->Nx, pml);
    for (size_t i = 0; i < n; i++) {
        D[i] /= Beta[i];
        vp[i] /= Beta[i];
        rho[i] *= Beta[i];
        /* "dt * dt * D * D" is a float product in the reference, the rest is double */
        real rdt = (real)dt;
        g->coef1[i] = (real)((2.0 - rdt * rdt * D[i] * D[i]) / (1.0 + rdt * D[i]));
        g->coef2[i] = (real)(-1.0 * (1.0 - rdt * D[i]) / (1.0 + rdt * D[i]));
        g->coef3[i] = (real)((rdt * rdt) / (1.0 + rdt * D[i]));
    }
    rgfd_parameter(vp, rho, g->Nx, g->Nz, (real)dx, (real)dz, g->K, g->invrho, g->invrhox, g->invrhoz);
    free(vp); free(rho); free(D); free(Beta);
    g->ixStart = 3;
    g->ixEnd = g->Nx - 3 - 1;
    g->izStart = (fs == 0) ? 3 : pml;
    g->izEnd = g->Nz - 3 - 1;
}

static void grid_free(Grid *g)
{
    free(g->coef1); free(g->coef2); free(g->coef3); free(g->K);
    free(g->invrho); free(g->invrhox); free(g->invrhoz);
}

void orc_setup(const float *vpm, const float *rhom, int nz, int nx, int pml,
               float dx, float dz, float dt, float fpeak,
               void *coef1, void *coef2, void *coef3, void *K,
               void *invrho, void *invrhox, void *invrhoz)
{
    Grid g;
    grid_build(&g, vpm, rhom, nz, nx, pml, dx, dz, dt, fpeak, 0);
    size_t n = (size_t)g.Nz * g.Nx * sizeof(real);
    memcpy(coef1, g.coef1, n); memcpy(coef2, g.coef2, n); memcpy(coef3, g.coef3, n);
    memcpy(K, g.K, n); memcpy(invrho, g.invrho, n); memcpy(invrhox, g.invrhox, n); memcpy(invrhoz, g.invrhoz, n);
    grid_free(&g);
}

/* ---------------------------------------------------------------- stepping */

/* acoustic_iso2d_fd_it_6order, propagation.c:13-74 */
static void fd_step(real *restrict p2, const real *restrict p1, const real *restrict p0, const Grid *g)
{
    const real C1 = (real)0.77793115f, C2 = (real)-0.17388691f, C3 = (real)0.02338713f;
    const real D0 = (real)-2.8215452f, D1 = (real)1.57663238f, D2 = (real)-0.18347238f, D3 = (real)0.01761260f;
    const int Nz = g->Nz;
    const real invdx = g->invdx, invdz = g->invdz, invdxdx = g->invdxdx, invdzdz = g->invdzdz;
#pragma omp parallel for schedule(static)
    for (int ix = g->ixStart; ix <= g->ixEnd; ++ix) {
        const real *c = p1 + (size_t)ix * Nz;
        const real *xm1 = c - Nz, *xm2 = c - 2 * Nz, *xm3 = c - 3 * Nz;
        const real *xp1 = c + Nz, *xp2 = c + 2 * Nz, *xp3 = c + 3 * Nz;
        for (int iz = g->izStart; iz <= g->izEnd; ++iz) {
            real dpdz = (C1 * (c[iz + 1] - c[iz - 1]) + C2 * (c[iz + 2] - c[iz - 2]) + C3 * (c[iz + 3] - c[iz - 3])) * invdz;
            real dpdx = (C1 * (xp1[iz] - xm1[iz]) + C2 * (xp2[iz] - xm2[iz]) + C3 * (xp3[iz] - xm3[iz])) * invdx;
            real dzz = (D0 * c[iz] + D1 * (c[iz + 1] + c[iz - 1]) + D2 * (c[iz + 2] + c[iz - 2]) + D3 * (c[iz + 3] + c[iz - 3])) * invdzdz;
            real dxx = (D0 * c[iz] + D1 * (xp1[iz] + xm1[iz]) + D2 * (xp2[iz] + xm2[iz]) + D3 * (xp3[iz] + xm3[iz])) * invdxdx;
            size_t i = (size_t)ix * Nz + iz;
            p2[i] = g->coef1[i] * c[iz] + g->coef2[i] * p0[i] +
                    g->coef3[i] * g->K[i] * (g->invrhox[i] * dpdx + g->invrhoz[i] * dpdz + g->invrho[i] * (dxx + dzz));
        }
    }
}

/* acoustic_iso2d_freesurface, propagation.c:76-101 */
static void free_surface(real *p2, const Grid *g)
{
    const int Nz = g->Nz, pml = g->pml;
    for (int ix = 0; ix < g->Nx; ix++) {
        real *c = p2 + (size_t)ix * Nz;
        c[pml] = (real)0.0;
        for (int iz = 0; iz <= pml; iz++) c[pml - iz] = -c[pml + iz];
    }
}

/* ------------------------------------------------------------- checkpoints */

/* dCheckPoint = MAX(roundf(sqrtf(2(nt-1))), 3), checkpoint.c:47 */
int orc_checkpoint_interval(int nt)
{
    float r = roundf(sqrtf(2.0f * (nt - 1)));
    return (int)(r > 3 ? r : 3);
}
int orc_checkpoint_count(int nt)
{
    int d = orc_checkpoint_interval(nt), n = 0;
    for (int it = 0; it < nt; it++)
        if (it % d == 0 || (it + 1) % d == 0) n++;
    return n;
}

/* The forward pass stores the pair (u(it-1), u(it)) at every it % d == 0
 * (save_acoustic2dCheckPoint, checkpoint.c:130-159).  During the adjoint pass a
 * step that is not stored is rebuilt once per segment from the checkpoint below
 * it (get_acoustic2dCheckPointStatus walk-back, checkpoint.c:236-265, and the
 * replay loop at propagation.c:641-673).  Frames are kept per time index. */
typedef struct {
    int nt, d;
    size_t frame;
    int *slot;      /* nt: slot of a stored step, or -1 */
    real *store;    /* stored frames */
    real *seg;      /* replayed frames of the current segment, d frames */
    int seg_c;      /* checkpoint the current segment was replayed from, -1 if none */
} Ckpt;

static int ck_is_stored(int t, int nt, int d) { return t % d == 0 || ((t + 1) % d == 0 && t + 1 < nt); }

/* Precision study of the checkpoint snapshots: 0 keeps them in the oracle's precision; 1 stores
 * each snapshot as FP16 with its own max-abs scale (the largest magnitude maps to 2^15); 2 as
 * BF16 (round to nearest even on the top 16 bits of the FP32 pattern).  The replay starts from,
 * and the imaging reads, the values as they come back. */
static int g_ck_precision = 0;
void orc_set_checkpoint_precision(int mode) { g_ck_precision = mode; }

static float bf16_round(float v)
{
    uint32_t b;
    memcpy(&b, &v, 4);
    b = (b + 0x7fffu + ((b >> 16) & 1u)) & 0xffff0000u;
    memcpy(&v, &b, 4);
    return v;
}

static void quantize_snapshot(real *u, size_t n)
{
    if (g_ck_precision == 0) return;
    double amax = 0.0;
    for (size_t i = 0; i < n; i++) amax = fmax(amax, fabs((double)u[i]));
    if (amax == 0.0) return;
    if (g_ck_precision == 1) {
        const double to = 32768.0 / amax, back = amax / 32768.0;
        for (size_t i = 0; i < n; i++) u[i] = (real)((double)(_Float16)((double)u[i] * to) * back);
    } else {
        for (size_t i = 0; i < n; i++) u[i] = (real)bf16_round((float)u[i]);
    }
}

static void ck_alloc(Ckpt *ck, int nt, size_t frame)
{
    ck->nt = nt;
    ck->d = orc_checkpoint_interval(nt);
    ck->frame = frame;
    ck->slot = malloc(sizeof(int) * nt);
    int ns = 0;
    for (int t = 0; t < nt; t++) ck->slot[t] = ck_is_stored(t, nt, ck->d) ? ns++ : -1;
    ck->store = calloc((size_t)(ns ? ns : 1) * frame, sizeof(real));
    ck->seg = calloc((size_t)ck->d * frame, sizeof(real));
    ck->seg_c = -1;
}
static void ck_free(Ckpt *ck) { free(ck->slot); free(ck->store); free(ck->seg); }

/* ------------------------------------------------------------------ engine */

static size_t frame_bytes(const Grid *g) { return (size_t)g->Nz * g->Nx * sizeof(real); }

/* forward time loop of iso_acoustic2d_propagation_engine, modes 0 and 1
 * (propagation.c:539-623).  traces: ntr*ns in the oracle precision.
 * H: nz*nxx double pseudo-Hessian (mode 1 with precondition), finalised. */
static void engine_forward(const Grid *g, const OrcShot *s, int nt, int mode, int precondition,
                           const real *vpm_w, const real *rhom_w, real *traces, Ckpt *ck, double *H)
{
    const int Nz = g->Nz, pml = g->pml;
    size_t n = (size_t)g->Nz * g->Nx;
    real *p0 = calloc(n, sizeof(real)), *p1 = calloc(n, sizeof(real)), *p2 = calloc(n, sizeof(real));
    const int isx = s->isx + pml, isz = s->isz + pml;
    const size_t is = IDX(isx, isz, Nz);
    const float dt = g->dt;
    if (H) memset(H, 0, sizeof(double) * g->nz * g->nxx);
    for (int it = 0; it < nt; ++it) {
        if (mode == 1 && it % ck->d == 0) {
            if (it - 1 >= 0) {
                memcpy(ck->store + (size_t)ck->slot[it - 1] * n, p0, frame_bytes(g));
                quantize_snapshot(ck->store + (size_t)ck->slot[it - 1] * n, n);
            }
            memcpy(ck->store + (size_t)ck->slot[it] * n, p1, frame_bytes(g));
            quantize_snapshot(ck->store + (size_t)ck->slot[it] * n, n);
        }
        fd_step(p2, p1, p0, g);
        /* source: the product is formed in double (the literal 1.0), propagation.c:558 */
        p2[is] = (real)((double)p2[is] + 1.0 * s->src[it] * g->K[is] * dt * dt * g->invdx * g->invdz);
        if (g->fs == 1) free_surface(p2, g);
        if (it % s->sampleRate == 0) {
            int k = it / s->sampleRate;
            for (int itr = 0; itr < s->ntr; ++itr)
                traces[(size_t)itr * s->ns + k] = p1[IDX(s->igx[itr] + pml, s->igz[itr] + pml, Nz)];
        }
        if (mode == 1 && it % MST == 0 && precondition == 1) {
#pragma omp parallel for schedule(static)
            for (int ix = pml; ix < pml + g->nxx; ix++)
                for (int iz = pml; iz < pml + g->nz; iz++) {
                    size_t i = IDX(ix, iz, Nz);
                    real t = (p2[i] - (real)2.0 * p1[i] + p0[i]) * g->invdtdt;
                    H[IDX(ix - pml, iz - pml, g->nz)] += (double)(t * t);
                }
        }
        real *tmp = p0; p0 = p1; p1 = p2; p2 = tmp;
    }
    if (mode == 1 && precondition == 1) {
        /* propagation.c:610-623: 4 H / (rho v)^2 with the unpadded model; (rho v)^2 in float */
        for (size_t i = 0; i < (size_t)g->nz * g->nxx; i++) {
            real rv = rhom_w[i] * vpm_w[i];
            H[i] = 4.0 * H[i] / ((double)(rv * rv));
        }
    }
    free(p0); free(p1); free(p2);
}

/* adjoint time loop, engine mode 2 (propagation.c:633-744).  adj: ntr*nt (already
 * interpolated to the engine step).  G: nz*nxx double, finalised 2 G / (rho v). */
static void engine_adjoint(const Grid *g, const OrcShot *s, int nt, const real *adj,
                           const real *vpm_w, const real *rhom_w, Ckpt *ck, double *G)
{
    const int Nz = g->Nz, pml = g->pml;
    size_t n = (size_t)g->Nz * g->Nx;
    real *p0 = calloc(n, sizeof(real)), *p1 = calloc(n, sizeof(real)), *p2 = calloc(n, sizeof(real));
    real *f0 = calloc(n, sizeof(real)), *f1 = calloc(n, sizeof(real)), *f2 = calloc(n, sizeof(real));
    const size_t is = IDX(s->isx + pml, s->isz + pml, Nz);
    const float dt = g->dt;
    const real rdt = (real)dt;
    memset(G, 0, sizeof(double) * g->nz * g->nxx);
    ck->seg_c = -1;
    for (int it = nt - 1; it >= 0; --it) {
        const real *u;
        if (ck->slot[it] >= 0) {
            u = ck->store + (size_t)ck->slot[it] * n;
        } else {
            int c = (it / ck->d) * ck->d;
            if (ck->seg_c != c) {
                /* replay u(c+1..it): FD, free surface, THEN the float source term (propagation.c:646-672) */
                if (c - 1 >= 0) memcpy(f0, ck->store + (size_t)ck->slot[c - 1] * n, frame_bytes(g));
                else memset(f0, 0, frame_bytes(g));
                memcpy(f1, ck->store + (size_t)ck->slot[c] * n, frame_bytes(g));
                for (int itt = c; itt < it; itt++) {
                    fd_step(f2, f1, f0, g);
                    if (g->fs == 1) free_surface(f2, g);
                    f2[is] += (real)s->src[itt] * g->K[is] * rdt * rdt * g->invdx * g->invdz;
                    memcpy(ck->seg + (size_t)(itt - c) * n, f2, frame_bytes(g));
                    real *tmp = f0; f0 = f1; f1 = f2; f2 = tmp;
                }
                ck->seg_c = c;
            }
            u = ck->seg + (size_t)(it - c - 1) * n;
        }
        /* adjoint source into p1 before the stencil (propagation.c:676-682) */
        for (int itr = 0; itr < s->ntr; ++itr) {
            size_t ig = IDX(s->igx[itr] + pml, s->igz[itr] + pml, Nz);
            p1[ig] -= adj[(size_t)itr * nt + it] * g->K[ig] * rdt * rdt * g->invdx * g->invdz;
        }
        fd_step(p2, p1, p0, g);
        if (g->fs == 1) free_surface(p2, g);
        if (it % MST == 0) {
#pragma omp parallel for schedule(static)
            for (int ix = pml; ix < pml + g->nxx; ++ix)
                for (int iz = pml; iz < pml + g->nz; ++iz) {
                    size_t i = IDX(ix, iz, Nz);
                    G[IDX(ix - pml, iz - pml, g->nz)] += (double)((p2[i] - (real)2.0 * p1[i] + p0[i]) * g->invdtdt * u[i]);
                }
        }
        real *tmp = p0; p0 = p1; p1 = p2; p2 = tmp;
    }
    for (size_t i = 0; i < (size_t)g->nz * g->nxx; i++) G[i] = 2.0 * G[i] / ((double)(rhom_w[i] * vpm_w[i]));
    free(p0); free(p1); free(p2); free(f0); free(f1); free(f2);
}

/* ------------------------------------------------------ adjoint source etc */

/* taper_traces, common.c:796-895; tr is ntr traces of nt samples */
static void taper_real(real *tr, int nt, int ntr, int taperLenTime, int taperLenTrace)
{
    if (taperLenTime > 0) {
        if (taperLenTime > nt / 3) taperLenTime = nt / 3;
        real *tc = malloc(sizeof(real) * (taperLenTime + 1));
        for (int it = 0; it <= taperLenTime; it++) {
            real x = (real)ORC_PI * it / taperLenTime;
            tc[it] = (real)0.5 * ((real)1.0 + RCOS(x));
        }
        for (int itr = 0; itr < ntr; itr++)
            for (int it = 0; it <= taperLenTime; it++) tr[(size_t)itr * nt + it] *= tc[taperLenTime - it];
        for (int itr = 0; itr < ntr; itr++)
            for (int it = 0; it <= taperLenTime; it++) tr[(size_t)itr * nt + nt - taperLenTime - 1 + it] *= tc[it];
        free(tc);
    }
    if (taperLenTrace > 0) {
        if (taperLenTrace > ntr / 3) taperLenTrace = ntr / 3;
        real *tc = malloc(sizeof(real) * (taperLenTrace + 1));
        for (int itr = 0; itr <= taperLenTrace; itr++) {
            real x = (real)ORC_PI * itr / taperLenTrace;
            tc[itr] = (real)0.5 * ((real)1.0 + RCOS(x));
        }
        for (int itr = 0; itr <= taperLenTrace; itr++)
            for (int it = 0; it < nt; it++) tr[(size_t)itr * nt + it] *= tc[taperLenTrace - itr];
        for (int itr = 0; itr <= taperLenTrace; itr++)
            for (int it = 0; it < nt; it++) tr[(size_t)(ntr - taperLenTrace - 1 + itr) * nt + it] *= tc[itr];
        free(tc);
    }
}

void orc_taper_traces(float *tr, int nt, int ntr, int taperLenTime, int taperLenTrace)
{
    size_t n = (size_t)nt * ntr;
    real *t = malloc(sizeof(real) * n);
    for (size_t i = 0; i < n; i++) t[i] = tr[i];
    taper_real(t, nt, ntr, taperLenTime, taperLenTrace);
    for (size_t i = 0; i < n; i++) tr[i] = (float)t[i];
    free(t);
}

/* taper lengths of compute_adjoint_source2d, optimization.c:347-365 */
static void adjoint_taper_lengths(const OrcShot *s, const float *vp_global, int nz, float freq,
                                  int *ltime, int *ltrace)
{
    double vp_sum = 0.0;
    for (int itr = 0; itr < s->ntr; itr++) /* window-local igx into the global model, as in the reference */
        vp_sum += vp_global[IDX(s->igx[itr], s->igz[itr], nz)];
    float vp_avg = (float)(vp_sum / s->ntr);
    if (freq == 0.0f) freq = s->fpeak;
    float kpass = freq / vp_avg;
    *ltime = (int)roundf((2.0f / freq) / s->dt) + 1;
    *ltrace = (int)roundf((2.0f / kpass) / s->dtr) + 1;
}

/* The cosine-tapered spectral windows of apply_traces_lowpass (common.c:584-687, filter 0)
 * and apply_traces_bandpass (common.c:689-794, filter 1), with the reference's float
 * expressions (PI is CWP's double constant: the bandpass argument is formed in double). */
static void filter_window(int filter, int n, float fpass, float fcut, float dt, float *win)
{
    float df = 1.0f / (n * dt);
    for (int it = 0; it < n; it++) {
        float f = it * df;
        if (filter == 0) {
            float taperLen = fcut - fpass;
            if (f < fpass) win[it] = 1.0f;
            else if (f >= fpass && f <= fcut) win[it] = 0.5f * (1.0f + cosf((float)3.141592653589793 * (f - fpass) / taperLen));
            else win[it] = 0.0f;
        } else {
            float lo = fpass, hi = fcut - fpass;
            if (f < fpass) win[it] = 0.5f * (1.0f + cosf(3.141592653589793 * (fpass - f) / lo));
            else if (f >= fpass && f <= fcut) win[it] = 0.5f * (1.0f + cosf(3.141592653589793 * (f - fpass) / hi));
            else win[it] = 0.0f;
        }
    }
}

/* The filter is FFT(real) -> window on the non-negative frequencies -> inverse FFT / n, i.e. a
 * circular convolution with h = IDFT(W_h) / n, W_h the window extended symmetrically.  Restated
 * as that convolution, h and the sums in double (the published operation; the reference's FFTW
 * rounding differs by ~1e-7 relative). tr: ntr traces of n samples, in place. */
static void filter_traces(real *tr, int n, int ntr, int filter, float fpass, float fcut, float dt)
{
    float *win = malloc(sizeof(float) * n);
    filter_window(filter, n, fpass, fcut, dt, win);
    double *cs = malloc(sizeof(double) * n), *h = malloc(sizeof(double) * n), *x = malloc(sizeof(double) * n);
    for (int m = 0; m < n; m++) cs[m] = cos(2.0 * 3.141592653589793 * m / n);
    for (int m = 0; m < n; m++) {
        double a = 0.0;
        for (int k = 0; k < n; k++) {
            int kk = k <= n / 2 ? k : n - k;
            a += (double)win[kk] * cs[(int)(((long long)k * m) % n)];
        }
        h[m] = a / n;
    }
    for (int itr = 0; itr < ntr; itr++) {
        real *t = tr + (size_t)itr * n;
        for (int i = 0; i < n; i++) x[i] = t[i];
        for (int j = 0; j < n; j++) {
            double a = 0.0;
            for (int i = 0; i < n; i++) a += h[(j - i + n) % n] * x[i];
            t[j] = (real)a;
        }
    }
    free(win); free(cs); free(h); free(x);
}

/* compute_adjoint_source2d, optimization.c:300-419: residual, then for filters 0/1 the time
 * taper, time filter, trace taper and trace (wavenumber) filter, then both tapers */
static int adjoint_source_real(const OrcShot *s, const float *vp_global, int nz, float freq, int filter,
                               const real *pre, const float *obs, real *adj)
{
    size_t n = (size_t)s->ns * s->ntr;
    for (size_t i = 0; i < n; i++) adj[i] = pre[i] - (real)obs[i];
    int lt, lr;
    adjoint_taper_lengths(s, vp_global, nz, freq, &lt, &lr);
    if (filter == 0 || filter == 1) {
        double vp_sum = 0.0;
        for (int itr = 0; itr < s->ntr; itr++) vp_sum += vp_global[IDX(s->igx[itr], s->igz[itr], nz)];
        float vp_avg = (float)(vp_sum / s->ntr);
        float f = freq == 0.0f ? s->fpeak : freq;
        float kpass = f / vp_avg;
        taper_real(adj, s->ns, s->ntr, lt, 0);
        filter_traces(adj, s->ns, s->ntr, filter, f, 2.0f * f, s->dt);
        taper_real(adj, s->ns, s->ntr, 0, lr);
        real *tp = malloc(sizeof(real) * n);  /* [ns][ntr]: one vector over the traces per sample */
        for (int itr = 0; itr < s->ntr; itr++)
            for (int it = 0; it < s->ns; it++) tp[(size_t)it * s->ntr + itr] = adj[(size_t)itr * s->ns + it];
        filter_traces(tp, s->ntr, s->ns, filter, kpass, 2.0f * kpass, s->dtr);
        for (int itr = 0; itr < s->ntr; itr++)
            for (int it = 0; it < s->ns; it++) adj[(size_t)itr * s->ns + it] = tp[(size_t)it * s->ntr + itr];
        free(tp);
    }
    taper_real(adj, s->ns, s->ntr, lt, lr);
    return 0;
}

void orc_adjoint_source(const OrcShot *shot, const float *vp_global, int nz, float freq, int filter,
                        const float *pre, const float *obs, float *adj)
{
    size_t n = (size_t)shot->ns * shot->ntr;
    real *p = malloc(sizeof(real) * n), *a = malloc(sizeof(real) * n);
    for (size_t i = 0; i < n; i++) p[i] = pre[i];
    adjoint_source_real(shot, vp_global, nz, freq, filter, p, obs, a);
    for (size_t i = 0; i < n; i++) adj[i] = (float)a[i];
    free(p); free(a);
}

/* apply_gradient_shot_precondition, optimization.c:58-97 */
static void shot_precondition_real(real *grad, real *precond, int n)
{
    double sum = 0.0;
    for (int i = 0; i < n; i++) sum += (double)precond[i];
    real avg = (real)(sum / n);
    for (int i = 0; i < n; i++) {
        real factor = (real)1.0 + precond[i] / ((real)7.0 * avg);
        grad[i] = grad[i] / factor;
        precond[i] = precond[i] / factor;
    }
}
void orc_shot_precondition(float *grad, float *precond, int n)
{
    real *g = malloc(sizeof(real) * n), *p = malloc(sizeof(real) * n);
    for (int i = 0; i < n; i++) { g[i] = grad[i]; p[i] = precond[i]; }
    shot_precondition_real(g, p, n);
    for (int i = 0; i < n; i++) { grad[i] = (float)g[i]; precond[i] = (float)p[i]; }
    free(g); free(p);
}

/* apply_gradient_precondition, optimization.c:13-56 */
static void global_precondition_real(real *grad, const real *precond, int n, real alpha)
{
    if (alpha <= (real)0.0) alpha = (real)0.005;
    double e = 0.0;
    for (int i = 0; i < n; i++) e += (double)precond[i] * (double)precond[i];
    real rms = (real)sqrt(e / n);
    for (int i = 0; i < n; i++) grad[i] = grad[i] / (precond[i] + alpha * rms);
}
void orc_global_precondition(float *grad, const float *precond, int n, float alpha)
{
    real *g = malloc(sizeof(real) * n), *p = malloc(sizeof(real) * n);
    for (int i = 0; i < n; i++) { g[i] = grad[i]; p[i] = precond[i]; }
    global_precondition_real(g, p, n, (real)alpha);
    for (int i = 0; i < n; i++) grad[i] = (float)g[i];
    free(g); free(p);
}

/* ------------------------------------------------------------ per-shot API */

static void window_model(const float *m, int nz, int ix_min, int nxx, float *out)
{
    memcpy(out, m + (size_t)ix_min * nz, sizeof(float) * (size_t)nz * nxx);
}

/* sources and receivers must sit where the stencil updates the field every step
 * (x in [3, Nx-4], z in [izStart, Nz-4] of the padded grid, propagation.c:534-537) */
static int in_fd_range(int x, int z, int nz, int nxx, int pml, int fs)
{
    int X = x + pml, Z = z + pml, Nx = nxx + 2 * pml, Nz = nz + 2 * pml;
    int z0 = fs ? pml : 3;
    return x >= 0 && x < nxx && z >= 0 && z < nz && X >= 3 && X <= Nx - 4 && Z >= z0 && Z <= Nz - 4;
}
static int check_shot(const OrcShot *s, int nt, int nz, int nxx, int pml, int fs)
{
    if (s->ntr <= 0 || s->ns <= 0 || s->sampleRate <= 0 || nt <= 0) return -1;
    if ((nt - 1) / s->sampleRate + 1 > s->ns) return -2;
    if (fs && pml < 3) return -5;
    if (!in_fd_range(s->isx, s->isz, nz, nxx, pml, fs)) return -3;
    for (int i = 0; i < s->ntr; i++)
        if (!in_fd_range(s->igx[i], s->igz[i], nz, nxx, pml, fs)) return -4;
    return 0;
}

int orc_forward(const OrcShot *s, const float *vpm, const float *rhom, int nz, int nx,
                float dx, float dz, float dt, int nt, int pml, int fs, float *traces)
{
    int rc = check_shot(s, nt, nz, nx, pml, fs);
    if (rc) return rc;
    Grid g;
    grid_build(&g, vpm, rhom, nz, nx, pml, dx, dz, dt, s->fpeak, fs);
    size_t n = (size_t)s->ntr * s->ns;
    real *tr = calloc(n, sizeof(real));
    for (size_t i = 0; i < n; i++) tr[i] = traces[i]; /* samples the loop never writes keep their value */
    engine_forward(&g, s, nt, 0, 0, NULL, NULL, tr, NULL, NULL);
    for (size_t i = 0; i < n; i++) traces[i] = (float)tr[i];
    free(tr);
    grid_free(&g);
    return 0;
}

/* interpolate_traces with r <= 1 is a copy (common.c:511-516) */
/* interpolate_traces, common.c:482-582: zero-stuffing by r, a rectangular window of height r
 * over |k| < N/(2r) of the length-N spectrum (N = (ns-1)r+1), inverse transform, real part / N.
 * Restated as y[i] = sum_j x[j] g[(i - jr) mod N] with g = IDFT(window) / N in double.  Samples
 * beyond N (when N < nt) are zero.  r <= 1 copies. */
static int interp_traces(const real *tr, int ntr, int ns, int r, int nt, real *out)
{
    memset(out, 0, sizeof(real) * (size_t)ntr * nt);
    if (r <= 1) {
        for (int itr = 0; itr < ntr; itr++)
            memcpy(out + (size_t)itr * nt, tr + (size_t)itr * ns, sizeof(real) * (size_t)ns);
        return 0;
    }
    const int N = (ns - 1) * r + 1, nkeep = N / (2 * r);
    double *g = malloc(sizeof(double) * N), *cs = malloc(sizeof(double) * N);
    for (int m = 0; m < N; m++) cs[m] = cos(2.0 * 3.141592653589793 * m / N);
    for (int m = 0; m < N; m++) {
        double a = 0.0;
        for (int k = 0; k < N; k++) {
            const int in_band = k < nkeep || k >= N - nkeep + 1;
            if (in_band) a += (double)r * cs[(int)(((long long)k * m) % N)];
        }
        g[m] = a / N;
    }
    const int nout = N < nt ? N : nt;
    for (int itr = 0; itr < ntr; itr++) {
        const real *x = tr + (size_t)itr * ns;
        real *y = out + (size_t)itr * nt;
        for (int i = 0; i < nout; i++) {
            double a = 0.0;
            for (int j = 0; j < ns; j++) a += g[((i - j * r) % N + N) % N] * (double)x[j];
            y[i] = (real)a;
        }
    }
    free(g); free(cs);
    return 0;
}

/* one shot of propagation.c:897-983 (problem 1), in the oracle precision */
static int shot_gradient_real(const OrcShot *s, const float *vp, const float *rho, int nz, int nx,
                              float dx, float dz, float dt, int nt, int pml, int fs, float freq, int filter,
                              int precondition, const float *obs, real *pre, real *g_shot, real *h_shot)
{
    int nxx = s->ix_max - s->ix_min + 1;
    int rc = check_shot(s, nt, nz, nxx, pml, fs);
    if (rc) return rc;
    if (filter < 0 || filter > 2) return -10;
    float *vpw = malloc(sizeof(float) * (size_t)nz * nxx), *rhow = malloc(sizeof(float) * (size_t)nz * nxx);
    window_model(vp, nz, s->ix_min, nxx, vpw);
    window_model(rho, nz, s->ix_min, nxx, rhow);
    real *vpr = malloc(sizeof(real) * (size_t)nz * nxx), *rhor = malloc(sizeof(real) * (size_t)nz * nxx);
    for (size_t i = 0; i < (size_t)nz * nxx; i++) { vpr[i] = vpw[i]; rhor[i] = rhow[i]; }
    Grid g;
    grid_build(&g, vpw, rhow, nz, nxx, pml, dx, dz, dt, s->fpeak, fs);
    Ckpt ck;
    ck_alloc(&ck, nt, (size_t)g.Nz * g.Nx);
    size_t m = (size_t)nz * nxx;
    double *H = calloc(m, sizeof(double)), *G = calloc(m, sizeof(double));
    engine_forward(&g, s, nt, 1, precondition, vpr, rhor, pre, &ck, H);
    size_t nrec = (size_t)s->ntr * s->ns;
    real *adj = malloc(sizeof(real) * nrec), *adjt = malloc(sizeof(real) * (size_t)s->ntr * nt);
    adjoint_source_real(s, vp, nz, freq, filter, pre, obs, adj);
    memcpy(pre, adj, sizeof(real) * nrec); /* the reference writes the adjoint source in place */
    interp_traces(pre, s->ntr, s->ns, s->sampleRate, nt, adjt);
    engine_adjoint(&g, s, nt, adjt, vpr, rhor, &ck, G);
    /* grad_per_shot and precond_per_shot are float arrays in the reference (FP32 round trip) */
    for (size_t i = 0; i < m; i++) {
        g_shot[i] = (real)G[i];
        if (precondition == 1) h_shot[i] = (real)H[i];
    }
    if (precondition == 1) shot_precondition_real(g_shot, h_shot, (int)m);
    free(H); free(G); free(adj); free(adjt); free(vpw); free(rhow); free(vpr); free(rhor);
    ck_free(&ck);
    grid_free(&g);
    return 0;
}

int orc_shot_gradient(const OrcShot *s, const float *vp, const float *rho, int nz, int nx, float dx, float dz,
                      float dt, int nt, int pml, int fs, float freq, int filter, int precondition,
                      const float *obs, float *traces_pre, float *grad_shot, float *precond_shot)
{
    int nxx = s->ix_max - s->ix_min + 1;
    size_t m = (size_t)nz * nxx, nrec = (size_t)s->ntr * s->ns;
    real *pre = malloc(sizeof(real) * nrec), *g = calloc(m, sizeof(real)), *h = calloc(m, sizeof(real));
    for (size_t i = 0; i < nrec; i++) pre[i] = traces_pre[i];
    int rc = shot_gradient_real(s, vp, rho, nz, nx, dx, dz, dt, nt, pml, fs, freq, filter, precondition, obs, pre, g, h);
    if (!rc) {
        for (size_t i = 0; i < nrec; i++) traces_pre[i] = (float)pre[i];
        for (size_t i = 0; i < m; i++) {
            grad_shot[i] = (float)g[i];
            if (precond_shot) precond_shot[i] = (float)h[i];
        }
    }
    free(pre); free(g); free(h);
    return rc;
}

int orc_propagation(const float *vp, const float *rho, const OrcShot *shots, int Nshot, int nz, int nx,
                    float dx, float dz, float dt, int nt, int pml, int fs, float freq, float filter,
                    int precondition, int problem, float *const *obs, float *const *pre, float *grad)
{
    int ifilter = (int)filter; /* the float argument meets an int parameter (optimization.h:17) */
    if (problem == 0 || problem == 2) {
        for (int is = 0; is < Nshot; is++) {
            const OrcShot *s = &shots[is];
            int nxx = s->ix_max - s->ix_min + 1;
            float *vpw = malloc(sizeof(float) * (size_t)nz * nxx), *rhow = malloc(sizeof(float) * (size_t)nz * nxx);
            window_model(vp, nz, s->ix_min, nxx, vpw);
            window_model(rho, nz, s->ix_min, nxx, rhow);
            int rc = orc_forward(s, vpw, rhow, nz, nxx, dx, dz, dt, nt, pml, fs, pre[is]);
            free(vpw); free(rhow);
            if (rc) return rc;
            if (problem == 2) {
                size_t nrec = (size_t)s->ntr * s->ns;
                real *p = malloc(sizeof(real) * nrec), *a = malloc(sizeof(real) * nrec);
                for (size_t i = 0; i < nrec; i++) p[i] = pre[is][i];
                rc = adjoint_source_real(s, vp, nz, freq, ifilter, p, obs[is], a);
                for (size_t i = 0; i < nrec; i++) pre[is][i] = (float)a[i];
                free(p); free(a);
                if (rc) return rc;
            }
        }
        return 0;
    }
    if (problem != 1) return -20;
    size_t m = (size_t)nz * nx;
    double *gc = calloc(m, sizeof(double)), *hc = calloc(m, sizeof(double));
    int rc = 0;
    for (int is = 0; is < Nshot && !rc; is++) {
        const OrcShot *s = &shots[is];
        int nxx = s->ix_max - s->ix_min + 1;
        size_t mw = (size_t)nz * nxx, nrec = (size_t)s->ntr * s->ns;
        real *p = malloc(sizeof(real) * nrec), *g = calloc(mw, sizeof(real)), *h = calloc(mw, sizeof(real));
        for (size_t i = 0; i < nrec; i++) p[i] = pre[is][i];
        rc = shot_gradient_real(s, vp, rho, nz, nx, dx, dz, dt, nt, pml, fs, freq, ifilter, precondition, obs[is], p, g, h);
        if (!rc) {
            for (size_t i = 0; i < nrec; i++) pre[is][i] = (float)p[i];
            /* stack in shot order, propagation.c:953-976 */
            for (int ix = s->ix_min; ix <= s->ix_max; ix++)
                for (int iz = 0; iz < nz; iz++) {
                    gc[IDX(ix, iz, nz)] += g[IDX(ix - s->ix_min, iz, nz)];
                    if (precondition == 1) hc[IDX(ix, iz, nz)] += h[IDX(ix - s->ix_min, iz, nz)];
                }
        }
        free(p); free(g); free(h);
    }
    if (!rc) {
        real *gr = malloc(sizeof(real) * m), *hr = malloc(sizeof(real) * m);
        for (size_t i = 0; i < m; i++) { gr[i] = (real)gc[i]; hr[i] = (real)hc[i]; }
        if (precondition == 1) global_precondition_real(gr, hr, (int)m, (real)0.005f);
        for (size_t i = 0; i < m; i++) grad[i] = (float)gr[i];
        free(gr); free(hr);
    }
    free(gc); free(hc);
    return rc;
}

/* ------------------------------------------------------ FWI-loop reductions */

/* calculate_objective_value, optimization.c:99-132 (shot order, sequential) */
float orc_objective(float *const *traces, const int *ntr, const int *ns, int Nshot)
{
    double fun = 0.0;
    for (int is = 0; is < Nshot; is++)
        for (size_t i = 0; i < (size_t)ntr[is] * ns[is]; i++) fun += traces[is][i] * traces[is][i];
    fun *= 0.5;
    return (float)fun;
}

/* calculate_step_length, optimization.c:134-176 */
float orc_step_length(float *const *pre0, float *const *pre1, const int *ntr, const int *ns, int Nshot)
{
    double num = 0.0, den = 0.0;
    for (int is = 0; is < Nshot; is++)
        for (size_t i = 0; i < (size_t)ntr[is] * ns[is]; i++) {
            float delta = pre0[is][i] - pre1[is][i];
            num += pre0[is][i] * delta;
            den += delta * delta;
        }
    if (den == 0.0) return 0.0f;
    return (float)(num / den);
}

/* compute_model_perturbation, optimization.c:178-298 */
float orc_model_perturbation(float fraction, const float *slowness, const float *gradient, float *out, int len)
{
    int hist[1001];
    float Max = 0.0f, Min = 0.0f, scalar;
    const float cap = 0.99f;
    double average = 0;
    for (int i = 0; i < 1001; i++) hist[i] = 0;
    for (int i = 0; i < len; i++) {
        if (gradient[i] > Max) Max = gradient[i];
        if (gradient[i] < Min) Min = gradient[i];
    }
    float interval = (Max - Min) / 1000.0;
    int pos = 0;
    for (int i = 0; i < len; i++) {
        pos = (int)((gradient[i] - Min) / interval + 0.5);
        hist[pos]++;
    }
    int peak = 0;
    for (int i = 0; i < 1001; i++)
        if (hist[i] > peak) { peak = hist[i]; pos = i; }
    int hi = pos, lo = pos;
    float acc = (float)hist[hi] / (float)len;
    while (acc < cap) {
        if (hi < 1000) { hi++; acc += (float)hist[hi] / (float)len; }
        if (lo > 0) { lo--; acc += (float)hist[lo] / (float)len; }
    }
    float a = fabsf(Min + lo * interval), b = fabsf(Min + hi * interval);
    scalar = a > b ? a : b;
    for (int i = 0; i < len; i++) average += slowness[i];
    scalar = (average / len * fraction) / scalar;
    for (int i = 0; i < len; i++) out[i] = -scalar * gradient[i];
    return scalar;
}

/* smooth2D, common.c:927-1040 */
void orc_smooth2d(const float *in, float *out, int nx, int nz, int N, int iszdirect)
{
    float *w = malloc(sizeof(float) * (2 * N + 1));
    for (int i = 0; i < 2 * N + 1; i++) {
        w[i] = cos(ORC_PI * (i - N) / (2.0 * N));
        w[i] *= w[i];
    }
    int n1 = iszdirect == 1 ? nz : nx;
    for (int j = 0; j < n1; j++) {
        int ws = j >= N ? 0 : N - j, ds = j >= N ? j - N : 0;
        int we = (n1 - 1 - j < N) ? 2 * N - (N - (n1 - 1 - j)) : 2 * N;
        int n2 = iszdirect == 1 ? nx : nz;
        for (int k = 0; k < n2; k++) {
            double a1 = 0.0, a2 = 0.0;
            for (int ic = ws, ic2 = ds; ic <= we; ic++, ic2++) {
                float v = iszdirect == 1 ? in[IDX(k, ic2, nz)] : in[IDX(ic2, k, nz)];
                a1 += w[ic] * v;
                a2 += w[ic];
            }
            float r = a1 / (a2 + FLT_MIN);
            if (iszdirect == 1) out[IDX(k, j, nz)] = r;
            else out[IDX(j, k, nz)] = r;
        }
    }
    free(w);
}

/* vp2density, common.c:298-330 (Gardner) */
void orc_vp2density(const float *vp, float *rho, int n)
{
    for (int i = 0; i < n; i++) rho[i] = 310.0f * powf(vp[i], 0.25f);
}

static void water(float *m, float v, int wd, int nx, int nz)
{
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < wd; iz++) m[IDX(ix, iz, nz)] = v;
}
static void clip(float *m, int n, float lo, float hi)
{
    for (int i = 0; i < n; i++) {
        if (m[i] > hi) m[i] = hi;
        else if (m[i] < lo) m[i] = lo;
    }
}
static void inv_or_zero(const float *a, float *b, int n)
{
    for (int i = 0; i < n; i++) b[i] = a[i] != 0.0f ? 1.0f / a[i] : 0.0f;
}

/* trial model of acoustic2d_fwi.c:428-439 */
void orc_fwi_trial(const float *slow, const float *perturb, float *vp, float *rho, int nx, int nz,
                   int waterdepth, float vp_water, float rho_water, float vpmin, float vpmax,
                   float rhomin, float rhomax, int gardner)
{
    int n = nx * nz;
    for (int i = 0; i < n; i++) vp[i] = slow[i] + perturb[i];
    inv_or_zero(vp, vp, n);
    water(vp, vp_water, waterdepth, nx, nz);
    clip(vp, n, vpmin, vpmax);
    if (gardner == 1) {
        orc_vp2density(vp, rho, n);
        water(rho, rho_water, waterdepth, nx, nz);
        clip(rho, n, rhomin, rhomax);
    }
}

/* model update of acoustic2d_fwi.c:452-465 */
void orc_fwi_update(float *slow, float *vp, float *rho, const float *perturb, float steplen,
                    int nx, int nz, int waterdepth, float vp_water, float rho_water,
                    float vpmin, float vpmax, float rhomin, float rhomax, int gardner)
{
    int n = nx * nz;
    for (int i = 0; i < n; i++) slow[i] = slow[i] + steplen * perturb[i];
    inv_or_zero(slow, vp, n);
    water(vp, vp_water, waterdepth, nx, nz);
    clip(vp, n, vpmin, vpmax);
    if (gardner == 1) {
        orc_vp2density(vp, rho, n);
        water(rho, rho_water, waterdepth, nx, nz);
        clip(rho, n, rhomin, rhomax);
    }
    inv_or_zero(vp, slow, n);
}
