// fwi_dropin.cu -- the reference-shaped entry points (Record2D, float**) on top of
// the native context API.  A process-wide context per device keeps the model,
// shots and buffers between calls, so the FWI loop of acoustic2d_fwi.c, which calls
// iso_acoustic2d_propagation three times per iteration with the same geometry,
// re-uploads only what changed.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/fwi_b200.h"

namespace {

struct DropIn {
    fwi_ctx *ctx = nullptr;
    int device = -1;
    std::vector<float> vp, rho;  // model of the last call
    int nz = 0, nx = 0, nt = 0, pml = -1, fs = -1;
    float dx = 0, dz = 0, dt = 0;
    std::vector<fwi_shot> shots;  // geometry of the last call (pointers into the caller's records)
    std::vector<std::vector<float>> src;
    std::vector<std::vector<int>> igx, igz;
};
DropIn g_di;
std::mutex g_mu;

int env_path()
{
    const char *p = getenv("FWI_PATH");
    if (p && (!strcmp(p, "plain") || !strcmp(p, "0"))) return FWI_PATH_PLAIN;
    return FWI_PATH_BATCHED;
}

int env_device()
{
    const char *p = getenv("FWI_DEVICE");
    return p ? atoi(p) : 0;
}

bool contiguous(float **rows, int n1, int n2)
{
    for (int i = 1; i < n2; i++)
        if (rows[i] != rows[0] + (size_t)i * n1) return false;
    return true;
}

bool same_shots(const Record2D *r, int n, int nt)
{
    if ((int)g_di.shots.size() != n) return false;
    for (int i = 0; i < n; i++) {
        const fwi_shot &s = g_di.shots[i];
        if (s.isx != r[i].isx || s.isz != r[i].isz || s.ntr != r[i].ntr || s.ns != r[i].ns ||
            s.sampleRate != r[i].sampleRate || s.ix_min != r[i].ix_min || s.ix_max != r[i].ix_max ||
            s.dt != r[i].dt || s.dtr != r[i].dtr || s.fpeak != r[i].fpeak || s.shotID != r[i].shotID)
            return false;
        if (memcmp(g_di.src[i].data(), r[i].src, (size_t)nt * 4) ||
            memcmp(g_di.igx[i].data(), r[i].igx, (size_t)r[i].ntr * 4) ||
            memcmp(g_di.igz[i].data(), r[i].igz, (size_t)r[i].ntr * 4))
            return false;
    }
    return true;
}

}  // namespace

extern "C" int fwi_iso_acoustic2d_propagation(float **vp, float **rho, Record2D *obs, int Nshot, int nz, int nx,
                                              float dx, float dz, float dt, int nt, int pml, int fs, float freq,
                                              float filter, int precondition, int problem, int iter, int verbose,
                                              Record2D *pre, float **grad)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!vp || !rho || !obs || !pre || Nshot <= 0) return FWI_ERR_ARG;
    if (problem == 1 && !grad) return FWI_ERR_ARG;
    if (!contiguous(vp, nz, nx) || !contiguous(rho, nz, nx)) return FWI_ERR_ARG;
    int rc;
    const int dev = env_device();
    if (!g_di.ctx || g_di.device != dev) {
        if (g_di.ctx) fwi_ctx_destroy(g_di.ctx);
        g_di = DropIn();
        if ((rc = fwi_ctx_create(&g_di.ctx, dev, 0)) != FWI_OK) return rc;
        g_di.device = dev;
    }
    fwi_ctx *c = g_di.ctx;
    const size_t m = (size_t)nz * nx;
    const bool same_grid = nz == g_di.nz && nx == g_di.nx && nt == g_di.nt && pml == g_di.pml && fs == g_di.fs &&
                           dx == g_di.dx && dz == g_di.dz && dt == g_di.dt;
    const bool same_model = same_grid && g_di.vp.size() == m && !memcmp(g_di.vp.data(), vp[0], m * 4) &&
                            !memcmp(g_di.rho.data(), rho[0], m * 4);
    bool reshot = !same_grid;
    if (!same_model) {
        if ((rc = fwi_ctx_set_model(c, vp[0], rho[0], nz, nx, dx, dz, dt, nt, pml, fs)) != FWI_OK) return rc;
        g_di.vp.assign(vp[0], vp[0] + m);
        g_di.rho.assign(rho[0], rho[0] + m);
        g_di.nz = nz; g_di.nx = nx; g_di.nt = nt; g_di.pml = pml; g_di.fs = fs;
        g_di.dx = dx; g_di.dz = dz; g_di.dt = dt;
    }
    if (reshot || !same_shots(obs, Nshot, nt)) {
        // the new geometry is built aside and becomes the cached one only once the context took it
        g_di.shots.clear();
        std::vector<fwi_shot> sh(Nshot);
        std::vector<std::vector<float>> src(Nshot);
        std::vector<std::vector<int>> igx(Nshot), igz(Nshot);
        for (int i = 0; i < Nshot; i++) {
            const Record2D &r = obs[i];
            if (!r.src || !r.igx || !r.igz || r.ntr < 0) return FWI_ERR_ARG;
            src[i].assign(r.src, r.src + nt);
            igx[i].assign(r.igx, r.igx + r.ntr);
            igz[i].assign(r.igz, r.igz + r.ntr);
            fwi_shot &s = sh[i];
            s.shotID = r.shotID; s.isx = r.isx; s.isz = r.isz; s.ntr = r.ntr; s.ns = r.ns;
            s.sampleRate = r.sampleRate; s.ix_min = r.ix_min; s.ix_max = r.ix_max;
            s.dt = r.dt; s.dtr = r.dtr; s.fpeak = r.fpeak;
            s.src = src[i].data(); s.igx = igx[i].data(); s.igz = igz[i].data();
        }
        if ((rc = fwi_ctx_set_shots(c, sh.data(), Nshot)) != FWI_OK) return rc;
        g_di.src.swap(src);  // the vectors' buffers move with them: sh's pointers stay valid
        g_di.igx.swap(igx);
        g_di.igz.swap(igz);
        g_di.shots = sh;
    }
    if (problem == 1 || problem == 2) {
        std::vector<const float *> o(Nshot);
        for (int i = 0; i < Nshot; i++) {
            if (!obs[i].traces_p || !contiguous(obs[i].traces_p, obs[i].ns, obs[i].ntr)) return FWI_ERR_ARG;
            o[i] = obs[i].traces_p[0];
        }
        if ((rc = fwi_ctx_set_observed(c, o.data())) != FWI_OK) return rc;
    }
    // the reference's intermediate files (shotInterval / snapInterval from the environment)
    if ((rc = fwi_ctx_set_verbose(c, verbose, iter, 0, 0, nullptr)) != FWI_OK) return rc;
    if ((rc = fwi_ctx_run(c, problem, freq, (int)filter, precondition, env_path())) != FWI_OK) return rc;
    for (int i = 0; i < Nshot; i++) {
        if (!pre[i].traces_p || !contiguous(pre[i].traces_p, pre[i].ns, pre[i].ntr)) return FWI_ERR_ARG;
        if ((rc = fwi_ctx_get_traces(c, i, pre[i].traces_p[0])) != FWI_OK) return rc;
    }
    if (problem == 1) {
        if (!contiguous(grad, nz, nx)) return FWI_ERR_ARG;
        if ((rc = fwi_ctx_get_gradient(c, grad[0])) != FWI_OK) return rc;
    }
    return FWI_OK;
}

extern "C" void iso_acoustic2d_propagation(float **vp, float **rho, Record2D *obs, int Nshot, int nz, int nx, float dx,
                                           float dz, float dt, int nt, int pml, int fs, float freq, float filter,
                                           int precondition, int problem, int iter, int verbose, Record2D *pre,
                                           float **grad)
{
    int rc = fwi_iso_acoustic2d_propagation(vp, rho, obs, Nshot, nz, nx, dx, dz, dt, nt, pml, fs, freq, filter,
                                            precondition, problem, iter, verbose, pre, grad);
    if (rc != FWI_OK)
        fprintf(stderr, "<error>: iso_acoustic2d_propagation failed (status %d): %s\n", rc, fwi_last_error());
}
