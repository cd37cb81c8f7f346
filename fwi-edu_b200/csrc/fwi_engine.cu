// fwi_engine.cu -- host side of the B200 engine and its C-ABI.
//
// A context (fwi_ctx) holds one model on the global grid, the shots, and every
// device buffer a run needs.  Shots that share a model window and wavelet peak
// frequency share one Plan (the coefficient fields of propagation.c:508-532),
// uploaded once per model version.  Each shot owns its wavefield storage:
// checkpoint frames, scratch frames, the replayed frames kept for imaging, FP64
// accumulators and its gathers.
//
// A run is a sequence of launches of k_step.  What each launch does for each
// shot is read from a small program on the device (int4 per launch: up to two
// items, e.g. a replay step of one segment next to an adjoint step of another),
// so the host loop only issues launches.  On the batched path all shots of a
// group go into every launch and the whole launch sequence is captured once as
// a CUDA graph and replayed; on the plain path shots run one after another, one
// launch per step, as the reference's shot loop does (propagation.c:857, :895).
#include <cuda.h>
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <deque>
#include <functional>
#include <tuple>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/fwi_b200.h"
#include "fwi_aux.cuh"
#include "fwi_kernels.cuh"
#include "fwi_setup.h"
#include "fwi_step.cuh"
#include "fwi_tile.cuh"
#include "fwi_tile2.cuh"
#include "fwi_wave.cuh"
#include "fwi_optim.cuh"
#include "fwi_fft.cuh"

using namespace fwi;

// ---------------------------------------------------------------- errors
static thread_local std::string g_err;
static int fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}
#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(FWI_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define TRY(call)                 \
    do {                          \
        int r_ = (call);          \
        if (r_ != FWI_OK) return r_; \
    } while (0)

extern "C" const char *fwi_last_error(void) { return g_err.c_str(); }
extern "C" const char *fwi_version(void) { return "fwi-b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------------- context
struct ShotHost {
    fwi_shot s;
    std::vector<float> src;
    std::vector<int> igx, igz;
};

struct Plan {
    int ix_min = 0, ix_max = -1;
    float fpeak = 0.f;
    unsigned long long version = ~0ull;
    fwi_coefs hc{};
    float *d_coef = nullptr;  // c1, c2, ck, irx, irz, ir, each Nx*ld
    int Nx = 0, Nz = 0, ld = 0, G = 0;
    size_t frame() const { return (size_t)Nx * ld; }
};

struct ShotRun {
    int shot = -1;
    Plan *plan = nullptr;
    ShotDesc d{};
    // per-run host-side extras
    int Lt = 0, Lr = 0;
    float fpass = 0.f, kpass = 0.f;  // residual filter pass frequency (Hz) and wavenumber (1/m)
    float *d_tct = nullptr, *d_tcr = nullptr;
    float *d_gshot = nullptr, *d_hshot = nullptr;  // [nxx][nz] FP32 per-shot gradient / preconditioner
    bool has_ck = false;
    std::vector<void *> allocs;
};

struct Program {
    std::vector<int4> items;
    int4 *d = nullptr;
    int depth = 1;  // 2: items of the two-step kernel (fwi_tile2.cuh)
};

struct fwi_ctx {
    int device = 0;
    size_t budget = 0, used = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // model and run constants
    int nz = 0, nx = 0, nt = 0, pml = 0, fs = 0;
    float dx = 0, dz = 0, dt = 0;
    std::vector<float> vp, rho;
    float *d_vp = nullptr, *d_rho = nullptr;
    unsigned long long version = 0;
    bool host_model_valid = false;
    // shots
    std::vector<ShotHost> shots;
    std::vector<float *> d_obs, d_pre, d_pre_alt;  // d_pre_alt: the other gather set of a line search
    std::vector<float> slow;                        // slowness carried by the FWI iteration
    std::vector<std::unique_ptr<Plan>> plans;
    std::vector<std::unique_ptr<ShotRun>> runs;  // one per shot (batched) or one reused (plain)
    ShotDesc *d_desc = nullptr;
    int desc_cap = 0;
    // survey-wide outputs
    float *d_grad = nullptr, *d_prec = nullptr;
    double *d_gc = nullptr, *d_hc = nullptr;
    double *d_red = nullptr;     // reduction partials + results
    void *d_scratch = nullptr;   // small descriptor arrays
    size_t scratch_cap = 0;
    // programs and graphs, keyed by (kind, overlap)
    std::map<std::string, Program> progs;
    std::map<std::string, cudaGraphExec_t> graphs;
    fwi_stats stats{};
    int math = 0;  // 0: bit-exact arithmetic, 1: contracted multiply-adds
    int depth = 1;  // time steps per launch of the step kernel (1 or 2): tuned per shape unless
                    // FWI_DEPTH pins it
    bool depth_pinned = false;
    bool use_graphs = true;  // capture the batched launch sequences as CUDA graphs
    bool pdl = true;         // consecutive steps as programmatic dependent launches
    bool tune = true;        // time the step kernel's launch shapes once per shape (autotune)
    bool wave = false;       // forward passes as one persistent wavefront launch where they fit (FWI_PERSIST=1)
    bool fine = true;        // step launches wait for their neighbouring tiles only (TileSync; FWI_FINE=0: whole grid)
    // the observed gathers go up on a stream of their own, overlapping the forward pass; the
    // residual waits for them (ev_obs) the first time it reads them
    cudaStream_t xstream = nullptr;
    cudaEvent_t ev_obs = nullptr, ev_tail = nullptr;
    bool obs_pending = false;
    int *d_tflags = nullptr; // their completion flags
    int tflags_cap = 0;
    int *d_wave = nullptr;   // its abort word and per-block item counters
    int wave_cap = 0;
    std::map<std::string, long long> graph_launches;  // kernels each captured graph holds
    int last_tx = 0, last_nst = 0, last_chunk = 0, last_gpt = 0, last_minb = 0;  // the shape of the last launch
    bool last_wave = false;  // the last pass ran as one persistent wavefront launch
    int *d_err = nullptr;  // set by a step kernel whose tile copy did not complete
    std::map<void *, size_t> sizes;  // live device blocks of this context
    size_t peak = 0;
    // exchange hook of a shot-sharded run (one context per GPU): sums device doubles over ranks
    fwi_allreduce_fn ar_fn = nullptr;
    void *ar_user = nullptr;
    double *d_xchg = nullptr;  // the scalar sums handed to the hook
    // frame pools: the frame blocks of a shot group, consecutive (key: first shot of the
    // group on the batched path, -1 for the plain path's single shot)
    struct Pool {
        float *p = nullptr;
        size_t bytes = 0;
        int nfr = 0, ng = 0;
        long long frame = 0;
    };
    std::map<int, Pool> pools;
    // residual filters and trace interpolation: FFT spectra and twiddles, keyed by filter and size
    std::map<std::string, std::pair<float *, size_t>> ops;
    float *d_fft_tmp = nullptr;
    size_t fft_tmp_bytes = 0;
    long long launches = 0;
    double last_obj = 0.0;
    // verbose output (the reference's intermediate files), fwi_ctx_set_verbose
    struct Dump {
        int verbose = 0, iter = 0;
        int shot_interval = 20;    // every shot_interval-th shot is written out
        int snap_interval = 1000;  // snapshot time steps (verbose > 1)
        std::string dir;           // "" = the working directory, as the reference writes
        bool warned = false;
    } dump;
    bool snapping = false;  // the launches being issued belong to a pass that writes snapshots
    // device time of the step-kernel passes of the last run, per pass kind (0 forward of a
    // gradient or modeling run, 1 adjoint pass with its replay): event pairs around every
    // program launch, read when the run ends
    struct PassTimer {
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
        size_t used = 0;
        double ms = 0.0;
        long long launches = 0;
    } pass[2];
};

// Device memory comes from the stream-ordered allocator on the context's stream: a context
// that frees or grows its state never synchronises the device, so contexts on other streams
// (concurrent requests of a server) keep running.  Every block's size is tracked for the budget.
static int dmalloc(fwi_ctx *c, void **p, size_t bytes)
{
    if (c->budget && c->used + bytes > c->budget)
        return fail(FWI_ERR_NOMEM, "device budget exceeded: %zu + %zu > %zu bytes", c->used, bytes, c->budget);
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, c->stream);
    if (e != cudaSuccess) return fail(FWI_ERR_NOMEM, "cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e));
    e = cudaStreamSynchronize(c->stream);  // usable from any stream and from synchronous copies
    if (e != cudaSuccess) return fail(FWI_ERR_CUDA, "cudaStreamSynchronize: %s", cudaGetErrorString(e));
    c->sizes[*p] = bytes;
    c->used += bytes;
    c->peak = std::max(c->peak, c->used);
    return FWI_OK;
}
static void dfree(fwi_ctx *c, void *p, size_t = 0)
{
    if (!p) return;
    auto it = c->sizes.find(p);
    if (it != c->sizes.end()) {
        c->used -= std::min(c->used, it->second);
        c->sizes.erase(it);
    }
    cudaFreeAsync(p, c->stream);
}

// the main stream waits for the observed gathers' upload (before the residual reads them, or
// before their buffers are freed)
static int obs_join(fwi_ctx *c)
{
    if (!c->obs_pending) return FWI_OK;
    cudaError_t e = cudaStreamWaitEvent(c->stream, c->ev_obs, 0);
    if (e != cudaSuccess) return fail(FWI_ERR_CUDA, "cudaStreamWaitEvent: %s", cudaGetErrorString(e));
    c->obs_pending = false;
    return FWI_OK;
}

static void free_run(fwi_ctx *c, ShotRun *r)
{
    for (void *p : r->allocs) dfree(c, p);
    r->allocs.clear();
}

static void drop_graphs(fwi_ctx *c)
{
    for (auto &kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
}

static void free_runs(fwi_ctx *c)
{
    drop_graphs(c);
    for (auto &r : c->runs) free_run(c, r.get());
    c->runs.clear();
    for (auto &kv : c->pools) dfree(c, kv.second.p, kv.second.bytes);
    c->pools.clear();
}

extern "C" int fwi_ctx_create(fwi_ctx **out, int device, size_t budget)
{
    if (!out) return fail(FWI_ERR_ARG, "ctx pointer is NULL");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return fail(FWI_ERR_NODEVICE, "no CUDA device: this engine runs on the GPU only");
    if (device < 0 || device >= n) return fail(FWI_ERR_ARG, "device %d out of range (%d devices)", device, n);
    CK(cudaSetDevice(device));
    fwi_ctx *c = new fwi_ctx();
    c->device = device;
    c->budget = budget;
    if (const char *e = getenv("FWI_MATH")) c->math = atoi(e) ? 1 : 0;
    if (const char *e = getenv("FWI_DEPTH")) {
        c->depth = atoi(e) == 2 ? 2 : 1;
        c->depth_pinned = true;
    }
    if (const char *e = getenv("FWI_GRAPH")) c->use_graphs = e[0] != '0';  // 0: direct launches (profilers)
    if (const char *e = getenv("FWI_PDL")) c->pdl = e[0] != '0';
    if (const char *e = getenv("FWI_TUNE")) c->tune = e[0] != '0';            // 0: heuristic launch shapes
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->xstream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_obs, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_tail, cudaEventDisableTiming));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    TRY(dmalloc(c, (void **)&c->d_err, sizeof(int)));
    CK(cudaMemset(c->d_err, 0, sizeof(int)));
    if (const char *e = getenv("FWI_PERSIST")) c->wave = e[0] != '0';  // 1: forward passes as one wavefront launch
    c->wave_cap = 4096;  // abort word + one counter per resident block (148 SMs x a few blocks)
    TRY(dmalloc(c, (void **)&c->d_wave, c->wave_cap * sizeof(int)));
    if (const char *e = getenv("FWI_FINE")) c->fine = e[0] != '0';
    c->tflags_cap = 1 << 16;  // 2 halves x chunks x tiles; larger launches wait for the whole grid
    TRY(dmalloc(c, (void **)&c->d_tflags, c->tflags_cap * sizeof(int)));
    *out = c;
    return FWI_OK;
}

extern "C" int fwi_ctx_destroy(fwi_ctx *c)
{
    if (!c) return FWI_OK;
    cudaSetDevice(c->device);
    obs_join(c);
    cudaStreamSynchronize(c->stream);
    free_runs(c);
    for (auto &p : c->plans) fwi_free_coefs(&p->hc);
    // everything left in the allocator table belongs to this context
    for (auto &kv : c->sizes) cudaFreeAsync(kv.first, c->stream);
    c->sizes.clear();
    cudaStreamSynchronize(c->stream);
    cudaEventDestroy(c->ev0); cudaEventDestroy(c->ev1);
    for (auto &t : c->pass)
        for (auto &e : t.ev) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    cudaStreamSynchronize(c->xstream);
    cudaStreamDestroy(c->xstream);
    cudaEventDestroy(c->ev_obs);
    cudaEventDestroy(c->ev_tail);
    cudaStreamDestroy(c->stream);
    delete c;
    return FWI_OK;
}

// ---------------------------------------------------------------- model / shots
static int set_model_common(fwi_ctx *c, int nz, int nx, float dx, float dz, float dt, int nt, int pml, int fs)
{
    if (nz <= 0 || nx <= 0 || nt <= 0 || pml < 0 || !(dx > 0) || !(dz > 0) || !(dt > 0))
        return fail(FWI_ERR_ARG, "invalid grid: nz=%d nx=%d nt=%d pml=%d dx=%g dz=%g dt=%g", nz, nx, nt, pml, dx, dz, dt);
    if (fs && pml < 3) return fail(FWI_ERR_ARG, "a free surface needs pmlThick >= 3 (got %d)", pml);
    bool same = nz == c->nz && nx == c->nx && nt == c->nt && pml == c->pml && fs == c->fs && dx == c->dx &&
                dz == c->dz && dt == c->dt;
    if (!same) {
        free_runs(c);
        for (auto &kv : c->progs) dfree(c, kv.second.d);
        c->progs.clear();
        for (auto &p : c->plans) {
            dfree(c, p->d_coef);
            fwi_free_coefs(&p->hc);
        }
        c->plans.clear();
        dfree(c, c->d_vp, 0); dfree(c, c->d_rho, 0);
        dfree(c, c->d_grad, 0); dfree(c, c->d_prec, 0); dfree(c, c->d_gc, 0);
        c->d_vp = c->d_rho = c->d_grad = c->d_prec = nullptr;
        c->d_gc = c->d_hc = nullptr;
        size_t m = (size_t)nz * nx;
        TRY(dmalloc(c, (void **)&c->d_vp, m * 4));
        TRY(dmalloc(c, (void **)&c->d_rho, m * 4));
        TRY(dmalloc(c, (void **)&c->d_grad, m * 4));
        TRY(dmalloc(c, (void **)&c->d_prec, m * 4));
        TRY(dmalloc(c, (void **)&c->d_gc, 2 * m * 8));  // FP64 stacks of g and H, one block for the exchange
        c->d_hc = c->d_gc + m;
    }
    c->nz = nz; c->nx = nx; c->nt = nt; c->pml = pml; c->fs = fs;
    c->dx = dx; c->dz = dz; c->dt = dt;
    c->version++;
    return FWI_OK;
}

extern "C" int fwi_ctx_set_model(fwi_ctx *c, const float *vp, const float *rho, int nz, int nx, float dx, float dz,
                                 float dt, int nt, int pml, int fs)
{
    if (!c || !vp || !rho) return fail(FWI_ERR_ARG, "NULL argument to fwi_ctx_set_model");
    CK(cudaSetDevice(c->device));
    TRY(set_model_common(c, nz, nx, dx, dz, dt, nt, pml, fs));
    size_t m = (size_t)nz * nx;
    for (size_t i = 0; i < m; i++)
        if (!(vp[i] > 0.0f) || !(rho[i] > 0.0f)) return fail(FWI_ERR_ARG, "vp and rho must be positive (cell %zu)", i);
    c->vp.assign(vp, vp + m);
    c->rho.assign(rho, rho + m);
    c->host_model_valid = true;
    CK(cudaMemcpyAsync(c->d_vp, vp, m * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_rho, rho, m * 4, cudaMemcpyHostToDevice, c->stream));
    return FWI_OK;
}

extern "C" int fwi_ctx_set_model_device(fwi_ctx *c, const float *d_vp, const float *d_rho, int nz, int nx, float dx,
                                        float dz, float dt, int nt, int pml, int fs)
{
    if (!c || !d_vp || !d_rho) return fail(FWI_ERR_ARG, "NULL argument to fwi_ctx_set_model_device");
    CK(cudaSetDevice(c->device));
    TRY(set_model_common(c, nz, nx, dx, dz, dt, nt, pml, fs));
    size_t m = (size_t)nz * nx;
    CK(cudaMemcpyAsync(c->d_vp, d_vp, m * 4, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_rho, d_rho, m * 4, cudaMemcpyDeviceToDevice, c->stream));
    // the coefficient set-up runs on the host with the C library's libm: bring the model over
    c->vp.resize(m);
    c->rho.resize(m);
    CK(cudaMemcpyAsync(c->vp.data(), c->d_vp, m * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->rho.data(), c->d_rho, m * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->host_model_valid = true;
    return FWI_OK;
}

static bool in_fd_range(int x, int z, int nz, int nxx, int pml, int fs)
{
    int X = x + pml, Z = z + pml, Nx = nxx + 2 * pml, Nz = nz + 2 * pml;
    int z0 = fs ? pml : 3;
    return x >= 0 && x < nxx && z >= 0 && z < nz && X >= 3 && X <= Nx - 4 && Z >= z0 && Z <= Nz - 4;
}

extern "C" int fwi_ctx_set_shots(fwi_ctx *c, const fwi_shot *shots, int nshot)
{
    if (!c || (!shots && nshot > 0) || nshot < 0) return fail(FWI_ERR_ARG, "invalid shots");
    if (c->nz <= 0) return fail(FWI_ERR_STATE, "set the model before the shots");
    CK(cudaSetDevice(c->device));
    for (int i = 0; i < nshot; i++) {
        const fwi_shot &s = shots[i];
        int nxx = s.ix_max - s.ix_min + 1;
        if (s.ix_min < 0 || s.ix_max >= c->nx || nxx <= 0) return fail(FWI_ERR_ARG, "shot %d: bad window [%d,%d]", i, s.ix_min, s.ix_max);
        if (s.ntr <= 0 || s.ns <= 0 || s.sampleRate <= 0 || !s.src || !s.igx || !s.igz)
            return fail(FWI_ERR_ARG, "shot %d: ntr=%d ns=%d sampleRate=%d", i, s.ntr, s.ns, s.sampleRate);
        // the step kernel's receiver tables encode a trace index in 23 bits
        if (s.ntr >= (1 << 23)) return fail(FWI_ERR_ARG, "shot %d: %d receivers (at most %d)", i, s.ntr, (1 << 23) - 1);
        if ((c->nt - 1) / s.sampleRate + 1 > s.ns) return fail(FWI_ERR_ARG, "shot %d: ns=%d too short for nt=%d", i, s.ns, c->nt);
        if (!in_fd_range(s.isx, s.isz, c->nz, nxx, c->pml, c->fs))
            return fail(FWI_ERR_ARG, "shot %d: source (%d,%d) outside the updated grid", i, s.isx, s.isz);
        for (int r = 0; r < s.ntr; r++)
            if (!in_fd_range(s.igx[r], s.igz[r], c->nz, nxx, c->pml, c->fs))
                return fail(FWI_ERR_ARG, "shot %d: receiver %d (%d,%d) outside the updated grid", i, r, s.igx[r], s.igz[r]);
    }
    TRY(obs_join(c));
    free_runs(c);
    for (float *p : c->d_obs) dfree(c, p, 0);
    for (float *p : c->d_pre) dfree(c, p, 0);
    for (float *p : c->d_pre_alt) dfree(c, p, 0);
    c->d_obs.clear();
    c->d_pre.clear();
    c->d_pre_alt.clear();
    c->shots.clear();
    for (int i = 0; i < nshot; i++) {
        ShotHost h;
        h.s = shots[i];
        h.src.assign(shots[i].src, shots[i].src + c->nt);
        h.igx.assign(shots[i].igx, shots[i].igx + shots[i].ntr);
        h.igz.assign(shots[i].igz, shots[i].igz + shots[i].ntr);
        h.s.src = h.src.data();
        h.s.igx = h.igx.data();
        h.s.igz = h.igz.data();
        c->shots.push_back(std::move(h));
        float *o = nullptr, *p = nullptr;
        size_t nb = (size_t)shots[i].ntr * shots[i].ns * 4;
        TRY(dmalloc(c, (void **)&o, nb));
        TRY(dmalloc(c, (void **)&p, nb));
        CK(cudaMemsetAsync(o, 0, nb, c->stream));
        CK(cudaMemsetAsync(p, 0, nb, c->stream));
        c->d_obs.push_back(o);
        c->d_pre.push_back(p);
        float *a = nullptr;
        TRY(dmalloc(c, (void **)&a, nb));
        CK(cudaMemsetAsync(a, 0, nb, c->stream));
        c->d_pre_alt.push_back(a);
    }
    return FWI_OK;
}

extern "C" int fwi_ctx_set_observed(fwi_ctx *c, const float *const *obs)
{
    if (!c || !obs) return fail(FWI_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(c->device));
    for (size_t i = 0; i < c->shots.size(); i++)
        if (!obs[i]) return fail(FWI_ERR_ARG, "observed gather %zu is NULL", i);
    // after everything issued so far (a run still reading the previous gathers), beside what
    // comes next: the residual waits for the copies (gather)
    CK(cudaEventRecord(c->ev_tail, c->stream));
    CK(cudaStreamWaitEvent(c->xstream, c->ev_tail, 0));
    for (size_t i = 0; i < c->shots.size(); i++)
        CK(cudaMemcpyAsync(c->d_obs[i], obs[i], (size_t)c->shots[i].s.ntr * c->shots[i].s.ns * 4,
                           cudaMemcpyHostToDevice, c->xstream));
    CK(cudaEventRecord(c->ev_obs, c->xstream));
    c->obs_pending = true;
    return FWI_OK;
}

// ---------------------------------------------------------------- plans
static int get_plan(fwi_ctx *c, const fwi_shot &s, Plan **out)
{
    Plan *p = nullptr;
    for (auto &q : c->plans)
        if (q->ix_min == s.ix_min && q->ix_max == s.ix_max && q->fpeak == s.fpeak) p = q.get();
    if (!p) {
        c->plans.emplace_back(new Plan());
        p = c->plans.back().get();
        p->ix_min = s.ix_min;
        p->ix_max = s.ix_max;
        p->fpeak = s.fpeak;
    }
    if (p->version != c->version) {
        if (!c->host_model_valid) return fail(FWI_ERR_STATE, "model not set");
        int nxx = s.ix_max - s.ix_min + 1;
        fwi_coefs nc;
        if (fwi_setup_coefs(c->vp.data() + (size_t)s.ix_min * c->nz, c->rho.data() + (size_t)s.ix_min * c->nz, c->nz,
                            nxx, c->pml, c->dx, c->dz, c->dt, s.fpeak, &nc))
            return fail(FWI_ERR_NOMEM, "host allocation failed in the coefficient set-up");
        size_t fr = (size_t)nc.Nx * nc.ld;
        if (!p->d_coef || p->Nx != nc.Nx || p->ld != nc.ld) {
            dfree(c, p->d_coef, 0);
            p->d_coef = nullptr;
            TRY(dmalloc(c, (void **)&p->d_coef, 6 * fr * 4));
        }
        fwi_free_coefs(&p->hc);
        p->hc = nc;
        p->Nx = nc.Nx; p->Nz = nc.Nz; p->ld = nc.ld; p->G = nc.ld / 4;
        const float *src[6] = {nc.c1, nc.c2, nc.ck, nc.irx, nc.irz, nc.ir};
        for (int k = 0; k < 6; k++)
            CK(cudaMemcpyAsync(p->d_coef + k * fr, src[k], fr * 4, cudaMemcpyHostToDevice, c->stream));
        // the host copy must outlive the asynchronous upload
        CK(cudaStreamSynchronize(c->stream));
        p->version = c->version;
    }
    *out = p;
    return FWI_OK;
}

// ---------------------------------------------------------------- per-shot state
static int ralloc(fwi_ctx *c, ShotRun *r, void **p, size_t bytes)
{
    TRY(dmalloc(c, p, bytes));
    r->allocs.push_back(*p);
    return FWI_OK;
}

// ---------------------------------------------------------------- TMA descriptors
// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// float tensor map of rank 3 or 4: dims[0] contiguous (z), then x, frames or planes, shots;
// out-of-range elements of a box read as zero
static int encode_map(CUtensorMap *m, const float *base, int rank, const long long *dims, const int *box)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return fail(FWI_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t gd[4], gs[3];
    cuuint32_t bx[4], es[4] = {1, 1, 1, 1};
    unsigned long long stride = 4;
    for (int i = 0; i < rank; i++) {
        gd[i] = (cuuint64_t)dims[i];
        bx[i] = (cuuint32_t)box[i];
        if (i > 0) gs[i - 1] = stride;
        stride *= (unsigned long long)dims[i];
    }
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, (void *)base, gd, gs, bx, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(FWI_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return FWI_OK;
}

// the three maps of a launch over nshot consecutive frame blocks starting at d0's
template <int TX>
static int encode_group_maps(const ShotDesc &d0, int nshot, const float *coef, CUtensorMap *p1, CUtensorMap *p0,
                             CUtensorMap *cf)
{
    using Geo = TileGeom<TX>;
    const long long pd[4] = {d0.ld, d0.Nx, d0.nfr, nshot}, cd[3] = {d0.ld, d0.Nx, 6};
    const int b1[4] = {Geo::ZP, Geo::XP, 1, 1}, b0[4] = {Geo::ZC, TX, 1, 1}, bc[3] = {Geo::ZC, TX, 6};
    TRY(encode_map(p1, d0.frames, 4, pd, b1));
    TRY(encode_map(p0, d0.frames, 4, pd, b0));
    TRY(encode_map(cf, coef, 3, cd, bc));
    return FWI_OK;
}

// the three maps of the two-step kernel: u(t) with a two-radius halo, u(t-1) and the
// coefficients on the tile grown by one radius
template <int TX>
static int encode_group_maps2(const ShotDesc &d0, int nshot, const float *coef, CUtensorMap *ma, CUtensorMap *mb,
                              CUtensorMap *cf)
{
    using Geo = Tile2Geom<TX>;
    const long long pd[4] = {d0.ld, d0.Nx, d0.nfr, nshot}, cd[3] = {d0.ld, d0.Nx, 6};
    const int ba[4] = {4 * Geo::AG, Geo::AX, 1, 1}, bb[4] = {4 * Geo::CG, Geo::CX, 1, 1}, bc[3] = {4 * Geo::CG, Geo::CX, 6};
    TRY(encode_map(ma, d0.frames, 4, pd, ba));
    TRY(encode_map(mb, d0.frames, 4, pd, bb));
    TRY(encode_map(cf, coef, 3, cd, bc));
    return FWI_OK;
}

// frame blocks of a group of runs, consecutive in one pool; a new pool or a new layout
// invalidates the captured launches (their tensor maps hold the old one)
static int assign_pool(fwi_ctx *c, int key, const std::vector<ShotRun *> &rs)
{
    const ShotDesc &d0 = rs[0]->d;
    const int ng = (int)rs.size();
    const size_t per = (size_t)d0.nfr * (size_t)d0.frame;
    const size_t need = per * ng * 4;
    fwi_ctx::Pool &pl = c->pools[key];
    if (pl.bytes < need || pl.nfr != d0.nfr || pl.ng != ng || pl.frame != d0.frame) {
        drop_graphs(c);
        if (pl.bytes < need) {
            dfree(c, pl.p, pl.bytes);
            pl.p = nullptr;
            pl.bytes = 0;
            TRY(dmalloc(c, (void **)&pl.p, need));
            pl.bytes = need;
        }
        pl.nfr = d0.nfr;
        pl.ng = ng;
        pl.frame = d0.frame;
    }
    for (int i = 0; i < ng; i++) {
        if (rs[i]->d.nfr != d0.nfr || rs[i]->d.frame != d0.frame)
            return fail(FWI_ERR_STATE, "shots of one group differ in frame layout");
        rs[i]->d.frames = pl.p + per * i;
    }
    return FWI_OK;
}

// fill the geometry/coefficients part of a descriptor; allocate what the run needs
static int prepare_run(fwi_ctx *c, ShotRun *r, int shot, bool gradient)
{
    const ShotHost &sh = c->shots[shot];
    const fwi_shot &s = sh.s;
    Plan *p = nullptr;
    TRY(get_plan(c, s, &p));
    const bool same_geom = r->plan && r->plan->Nx == p->Nx && r->plan->ld == p->ld && r->shot >= 0 &&
                           c->shots[r->shot].s.ntr == s.ntr && c->shots[r->shot].s.ns == s.ns;
    const bool realloc = !same_geom || (gradient && !r->has_ck) || r->allocs.empty();
    if (realloc) {
        free_run(c, r);
        r->has_ck = false;
    }
    r->shot = shot;
    r->plan = p;
    ShotDesc &d = r->d;
    const fwi_coefs &hc = p->hc;
    d.Nx = p->Nx; d.Nz = p->Nz; d.ld = p->ld; d.G = p->G; d.pml = c->pml;
    d.nz = c->nz; d.nxx = s.ix_max - s.ix_min + 1; d.fs = c->fs; d.izStart = c->fs ? c->pml : 3;
    d.nt = c->nt; d.d = fwi_ck_interval(c->nt); d.K = (c->nt - 1) / d.d;
    d.ns = s.ns; d.sr = s.sampleRate; d.ntr = s.ntr;
    d.S5 = d.d / MST + 2;
    d.isx = s.isx + c->pml; d.isz = s.isz + c->pml;
    d.invdx = hc.invdx; d.invdz = hc.invdz; d.invdxdx = hc.invdxdx; d.invdzdz = hc.invdzdz;
    d.negzero = -0.0f;
    d.invdtdt = hc.invdtdt; d.dt = c->dt;
    const size_t fr = p->frame();
    d.frame = (long long)fr;
    d.c1 = p->d_coef; d.c2 = p->d_coef + fr; d.ck = p->d_coef + 2 * fr;
    d.irx = p->d_coef + 3 * fr; d.irz = p->d_coef + 4 * fr; d.ir = p->d_coef + 5 * fr;
    const int nt = c->nt, ntr = s.ntr;
    if (realloc) {
        void *q;
        TRY(ralloc(c, r, &q, (size_t)nt * 8)); d.srcd = (double *)q;
        TRY(ralloc(c, r, &q, (size_t)nt * 4)); d.srcf = (float *)q;
        TRY(ralloc(c, r, &q, (size_t)(d.Nx + 1) * 4)); d.colptr = (int *)q;
        TRY(ralloc(c, r, &q, (size_t)ntr * 8)); d.rec = (int2 *)q;
        TRY(ralloc(c, r, &q, (size_t)ntr * 4)); d.recK = (float *)q;
        TRY(ralloc(c, r, &q, (size_t)ntr * 4)); d.rec_off = (int *)q;
        TRY(ralloc(c, r, &q, (size_t)s.ns * ntr * 4)); d.traces_t = (float *)q;
        d.nfr = gradient ? nframes_gradient(d.K, d.S5) : NROT;
        d.frames = nullptr;  // in the group's pool (assign_pool)
        d.H = d.Gacc = nullptr;
        d.adj_t = nullptr;
        if (gradient) {
            TRY(ralloc(c, r, &q, fr * 8)); d.H = (double *)q;
            TRY(ralloc(c, r, &q, fr * 8)); d.Gacc = (double *)q;
            TRY(ralloc(c, r, &q, (size_t)nt * ntr * 4)); d.adj_t = (float *)q;
            size_t m = (size_t)c->nz * d.nxx;
            TRY(ralloc(c, r, &q, m * 4)); r->d_gshot = (float *)q;
            TRY(ralloc(c, r, &q, m * 4)); r->d_hshot = (float *)q;
            TRY(ralloc(c, r, &q, (size_t)(s.ns + 1) * 4)); r->d_tct = (float *)q;
            TRY(ralloc(c, r, &q, (size_t)(ntr + 1) * 4)); r->d_tcr = (float *)q;
            r->has_ck = true;
        } else {
            void *q2;
            TRY(ralloc(c, r, &q2, (size_t)(s.ns + 1) * 4)); r->d_tct = (float *)q2;
            TRY(ralloc(c, r, &q2, (size_t)(ntr + 1) * 4)); r->d_tcr = (float *)q2;
        }
    }
    d.hessian = 0;
    d.snap = c->dump.verbose > 1 ? c->dump.snap_interval : 0;
    // per-step source terms in the reference's precision (propagation.c:558 double, :662 float)
    const float Ks = hc.K[(size_t)d.isx * d.ld + d.isz];
    std::vector<double> sd(nt);
    std::vector<float> sf(nt);
    for (int it = 0; it < nt; it++) {
        sd[it] = fwi_src_term_f64(sh.src[it], Ks, c->dt, hc.invdx, hc.invdz);
        sf[it] = fwi_src_term_f32(sh.src[it], Ks, c->dt, hc.invdx, hc.invdz);
    }
    // receivers as per-column lists sorted by (x, z, trace): duplicates stay in trace order
    std::vector<int> order(ntr);
    for (int i = 0; i < ntr; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        if (sh.igx[a] != sh.igx[b]) return sh.igx[a] < sh.igx[b];
        return sh.igz[a] < sh.igz[b];
    });
    std::vector<int> colptr(d.Nx + 1, 0);
    std::vector<int2> rec(ntr);
    std::vector<float> recK(ntr);
    std::vector<int> rec_off(ntr);
    for (int i = 0; i < ntr; i++) rec_off[i] = (sh.igx[i] + c->pml) * d.ld + sh.igz[i] + c->pml;
    for (int e = 0; e < ntr; e++) {
        int i = order[e];
        int X = sh.igx[i] + c->pml, Z = sh.igz[i] + c->pml;
        rec[e] = make_int2(Z, i);
        recK[e] = hc.K[(size_t)X * d.ld + Z];
        colptr[X + 1]++;
    }
    for (int x = 0; x < d.Nx; x++) colptr[x + 1] += colptr[x];
    d.rz0 = 1 << 30;
    d.rz1 = -1;
    for (int i = 0; i < ntr; i++) {
        d.rz0 = std::min(d.rz0, sh.igz[i] + c->pml);
        d.rz1 = std::max(d.rz1, sh.igz[i] + c->pml);
    }
    CK(cudaMemcpyAsync((void *)d.srcd, sd.data(), nt * 8, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync((void *)d.srcf, sf.data(), nt * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync((void *)d.colptr, colptr.data(), (d.Nx + 1) * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync((void *)d.rec, rec.data(), ntr * 8, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync((void *)d.recK, recK.data(), ntr * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync((void *)d.rec_off, rec_off.data(), ntr * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));  // host staging vectors go out of scope
    return FWI_OK;
}

// taper lengths of compute_adjoint_source2d (optimization.c:347-365) and the taper_traces caps
static int prepare_taper(fwi_ctx *c, ShotRun *r, float freq)
{
    const fwi_shot &s = c->shots[r->shot].s;
    double vp_sum = 0.0;
    for (int i = 0; i < s.ntr; i++)  // window-local igx into the global model, as the reference does
        vp_sum += c->vp[(size_t)s.igx[i] * c->nz + s.igz[i]];
    float vp_avg = (float)(vp_sum / s.ntr);
    if (freq == 0.0f) freq = s.fpeak;
    float kpass = freq / vp_avg;
    int Lt = (int)roundf((2.0f / freq) / s.dt) + 1;
    int Lr = (int)roundf((2.0f / kpass) / s.dtr) + 1;
    if (Lt > 0 && Lt > s.ns / 3) Lt = s.ns / 3;
    if (Lr > 0 && Lr > s.ntr / 3) Lr = s.ntr / 3;
    if (Lt < 0) Lt = 0;
    if (Lr < 0) Lr = 0;
    r->Lt = Lt;
    r->Lr = Lr;
    r->fpass = freq;
    r->kpass = kpass;
    std::vector<float> a(Lt + 1), b(Lr + 1);
    if (Lt > 0) fwi_taper_coefs(Lt, a.data());
    if (Lr > 0) fwi_taper_coefs(Lr, b.data());
    // pageable sources: staged before the calls return
    CK(cudaMemcpyAsync(r->d_tct, a.data(), (Lt + 1) * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(r->d_tcr, b.data(), (Lr + 1) * 4, cudaMemcpyHostToDevice, c->stream));
    return FWI_OK;
}

// ---------------------------------------------------------------- programs
static bool is_stored(int t, int nt, int d) { return t % d == 0 || ((t + 1) % d == 0 && t + 1 < nt); }

static std::vector<int4> program_forward(int nt, int kind)
{
    std::vector<int4> p(nt);
    for (int it = 0; it < nt; it++) p[it] = make_int4(kind, it, K_NONE, 0);
    return p;
}

// adjoint pass: replay segments and adjoint steps.  Without overlap this is the
// reference's order (replay a whole segment when the reverse loop reaches its top,
// propagation.c:641-673).  With overlap the replay of segment k-1 runs in the same
// launches as the adjoint steps of segment k; segments alternate between two frame
// buffers, so segment k may start once the adjoint no longer needs segment k+2.
static std::vector<int4> program_adjoint(int nt, bool overlap)
{
    const int d = fwi_ck_interval(nt), K = (nt - 1) / d;
    auto top_of = [&](int k) { return k == K ? nt - 1 : k * d + d - 2; };
    std::vector<int4> prog;
    if (!overlap) {
        for (int it = nt - 1; it >= 0; --it) {
            if (!is_stored(it, nt, d)) {
                int k = it / d, c = k * d;
                if (it == top_of(k))
                    for (int itt = c; itt < it; ++itt) prog.push_back(make_int4(K_REP, itt, K_NONE, 0));
            }
            prog.push_back(make_int4(K_ADJ, it, K_NONE, 0));
        }
        return prog;
    }
    std::deque<int2> rq;
    std::vector<int> need(K + 1, 0), done(K + 1, 0);
    for (int k = K; k >= 0; --k) {
        int c = k * d, top = top_of(k);
        for (int itt = c; itt < top; ++itt) rq.push_back(make_int2(k, itt));
        need[k] = std::max(0, top - c);
    }
    int a = nt - 1;
    while (!rq.empty() || a >= 0) {
        int4 item = make_int4(K_NONE, 0, K_NONE, 0);
        int rep_k = -1;
        if (!rq.empty()) {
            int k = rq.front().x;
            bool ok = (k + 2 > K) || (a <= (k + 2) * d);
            if (ok) {
                item.x = K_REP;
                item.y = rq.front().y;
                rep_k = k;
                rq.pop_front();
            }
        }
        if (a >= 0) {
            bool ok = is_stored(a, nt, d) || done[a / d] >= need[a / d];
            if (ok) {
                item.z = K_ADJ;
                item.w = a;
                --a;
            }
        }
        if (rep_k >= 0) done[rep_k]++;
        prog.push_back(item);
    }
    return prog;
}

// Programs of the two-step kernel (fwi_tile2.cuh): an item flagged K_DEPTH2 advances two
// consecutive steps of its kind.  Forward: pairs (0, 1), (2, 3), ... and a last single step when
// nt is odd.
static std::vector<int4> program_forward2(int nt, int kind)
{
    std::vector<int4> p;
    for (int it = 0; it < nt; it += 2) p.push_back(make_int4(it + 1 < nt ? kind | K_DEPTH2 : kind, it, K_NONE, 0));
    return p;
}

// Adjoint pass of the two-step kernel: the overlapped schedule of program_adjoint with up to two
// replay steps (consecutive, one segment) and up to two adjoint steps (it, it - 1) per launch.  A
// replay step may run once the adjoint no longer needs the kept frames its segment overwrites;
// an adjoint step once its imaging step's segment was replayed in an earlier launch.
static std::vector<int4> program_adjoint2(int nt)
{
    const int d = fwi_ck_interval(nt), K = (nt - 1) / d;
    auto top_of = [&](int k) { return k == K ? nt - 1 : k * d + d - 2; };
    std::deque<int2> rq;
    std::vector<int> need(K + 1, 0), done(K + 1, 0);
    for (int k = K; k >= 0; --k) {
        int cc = k * d, top = top_of(k);
        for (int itt = cc; itt < top; ++itt) rq.push_back(make_int2(k, itt));
        need[k] = std::max(0, top - cc);
    }
    std::vector<int4> prog;
    int a = nt - 1;
    while (!rq.empty() || a >= 0) {
        int4 item = make_int4(K_NONE, 0, K_NONE, 0);
        int nrep = 0, rep_k = -1, rep0 = 0;
        while (nrep < 2 && !rq.empty()) {
            const int k = rq.front().x, itt = rq.front().y;
            if (nrep && (k != rep_k || itt != rep0 + 1)) break;
            if (!((k + 2 > K) || (a <= (k + 2) * d))) break;
            if (!nrep) rep0 = itt;
            rep_k = k;
            rq.pop_front();
            ++nrep;
        }
        int nadj = 0, adj0 = a;
        while (nadj < 2 && a >= 0 && (is_stored(a, nt, d) || done[a / d] >= need[a / d])) {
            --a;
            ++nadj;
        }
        if (nrep) item.x = nrep == 2 ? K_REP | K_DEPTH2 : K_REP, item.y = rep0;
        if (nadj) item.z = nadj == 2 ? K_ADJ | K_DEPTH2 : K_ADJ, item.w = adj0;
        if (rep_k >= 0) done[rep_k] += nrep;
        prog.push_back(item);
    }
    return prog;
}

static int get_program(fwi_ctx *c, const std::string &key, const std::vector<int4> &items, Program **out)
{
    auto it = c->progs.find(key);
    if (it == c->progs.end()) {
        Program p;
        p.items = items;
        for (const int4 &w : items)
            if ((w.x & K_DEPTH2) || (w.z & K_DEPTH2)) p.depth = 2;
        TRY(dmalloc(c, (void **)&p.d, items.size() * sizeof(int4)));
        CK(cudaMemcpy(p.d, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
        it = c->progs.emplace(key, std::move(p)).first;
    }
    *out = &it->second;
    return FWI_OK;
}

// ---------------------------------------------------------------- launching
typedef void (*StepFn)(const ShotDesc *, const int4 *, int, int, int);

template <int S, int MATH>
static StepFn step_fn(int tx)
{
    StepFn f;
    switch (tx) {
    case 8: f = k_step<8, S, MATH>; break;
    default: f = k_step<16, S, MATH>; break;
    }
    // the tiles live in shared memory: prefer the largest carve-out so more blocks fit per SM
    cudaFuncSetAttribute((const void *)f, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    return f;
}

// launch shape: tiles of 16 z-groups x TX columns, S shots per block sharing one coefficient load
struct LaunchCfg {
    int tx, S, math;
    StepFn fn;
};
static LaunchCfg pick_launch(int Nx, int nshot, bool batched, int math)
{
    LaunchCfg L;
    L.tx = batched ? 16 : 8;
    L.S = (batched && nshot >= 2) ? 2 : 1;
    L.math = math;
    (void)Nx;
    if (const char *e = getenv("FWI_TX")) L.tx = atoi(e);
    if (const char *e = getenv("FWI_S")) L.S = atoi(e);
    if (L.tx != 8) L.tx = 16;
    if (L.S != 1) L.S = 2;
    if (L.S == 1) L.fn = L.math ? step_fn<1, 1>(L.tx) : step_fn<1, 0>(L.tx);
    else L.fn = L.math ? step_fn<2, 1>(L.tx) : step_fn<2, 0>(L.tx);
    return L;
}

typedef void (*TileFn)(const CUtensorMap, const CUtensorMap, const CUtensorMap, const ShotDesc *, const int4 *, int,
                       int, int, int, int, int *, const TileSync);

template <int TX, int NST, int MATH, int GPT, int MINB>
static TileFn tile_fn()
{
    static bool ready = false;
    TileFn f;
    if constexpr (MINB == 3) f = k_tile3<TX, NST, MATH>;
    else f = k_tile<TX, NST, MATH, GPT>;
    if (!ready) {
        cudaFuncSetAttribute((const void *)f, cudaFuncAttributeMaxDynamicSharedMemorySize, TileGeom<TX>::smem(NST));
        cudaFuncSetAttribute((const void *)f, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        ready = true;
    }
    return f;
}

template <int TX, int MATH, int GPT, int MINB>
static TileFn tile_fn_nst(int nst)
{
    return nst == 2   ? tile_fn<TX, 2, MATH, GPT, MINB>()
           : nst == 4 ? tile_fn<TX, 4, MATH, GPT, MINB>()
                      : tile_fn<TX, 3, MATH, GPT, MINB>();
}

// MINB 3 (coefficients from shared memory, three blocks per SM) exists for 16-column tiles with
// one group per thread, the shape that register use limits to two blocks
template <int TX, int MATH>
static TileFn tile_fn_gpt(int nst, int gpt, int minb)
{
    if (gpt == 2) return tile_fn_nst<TX, MATH, 2, 1>(nst);
    if (TX == 16 && minb == 3) return tile_fn_nst<TX, MATH, 1, TX == 16 ? 3 : 1>(nst);
    return tile_fn_nst<TX, MATH, 1, 1>(nst);
}

// shots per block: split the group into equal chunks (at most 12 shots each, the measured
// best for 60-shot groups) and take the fewest chunks whose grid fills its last wave of
// resident blocks about as well as the best split does
static int pick_chunk(int tiles, int nshot, int resident)
{
    const int cap = 12;
    const int slots = 148 * resident;
    auto fill = [&](int nch) {
        const long long blocks = (long long)tiles * nch;
        const long long waves = (blocks + slots - 1) / slots;
        return (double)blocks / (double)(waves * slots);
    };
    const int nmin = (nshot + cap - 1) / cap;
    double best = 0.0;
    for (int nch = nmin; nch <= nshot; nch++) best = std::max(best, fill(nch));
    for (int nch = nmin; nch <= nshot; nch++)
        if (fill(nch) >= 0.9 * best) return (nshot + nch - 1) / nch;
    return 1;
}

static int check_kernel_error(fwi_ctx *c);
static int snapshots_after(fwi_ctx *c, const Program *prog, int L, int shot_base, int nshot);

// ---------------------------------------------------------------- tile configuration and autotuner
// A launch shape of the step kernel: tile width (8 or 16 columns), depth of the shared-memory
// ring (2..4 shots in flight) and shots per block (the chunk).
struct TileCfg {
    int tx = 16, nst = 4, chunk = 1, gpt = 1;  // gpt: z-groups per consumer thread (1 or 2)
    int minb = 1;                              // 3: the three-blocks-per-SM variant (tx 16, gpt 1)
};

typedef void (*Tile2Fn)(const CUtensorMap, const CUtensorMap, const CUtensorMap, const ShotDesc *, const int4 *, int,
                        int, int, int, int *);

template <int NST, int MATH>
static Tile2Fn tile2_fn()
{
    static bool ready = false;
    Tile2Fn f = k_tile2<16, NST, MATH>;
    if (!ready) {
        cudaFuncSetAttribute((const void *)f, cudaFuncAttributeMaxDynamicSharedMemorySize, Tile2Geom<16>::smem(NST));
        cudaFuncSetAttribute((const void *)f, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        ready = true;
    }
    return f;
}

// launches of a two-step program: 16-column tiles, ring depth 2 or 3, the shape's chunk
static int launch_tiles2(fwi_ctx *c, const Program *prog, int L0, int L1, int shot_base, int nshot, const ShotRun *r0,
                         const TileCfg &cfg)
{
    const Plan *p = r0->plan;
    const int zt = (p->G + TG - 1) / TG, tx = 16;
    const int nst = cfg.nst >= 3 ? 3 : 2, chunk = cfg.chunk;
    Tile2Fn fn = c->math ? (nst == 3 ? tile2_fn<3, 1>() : tile2_fn<2, 1>()) : (nst == 3 ? tile2_fn<3, 0>() : tile2_fn<2, 0>());
    const int ntx = (p->Nx + tx - 1) / tx, nchunks = (nshot + chunk - 1) / chunk;
    CUtensorMap ma, mb, mc;
    TRY(encode_group_maps2<16>(r0->d, nshot, p->d_coef, &ma, &mb, &mc));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(ntx, 2 * nchunks, zt);
    lc.blockDim = dim3(TG, tx + 32 / TG);
    lc.dynamicSmemBytes = Tile2Geom<16>::smem(nst);
    lc.stream = c->stream;
    lc.attrs = attr;
    lc.numAttrs = c->pdl ? 1 : 0;
    for (int L = L0; L < L1; L++) {
        const int4 &pw = prog->items[L];
        if (pw.x == K_NONE && pw.z == K_NONE) continue;
        CK(cudaLaunchKernelEx(&lc, fn, ma, mb, mc, (const ShotDesc *)c->d_desc, (const int4 *)prog->d, L, shot_base,
                              nshot, chunk, c->d_err));
        c->launches++;
    }
    CK(cudaGetLastError());
    return FWI_OK;
}

static int launch_tiles(fwi_ctx *c, const Program *prog, int L0, int L1, int shot_base, int nshot, const ShotRun *r0,
                        const TileCfg &cfg)
{
    if (prog->depth == 2) return launch_tiles2(c, prog, L0, L1, shot_base, nshot, r0, cfg);
    const Plan *p = r0->plan;
    const int zt = (p->G + TG - 1) / TG;
    const int tx = cfg.tx, nst = cfg.nst, chunk = cfg.chunk, gpt = cfg.gpt, nl = TG / gpt;
    const int minb = cfg.minb;
    TileFn fn = tx == 16 ? (c->math ? tile_fn_gpt<16, 1>(nst, gpt, minb) : tile_fn_gpt<16, 0>(nst, gpt, minb))
                         : (c->math ? tile_fn_gpt<8, 1>(nst, gpt, minb) : tile_fn_gpt<8, 0>(nst, gpt, minb));
    const int smem = tx == 16 ? TileGeom<16>::smem(nst) : TileGeom<8>::smem(nst);
    const int ntx = (p->Nx + tx - 1) / tx, nchunks = (nshot + chunk - 1) / chunk;
    // items whose second half is empty throughout (a forward pass) need no blocks for it
    int halves = 1;
    for (int L = L0; L < L1 && halves == 1; L++)
        if (prog->items[L].z != K_NONE) halves = 2;
    // consecutive launches wait for their neighbouring tiles only (TileSync) where the flags fit;
    // a one-shot launch (the plain path) is a few microseconds long, too short for the flags' fences
    // and polls to pay off, and waits for the whole grid before it
    const size_t nflags = (size_t)2 * nchunks * zt * ntx;
    const bool fine = c->fine && nshot >= 2 && nflags <= (size_t)c->tflags_cap;
    dim3 grid(fine ? ntx : ntx + 1, halves * nchunks, zt);
    if (fine) CK(cudaMemsetAsync(c->d_tflags, 0, nflags * sizeof(int), c->stream));
    TileSync ts{fine ? c->d_tflags : nullptr, -1, ntx, zt, halves};
    CUtensorMap m1, m0, mc;
    if (tx == 16) TRY(encode_group_maps<16>(r0->d, nshot, p->d_coef, &m1, &m0, &mc));
    else TRY(encode_group_maps<8>(r0->d, nshot, p->d_coef, &m1, &m0, &mc));
    // each step may launch while the previous one drains: its blocks set up barriers and
    // per-shot scalars, then wait (griddepcontrol.wait) before touching any field
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = grid;
    lc.blockDim = dim3(nl, tx + 32 / nl);
    lc.dynamicSmemBytes = smem;
    lc.stream = c->stream;
    lc.attrs = attr;
    lc.numAttrs = c->pdl ? 1 : 0;
    for (int L = L0; L < L1; L++) {
        const int4 &pw = prog->items[L];
        if (pw.x == K_NONE && pw.z == K_NONE) continue;
        CK(cudaLaunchKernelEx(&lc, fn, m1, m0, mc, (const ShotDesc *)c->d_desc, (const int4 *)prog->d, L, shot_base,
                              nshot, chunk, halves, c->d_err, ts));
        ts.Lprev = L;
        c->launches++;
        if (c->snapping) TRY(snapshots_after(c, prog, L, shot_base, nshot));
    }
    CK(cudaGetLastError());
    return FWI_OK;
}

// the measured best configuration per launch shape, shared by every context of the process
struct TuneKey {
    int Nx, G, nshot, math, batched, depth;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(Nx, G, nshot, math, batched, depth) < std::tie(o.Nx, o.G, o.nshot, o.math, o.batched, o.depth);
    }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TileCfg> g_tune;
static std::map<TuneKey, float> g_tune_ms;  // the best shape's time for the tuner's forward steps

// the heuristic shape, or the tuned one, with the environment's overrides applied last
static TileCfg tile_config(fwi_ctx *c, const Plan *p, int nshot, bool batched, int depth = 1)
{
    TileCfg cfg;
    cfg.tx = batched || depth == 2 ? 16 : 8;
    cfg.nst = depth == 2 ? 2 : 4;
    const int zt = (p->G + TG - 1) / TG;
    cfg.chunk = pick_chunk(((p->Nx + cfg.tx - 1) / cfg.tx) * zt, nshot, cfg.tx == 16 ? 2 : 4);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find({p->Nx, p->G, nshot, c->math, batched ? 1 : 0, depth});
        if (it != g_tune.end()) cfg = it->second;
    }
    if (const char *e = getenv("FWI_TX")) cfg.tx = atoi(e) == 8 ? 8 : 16;
    if (const char *e = getenv("FWI_NST")) cfg.nst = std::min(4, std::max(2, atoi(e)));
    if (const char *e = getenv("FWI_CHUNK")) cfg.chunk = std::min(TILE_CH_MAX, std::max(1, atoi(e)));
    if (const char *e = getenv("FWI_GPT")) cfg.gpt = atoi(e) == 2 ? 2 : 1;
    if (const char *e = getenv("FWI_OCC")) cfg.minb = atoi(e) == 3 ? 3 : 1;
    cfg.chunk = std::min(cfg.chunk, std::max(1, nshot));
    c->last_tx = cfg.tx;
    c->last_nst = cfg.nst;
    c->last_chunk = cfg.chunk;
    c->last_gpt = cfg.gpt;
    c->last_minb = cfg.minb;
    c->last_wave = false;
    return cfg;
}

// Time candidate shapes on this group's own forward scratch frames (forward steps 1..12 of the
// real shots, three warm-up launches first) and keep the fastest for this launch shape.  The
// scratch frames are zeroed again afterwards, which is the state a pass starts from; the
// samples the probe wrote are overwritten by the pass.  Candidates: tile width 8/16, ring
// depth 2..4, and chunks of at most 4/8/12/16/24 shots (split evenly).
static int autotune(fwi_ctx *c, int shot_base, int nshot, const ShotRun *r0, bool batched, int depth = 1)
{
    const Plan *p = r0->plan;
    const TuneKey key{p->Nx, p->G, nshot, c->math, batched ? 1 : 0, depth};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        if (g_tune.count(key)) return FWI_OK;
    }
    const int steps = std::min(12, std::max(2, c->nt - 2));
    std::vector<int4> items;
    if (depth == 2)  // the same steps, two per launch
        for (int it = 1; it + 1 <= steps; it += 2) items.push_back(make_int4(K_FWD0 | K_DEPTH2, it, K_NONE, 0));
    else
        for (int it = 1; it <= steps; it++) items.push_back(make_int4(K_FWD0, it, K_NONE, 0));
    const int launches = (int)items.size();
    Program *prog;
    TRY(get_program(c, (depth == 2 ? "tune2/" : "tune/") + std::to_string(steps), items, &prog));
    std::vector<TileCfg> cands;
    std::set<int> chunks;  // even splits of the shots into blocks of at most 4 .. 24
    for (int cap : {4, 8, 12, 16, 24}) {
        const int nch = (nshot + cap - 1) / cap;
        chunks.insert((nshot + nch - 1) / nch);
    }
    if (depth == 2)  // the two-step kernel: 16-column tiles, ring depth 2 or 3
        for (int nst : {2, 3})
            for (int ch : chunks) {
                if (nshot == 1 && nst != 2) continue;
                TileCfg t;
                t.tx = 16;
                t.nst = nst;
                t.chunk = ch;
                cands.push_back(t);
            }
    else
    for (int gpt : {1, 2})
        for (int tx : {16, 8})
            for (int minb : {1, 3}) {
                if (minb == 3 && (tx != 16 || gpt != 1)) continue;  // k_tile3 exists for this shape only
                for (int nst : {2, 3, 4})
                    for (int ch : chunks) {
                        if (nshot == 1 && nst != 2) continue;  // one shot: the ring depth does not matter
                        TileCfg t;
                        t.tx = tx;
                        t.nst = nst;
                        t.chunk = ch;
                        t.gpt = gpt;
                        t.minb = minb;
                        cands.push_back(t);
                    }
            }
    const long long l0 = c->launches;
    float best_ms = 1e30f;
    TileCfg best;
    cudaEvent_t e0, e1;  // the context's own events time the whole run
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (const TileCfg &t : cands) {
        TRY(launch_tiles(c, prog, 0, std::min(3, launches), shot_base, nshot, r0, t));  // warm-up
        CK(cudaEventRecord(e0, c->stream));
        TRY(launch_tiles(c, prog, 0, launches, shot_base, nshot, r0, t));
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->launches = l0;  // probe launches are not part of the run
    for (int i = 0; i < nshot; i++) {
        const ShotRun *r = c->runs.size() == 1 ? c->runs[0].get() : c->runs[shot_base + i].get();
        CK(cudaMemsetAsync(frame_ptr(r->d, F_FWD), 0, NROT * (size_t)r->d.frame * 4, c->stream));
    }
    TRY(check_kernel_error(c));
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
    g_tune_ms[key] = best_ms;
    return FWI_OK;
}

// Halo depth as a tuned dimension: the first batched run of a shape tunes the one-step and the
// two-step kernel on the same forward steps (the probes run before the pass that writes the
// frames) and the context keeps the faster depth for its passes.  FWI_DEPTH pins the depth, and
// so do the launch-shape overrides, a disabled tuner, snapshots and the comparison kernel.
static int choose_depth(fwi_ctx *c, int shot_base, int nshot, const ShotRun *r0, bool batched)
{
    const char *ke = getenv("FWI_KERNEL");
    if (c->depth_pinned || !batched || !c->tune || c->dump.verbose > 1 || (ke && strcmp(ke, "step") == 0) ||
        getenv("FWI_TX") || getenv("FWI_NST") || getenv("FWI_CHUNK") || getenv("FWI_GPT") || getenv("FWI_OCC"))
        return FWI_OK;
    TRY(autotune(c, shot_base, nshot, r0, batched, 1));
    TRY(autotune(c, shot_base, nshot, r0, batched, 2));
    const Plan *p = r0->plan;
    const TuneKey k1{p->Nx, p->G, nshot, c->math, 1, 1}, k2{p->Nx, p->G, nshot, c->math, 1, 2};
    std::lock_guard<std::mutex> lk(g_tune_mu);
    c->depth = g_tune_ms.count(k2) && g_tune_ms.count(k1) && g_tune_ms[k2] < g_tune_ms[k1] ? 2 : 1;
    return FWI_OK;
}

// ---------------------------------------------------------------- persistent forward launch
// Blocks of k_wave one SM holds at once (the launch is cooperative: every block resident).
template <int NST, int MATH>
static int wave_resident()
{
    static const int nb = [] {
        auto f = k_wave<NST, MATH>;
        const int smem = TileGeom<WAVE_TX>::smem(NST);
        cudaFuncSetAttribute((const void *)f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute((const void *)f, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, TG * (WAVE_TX + 32 / TG), smem) != cudaSuccess) b = 0;
        return b;
    }();
    return nb;
}

static constexpr int WAVE_NST = 4;

// The wavefront launch's shape for items L0 .. L1-1 of a program over nshot shots of one group,
// or false where it does not apply: the items must be consecutive forward steps, the run must
// not write snapshots (the host copies them out between steps), and one block per 16-column
// tile and shot range of 2 to WAVE_CH_MAX shots must fit the resident blocks.
static bool wave_shape(fwi_ctx *c, const Program *prog, int L0, int L1, int nshot, const ShotRun *r0, int *ranges,
                       int *per_range)
{
    const char *ke = getenv("FWI_KERNEL");
    if (!c->wave || c->snapping || prog->depth != 1 || L1 <= L0 || nshot < 2 || (ke && strcmp(ke, "step") == 0))
        return false;
    for (int L = L0; L < L1; L++) {
        const int4 &pw = prog->items[L];
        if ((pw.x != K_FWD0 && pw.x != K_FWD1) || pw.z != K_NONE || pw.y != prog->items[L0].y + (L - L0)) return false;
    }
    const Plan *p = r0->plan;
    const int tiles = ((p->Nx + WAVE_TX - 1) / WAVE_TX) * ((p->G + TG - 1) / TG);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) return false;
    const int slots = sms * (c->math ? wave_resident<WAVE_NST, 1>() : wave_resident<WAVE_NST, 0>());
    if (tiles > slots) return false;
    for (int nr = std::min(slots / tiles, nshot / 2); nr >= 1; --nr) {
        const int n = (nshot + nr - 1) / nr;
        if (n <= WAVE_CH_MAX && nshot - (nr - 1) * n >= 2 && tiles * nr + 1 <= c->wave_cap) {
            *ranges = nr;
            *per_range = n;
            return true;
        }
    }
    return false;
}

// the whole forward program as one launch of k_wave (fwi_wave.cuh)
static int launch_wave(fwi_ctx *c, const Program *prog, int L0, int L1, int shot_base, int nshot, const ShotRun *r0,
                       int nranges, int n)
{
    const Plan *p = r0->plan;
    const int ntx = (p->Nx + WAVE_TX - 1) / WAVE_TX, zt = (p->G + TG - 1) / TG;
    const int blocks = ntx * zt * nranges;
    CUtensorMap m1, m0, mc;
    TRY(encode_group_maps<WAVE_TX>(r0->d, nshot, p->d_coef, &m1, &m0, &mc));
    CK(cudaMemsetAsync(c->d_wave, 0, (size_t)(blocks + 1) * sizeof(int), c->stream));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(blocks);
    lc.blockDim = dim3(TG, WAVE_TX + 32 / TG);
    lc.dynamicSmemBytes = TileGeom<WAVE_TX>::smem(WAVE_NST);
    lc.stream = c->stream;
    lc.attrs = attr;
    lc.numAttrs = 1;
    auto fn = c->math ? k_wave<WAVE_NST, 1> : k_wave<WAVE_NST, 0>;
    CK(cudaLaunchKernelEx(&lc, fn, m1, m0, mc, (const ShotDesc *)c->d_desc, (const int4 *)prog->d, L0, L1, shot_base,
                          nshot, n, ntx, zt, nranges, c->d_wave, c->d_err));
    c->launches++;
    c->last_tx = WAVE_TX;
    c->last_nst = WAVE_NST;
    c->last_chunk = n;
    c->last_gpt = 1;
    c->last_minb = c->math ? wave_resident<WAVE_NST, 1>() : wave_resident<WAVE_NST, 0>();
    c->last_wave = true;
    return FWI_OK;
}

static int launch_steps(fwi_ctx *c, const Program *prog, int shot_base, int nshot, const ShotRun *r0, bool batched)
{
    {
        int nranges = 0, n = 0;
        if (batched && wave_shape(c, prog, 0, (int)prog->items.size(), nshot, r0, &nranges, &n))
            return launch_wave(c, prog, 0, (int)prog->items.size(), shot_base, nshot, r0, nranges, n);
    }
    const Plan *p = r0->plan;
    const int zt = (p->G + TG - 1) / TG;
    const int n = (int)prog->items.size();
    const char *ke = getenv("FWI_KERNEL");  // "step": the cp.async kernel, kept for comparison
    if (ke && strcmp(ke, "step") == 0) {
        LaunchCfg cfg = pick_launch(p->Nx, nshot, batched, c->math);
        const int groups = (nshot + cfg.S - 1) / cfg.S;
        dim3 grid((p->Nx + cfg.tx - 1) / cfg.tx + 1, 2 * groups, zt);
        for (int L = 0; L < n; L++) {
            const int4 &pw = prog->items[L];
            if (pw.x == K_NONE && pw.z == K_NONE) continue;
            cfg.fn<<<grid, dim3(TG, TYX), 0, c->stream>>>(c->d_desc, prog->d, L, shot_base, nshot);
            c->launches++;
        }
        CK(cudaGetLastError());
        return FWI_OK;
    }
    const TileCfg cfg = tile_config(c, p, nshot, batched, prog->depth);
    return launch_tiles(c, prog, 0, n, shot_base, nshot, r0, cfg);
}

// a step kernel that gave up waiting for a tile copy leaves its mark in the error word
static int check_kernel_error(fwi_ctx *c)
{
    int e = 0;
    CK(cudaMemcpy(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        CK(cudaMemset(c->d_err, 0, sizeof(int)));
        return fail(FWI_ERR_CUDA, "step kernel: a tile copy did not complete within 2 s; results are invalid");
    }
    return FWI_OK;
}

// ---------------------------------------------------------------- verbose output
// With verbose > 0 the reference writes intermediate results as raw float32 files (write_bin,
// dataio.c:277-302) into the working directory: per written-out shot of a gradient run the
// predicted traces, the adjoint source and the raw shot gradient, and per gradient the stacked
// gradient and preconditioner (propagation.c:917-944, 996-1005); with verbose > 1 also wavefield
// snapshots every snap_interval steps (propagation.c:597-601, 717-723).  File names and contents
// are the reference's.
static int write_floats(fwi_ctx *c, const char *name, const float *h, size_t n)
{
    const std::string path = c->dump.dir.empty() ? std::string(name) : c->dump.dir + "/" + name;
    FILE *fp = fopen(path.c_str(), "wb");
    if (!fp) return fail(FWI_ERR_ARG, "verbose output: cannot open %s for writing", path.c_str());
    const size_t w = fwrite(h, 4, n, fp);
    const int e = fclose(fp);
    if (w != n || e) return fail(FWI_ERR_ARG, "verbose output: short write to %s", path.c_str());
    return FWI_OK;
}

// n device floats (stream-ordered after the work queued so far) into a file
static int dump_device(fwi_ctx *c, const char *name, const float *dev, size_t n)
{
    std::vector<float> h(n);
    CK(cudaMemcpyAsync(h.data(), dev, n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return write_floats(c, name, h.data(), n);
}

// one padded field [Nx][ld] of a shot as the reference's [Nx][Nz] array
static int dump_frame(fwi_ctx *c, const char *name, const ShotDesc &d, int fi)
{
    std::vector<float> h((size_t)d.Nx * d.Nz);
    CK(cudaMemcpy2DAsync(h.data(), (size_t)d.Nz * 4, frame_ptr(d, fi), (size_t)d.ld * 4, (size_t)d.Nz * 4, d.Nx,
                         cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return write_floats(c, name, h.data(), h.size());
}

// driver-level files of a gradient run for the shots of one group, written once their adjoint
// sources exist: predicted traces (before the residual; the forward gathers are kept time-major
// in traces_t), adjoint source ([ntr][ns] in d_pre) -- propagation.c:917-934
static int dump_shot_traces(fwi_ctx *c, const std::vector<ShotRun *> &rs)
{
    if (c->dump.verbose < 1) return FWI_OK;
    char name[256];
    for (ShotRun *r : rs) {
        if (r->shot % c->dump.shot_interval != 0) continue;
        const fwi_shot &s = c->shots[r->shot].s;
        const int ns = r->d.ns, ntr = r->d.ntr;
        std::vector<float> t((size_t)ns * ntr), p((size_t)ns * ntr);
        CK(cudaMemcpyAsync(t.data(), r->d.traces_t, t.size() * 4, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int k = 0; k < ns; k++)
            for (int i = 0; i < ntr; i++) p[(size_t)i * ns + k] = t[(size_t)k * ntr + i];
        snprintf(name, sizeof name, "predicted_iter%03d_shot%05d_%d_%d_%.2fms_%.2fm.bin", c->dump.iter, r->shot + 1, ns,
                 ntr, s.dt * 1e3, s.dtr);
        TRY(write_floats(c, name, p.data(), p.size()));
        snprintf(name, sizeof name, "adjsource_iter%03d_shot%05d_%d_%d_%.2fms_%.2fm.bin", c->dump.iter, r->shot + 1, ns,
                 ntr, s.dt * 1e3, s.dtr);
        TRY(dump_device(c, name, c->d_pre[r->shot], (size_t)ns * ntr));
    }
    return FWI_OK;
}

// the raw shot gradient (mode 2's output, before the per-shot preconditioning) -- propagation.c:939-944
static int dump_shot_gradients(fwi_ctx *c, const std::vector<ShotRun *> &rs)
{
    if (c->dump.verbose < 1) return FWI_OK;
    char name[256];
    for (ShotRun *r : rs) {
        if (r->shot % c->dump.shot_interval != 0) continue;
        snprintf(name, sizeof name, "gradient_raw_iter%03d_shot%05d_%d_%d_%.2fm_%.2fm.bin", c->dump.iter, r->shot + 1,
                 c->nz, r->d.nxx, c->dz, c->dx);
        TRY(dump_device(c, name, r->d_gshot, (size_t)c->nz * r->d.nxx));
    }
    return FWI_OK;
}

// snapshots after launch L of a program (verbose > 1): the forward field u(t) a forward step has
// just written (t % snap_interval == 0; u(0) is the zero field), and at adjoint step it the adjoint
// field with this step's injection and the reconstructed forward field the imaging reads
// (propagation.c:597-601, 717-723).  Shots whose (shotID - 1) % shot_interval == 0, as the
// reference's engine selects them.  The reference's reconstructed field at a step that is not an
// imaging step (it % 5 != 0) is whatever its replay buffers last held; this engine keeps the
// reconstructed field of imaging steps only, so that file is not written (with a warning) when
// snap_interval is not a multiple of 5.
static int snapshots_after(fwi_ctx *c, const Program *prog, int L, int shot_base, int nshot)
{
    const int snap = c->dump.snap_interval;
    const int4 pw = prog->items[L];
    char name[256];
    for (int part = 0; part < 2; part++) {
        const int kind = part ? pw.z : pw.x, it = part ? pw.w : pw.y;
        if (kind == K_NONE || kind == K_REP) continue;
        const bool fwd = kind == K_FWD0 || kind == K_FWD1;
        const int t = fwd ? it + 1 : it;
        const bool at0 = fwd && it == 0;  // u(0), the initial zero field, is a snapshot too
        if (!at0 && (t >= c->nt || t % snap != 0)) continue;
        for (int i = 0; i < nshot; i++) {
            const ShotRun *r = c->runs.size() == 1 ? c->runs[0].get() : c->runs[shot_base + i].get();
            const int ishot = c->shots[r->shot].s.shotID - 1;
            if (ishot % c->dump.shot_interval != 0) continue;
            const ShotDesc &d = r->d;
            if (fwd) {
                if (at0) {
                    std::vector<float> z((size_t)d.Nx * d.Nz, 0.0f);
                    snprintf(name, sizeof name, "wavefield_forward_iter%03d_ishot%04d_it%05d_%d_%d_%.2fm_%.2fm.bin",
                             c->dump.iter, ishot, 0, d.Nz, d.Nx, c->dz, c->dx);
                    TRY(write_floats(c, name, z.data(), z.size()));
                }
                if (t < c->nt && t % snap == 0) {
                    snprintf(name, sizeof name, "wavefield_forward_iter%03d_ishot%04d_it%05d_%d_%d_%.2fm_%.2fm.bin",
                             c->dump.iter, ishot, t, d.Nz, d.Nx, c->dz, c->dx);
                    TRY(dump_frame(c, name, d, fwd_idx(d, t, kind == K_FWD1)));
                }
            } else {
                if (it % MST == 0) {
                    snprintf(name, sizeof name,
                             "wavefield_forward_reconstruction_iter%03d_ishot%04d_it%05d_%d_%d_%.2fm_%.2fm.bin",
                             c->dump.iter, ishot, it, d.Nz, d.Nx, c->dz, c->dx);
                    TRY(dump_frame(c, name, d, img_idx(d, it)));
                } else if (!c->dump.warned) {
                    c->dump.warned = true;
                    fprintf(stderr, "<warning>: snapInterval %d is not a multiple of %d: the reconstructed forward "
                                    "wavefields of steps that are not imaging steps are not written\n", snap, MST);
                }
                snprintf(name, sizeof name, "wavefield_backward_iter%03d_ishot%04d_it%05d_%d_%d_%.2fm_%.2fm.bin",
                         c->dump.iter, ishot, it, d.Nz, d.Nx, c->dz, c->dx);
                TRY(dump_frame(c, name, d, adj_idx(d, it)));
            }
        }
    }
    return FWI_OK;
}

extern "C" int fwi_ctx_set_verbose(fwi_ctx *c, int verbose, int iter, int shot_interval, int snap_interval,
                                   const char *dir)
{
    if (!c) return fail(FWI_ERR_ARG, "NULL context");
    if (shot_interval <= 0) {  // the reference's environment variable, default 20 (propagation.c:846-852)
        const char *e = getenv("shotInterval");
        shot_interval = e ? atoi(e) : 20;
    }
    if (snap_interval <= 0) {  // propagation.c:432-440
        const char *e = getenv("snapInterval");
        snap_interval = e ? atoi(e) : 1000;
    }
    if (verbose > 0 && (shot_interval <= 0 || (verbose > 1 && snap_interval <= 0)))
        return fail(FWI_ERR_ARG, "shotInterval %d / snapInterval %d must be positive", shot_interval, snap_interval);
    if ((verbose > 1) != (c->dump.verbose > 1) || (verbose > 1 && snap_interval != c->dump.snap_interval))
        drop_graphs(c);  // the step kernels' snapshot steps change
    c->dump.verbose = verbose;
    c->dump.iter = iter;
    c->dump.shot_interval = shot_interval;
    c->dump.snap_interval = snap_interval;
    c->dump.dir = dir ? dir : "";
    c->dump.warned = false;
    return FWI_OK;
}

// ---------------------------------------------------------------- bounded-wait self-test
// One block waits on an mbarrier phase that nothing completes, with the step kernel's bounded
// wait: it must give up after limit_ns, set the context's error word and return, so that the
// host reports FWI_ERR_CUDA and the context stays usable.  No copy, fault or trap is involved.
static __global__ void k_wait_probe(int *err, unsigned long long limit_ns)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const bool ok = mbar_wait(smem_u32(&bar), 0, limit_ns);
    if (!__all_sync(0xffffffffu, ok) && (threadIdx.x & 31) == 0) atomicExch(err, 1);
}

extern "C" int fwi_ctx_selftest_wait(fwi_ctx *c, int limit_ms)
{
    if (!c) return fail(FWI_ERR_ARG, "NULL context");
    if (limit_ms < 1 || limit_ms > 2000) return fail(FWI_ERR_ARG, "limit_ms %d outside [1, 2000]", limit_ms);
    CK(cudaSetDevice(c->device));
    k_wait_probe<<<1, 64, 0, c->stream>>>(c->d_err, (unsigned long long)limit_ms * 1000000ull);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return check_kernel_error(c);
}

static int upload_descs(fwi_ctx *c, const std::vector<ShotDesc> &v)
{
    if ((int)v.size() > c->desc_cap) {
        drop_graphs(c);  // captured launches hold the old descriptor array
        dfree(c, c->d_desc, 0);
        c->d_desc = nullptr;
        c->desc_cap = std::max<int>((int)v.size(), 8);
        TRY(dmalloc(c, (void **)&c->d_desc, c->desc_cap * sizeof(ShotDesc)));
    }
    CK(cudaMemcpyAsync(c->d_desc, v.data(), v.size() * sizeof(ShotDesc), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FWI_OK;
}

static int scratch(fwi_ctx *c, size_t bytes, void **out)
{
    if (bytes > c->scratch_cap) {
        dfree(c, c->d_scratch, 0);
        c->d_scratch = nullptr;
        c->scratch_cap = std::max<size_t>(bytes, 1 << 16);
        TRY(dmalloc(c, &c->d_scratch, c->scratch_cap));
    }
    *out = c->d_scratch;
    return FWI_OK;
}

// small descriptor arrays into the scratch area, ordered on the stream: a copy from pageable host
// memory is staged before cudaMemcpyAsync returns (the host vector may go), and the kernels that
// read the previous contents of the area run before the copy on the same stream
template <class T>
static int put(fwi_ctx *c, const std::vector<T> &v, T **dev, size_t offset_bytes)
{
    void *base;
    TRY(scratch(c, offset_bytes + v.size() * sizeof(T) + 256, &base));
    *dev = (T *)((char *)base + offset_bytes);
    CK(cudaMemcpyAsync(*dev, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return FWI_OK;
}

static int ensure_red(fwi_ctx *c)
{
    if (!c->d_red) TRY(dmalloc(c, (void **)&c->d_red, (size_t)(2 * 1024 + 4096) * 8 * 64));
    return FWI_OK;
}

// FP64 sums of several arrays: results on the device (2 per descriptor, *out_dev) and, unless
// to_host is false, in out_host (a host round trip)
static int reduce(fwi_ctx *c, std::vector<SumDesc> sd, std::vector<double> &out_host, double **out_dev = nullptr,
                  bool to_host = true)
{
    TRY(ensure_red(c));
    const int NP = 592;  // partials per array: 4 per SM
    const int nd = (int)sd.size();
    if (nd > 64) return fail(FWI_ERR_ARG, "too many reduction operands");
    for (int i = 0; i < nd; i++) sd[i].partial = c->d_red + (size_t)i * 2 * NP;
    double *res = c->d_red + (size_t)64 * 2 * NP;
    SumDesc *d;
    TRY(put(c, sd, &d, 0));
    k_sum_partial<256><<<dim3(NP, nd), 256, 0, c->stream>>>(d);
    k_sum_final<<<nd, 32, 0, c->stream>>>(d, NP, res);
    c->launches += 2;
    CK(cudaGetLastError());
    if (out_dev) *out_dev = res;
    if (!to_host) return FWI_OK;
    out_host.resize(2 * nd);
    CK(cudaMemcpyAsync(out_host.data(), res, 2 * nd * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FWI_OK;
}

// ---------------------------------------------------------------- runs
static int gather(fwi_ctx *c, const std::vector<ShotRun *> &rs, int mode, bool with_adj, bool trace_taper = true)
{
    if (mode == 1) TRY(obs_join(c));  // the residual reads the observed gathers
    std::vector<GatherDesc> gd;
    int maxns = 1, maxtr = 1;
    for (ShotRun *r : rs) {
        GatherDesc g;
        g.traces_t = r->d.traces_t;
        g.pre = c->d_pre[r->shot];
        g.obs = c->d_obs[r->shot];
        g.adj_t = with_adj ? (float *)r->d.adj_t : nullptr;
        g.tct = r->d_tct;
        g.tcr = r->d_tcr;
        g.ns = r->d.ns;
        g.ntr = r->d.ntr;
        g.Lt = mode == 1 ? r->Lt : 0;
        g.Lr = mode == 1 && trace_taper ? r->Lr : 0;
        g.adj_rows = c->nt;
        gd.push_back(g);
        maxns = std::max(maxns, g.ns);
        maxtr = std::max(maxtr, g.ntr);
    }
    GatherDesc *d;
    TRY(put(c, gd, &d, 0));
    dim3 grid((maxns + 31) / 32, (maxtr + 31) / 32, (unsigned)gd.size());
    k_gather<<<grid, dim3(32, 8), 0, c->stream>>>(d, mode);
    c->launches++;
    CK(cudaGetLastError());
    return FWI_OK;
}

static __global__ void k_to_time_major(const float *__restrict__ a, float *__restrict__ out, int ntr, int ns, int nt);

// ---------------------------------------------------------------- residual filters
static std::string bits(float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    return std::to_string(u);
}

// an operator matrix built once on the host (FP64 sums, stored as float) and kept on the device
template <class Build>
static int device_operator(fwi_ctx *c, const std::string &key, size_t count, Build build, const float **out)
{
    auto it = c->ops.find(key);
    if (it == c->ops.end()) {
        std::vector<float> h(count);
        build(h.data());
        float *d = nullptr;
        TRY(dmalloc(c, (void **)&d, count * 4));
        CK(cudaMemcpy(d, h.data(), count * 4, cudaMemcpyHostToDevice));
        it = c->ops.emplace(key, std::make_pair(d, count * 4)).first;
    }
    *out = it->second.first;
    return FWI_OK;
}

// The residual filters and the trace interpolation as FFT convolutions (fwi_fft.cuh): the
// spectrum of the filter's circular kernel and the FFT twiddles, built once on the host in FP64
// and kept on the device (2M floats each, M = fwi_conv_size(n)).
static int conv_tables(fwi_ctx *c, const std::string &key, int n, const std::function<void(double *)> &kernel,
                       ConvDesc *d)
{
    const int M = fwi_conv_size(n);
    if (M > FFT_CONV_MAX)
        return fail(FWI_ERR_UNSUPPORTED, "FFT convolution of length %d needs %d points (at most %d)", n, M,
                    FFT_CONV_MAX);
    const bool f64 = conv_in_f64(M);
    const float *G, *tw;
    // FP64 tables take 4M / 2M floats' room (double2), FP32 ones 2M / M
    TRY(device_operator(c, (f64 ? "spec64/" : "spec/") + key, (size_t)(f64 ? 4 : 2) * M, [&](float *out) {
        std::vector<double> h(n);
        kernel(h.data());
        if (f64) fwi_conv_spectrum_f64(h.data(), n, M, reinterpret_cast<double *>(out));
        else fwi_conv_spectrum(h.data(), n, M, out);
    }, &G));
    TRY(device_operator(c, (f64 ? "tw64/" : "tw/") + std::to_string(M), (size_t)(f64 ? 2 : 1) * M, [&](float *out) {
        if (f64) fwi_fft_twiddles_f64(M, reinterpret_cast<double *>(out));
        else fwi_fft_twiddles(M, out);
    }, &tw));
    d->G = G;
    d->tw = tw;
    d->dbl = f64 ? 1 : 0;
    d->N = n;
    return FWI_OK;
}

// apply_traces_lowpass (filter 0) / apply_traces_bandpass (1) along `n`-sample sequences
static int filter_tables(fwi_ctx *c, int filter, int n, float fpass, float fcut, float dt, ConvDesc *d)
{
    const std::string key = "filter" + std::to_string(filter) + "/" + std::to_string(n) + "/" + bits(fpass) + "/" +
                            bits(fcut) + "/" + bits(dt);
    return conv_tables(c, key, n, [&](double *h) { fwi_filter_kernel(filter, n, fpass, fcut, dt, h); }, d);
}

static int run_conv(fwi_ctx *c, const ConvDesc &d)
{
    const cudaError_t e = launch_fft_conv(d, c->stream);
    if (e != cudaSuccess) return fail(FWI_ERR_CUDA, "FFT convolution: %s", cudaGetErrorString(e));
    c->launches++;
    return FWI_OK;
}

static int taper(fwi_ctx *c, float *a, const ShotRun *r, int Lt, int Lr)
{
    TaperDesc t{a, r->d_tct, r->d_tcr, r->d.ns, r->d.ntr, Lt, Lr};
    TaperDesc *d;
    TRY(put(c, std::vector<TaperDesc>{t}, &d, 0));
    k_taper<<<dim3(148, 1), 256, 0, c->stream>>>(d);
    c->launches++;
    CK(cudaGetLastError());
    return FWI_OK;
}

// compute_adjoint_source2d for filters 0/1 (optimization.c:368-415) and the injection layout for
// sampleRate > 1 (interpolate_traces, common.c:482-582): residual and time taper in k_gather, then
// per shot the time filter (FFT convolution along each trace), the trace taper, the trace filter
// (FFT convolution across the traces of each time sample), both tapers; the adjoint source for the
// injection is the interpolation (FFT convolution of the zero-stuffed traces) written straight
// into adj_t [nt][ntr], or a transpose for sampleRate 1.
static int adjoint_source_filtered(fwi_ctx *c, const std::vector<ShotRun *> &rs, int filter, bool with_adj)
{
    const bool fft = filter == 0 || filter == 1;
    TRY(gather(c, rs, 1, false, /*trace_taper=*/!fft));
    for (ShotRun *r : rs) {
        const int ns = r->d.ns, ntr = r->d.ntr;
        const fwi_shot &s = c->shots[r->shot].s;
        float *pre = c->d_pre[r->shot];
        if (fft) {
            const size_t need = (size_t)ns * ntr * 4;
            if (need > c->fft_tmp_bytes) {
                dfree(c, c->d_fft_tmp, c->fft_tmp_bytes);
                c->d_fft_tmp = nullptr;
                c->fft_tmp_bytes = 0;
                TRY(dmalloc(c, (void **)&c->d_fft_tmp, need));
                c->fft_tmp_bytes = need;
            }
            // time filter: each trace, a row of the [ntr][ns] gather
            ConvDesc t{};
            TRY(filter_tables(c, filter, ns, r->fpass, 2.0f * r->fpass, s.dt, &t));
            t.in = pre; t.in_es = 1; t.in_ss = ns; t.n_in = ns; t.stuff = 1;
            t.out = c->d_fft_tmp; t.out_es = 1; t.out_ss = ns; t.n_out = ns; t.nseq = ntr;
            TRY(run_conv(c, t));
            TRY(taper(c, c->d_fft_tmp, r, 0, r->Lr));
            // trace filter: each time sample's vector over the traces
            ConvDesc x{};
            TRY(filter_tables(c, filter, ntr, r->kpass, 2.0f * r->kpass, s.dtr, &x));
            x.in = c->d_fft_tmp; x.in_es = ns; x.in_ss = 1; x.n_in = ntr; x.stuff = 1;
            x.out = pre; x.out_es = ns; x.out_ss = 1; x.n_out = ntr; x.nseq = ns;
            TRY(run_conv(c, x));
            TRY(taper(c, pre, r, r->Lt, r->Lr));
        }
        if (!with_adj) continue;
        float *adj = (float *)r->d.adj_t;
        if (r->d.sr > 1) {
            // adj_t[k][r] = sum_j g[(k - j sr) mod N] pre[r][j] for k < N, 0 for N <= k < nt
            const int sr = r->d.sr, N = (ns - 1) * sr + 1;
            ConvDesc q{};
            TRY(conv_tables(c, "interp/" + std::to_string(ns) + "/" + std::to_string(sr), N,
                            [&](double *g) { fwi_interp_kernel(ns, sr, g); }, &q));
            q.in = pre; q.in_es = 1; q.in_ss = ns; q.n_in = ns; q.stuff = sr;
            q.out = adj; q.out_es = ntr; q.out_ss = 1; q.n_out = c->nt; q.nseq = ntr;
            TRY(run_conv(c, q));
        } else {
            k_to_time_major<<<296, 256, 0, c->stream>>>(pre, adj, ntr, ns, c->nt);
            c->launches++;
            CK(cudaGetLastError());
        }
    }
    return FWI_OK;
}

static int finalize(fwi_ctx *c, const std::vector<ShotRun *> &rs, int which)
{
    std::vector<FinDesc> fd;
    for (ShotRun *r : rs) {
        FinDesc f;
        f.acc = which == 0 ? r->d.H : r->d.Gacc;
        f.out = which == 0 ? r->d_hshot : r->d_gshot;
        f.vp = c->d_vp;
        f.rho = c->d_rho;
        f.ix_min = c->shots[r->shot].s.ix_min;
        f.nxx = r->d.nxx;
        f.nz = c->nz;
        f.pml = c->pml;
        f.ld = r->d.ld;
        fd.push_back(f);
    }
    FinDesc *d;
    TRY(put(c, fd, &d, 0));
    k_finalize<<<dim3(148, (unsigned)fd.size()), 256, 0, c->stream>>>(d, which);
    c->launches++;
    CK(cudaGetLastError());
    return FWI_OK;
}

static int shot_precondition(fwi_ctx *c, const std::vector<ShotRun *> &rs)
{
    std::vector<SumDesc> sd;
    for (ShotRun *r : rs) {
        SumDesc s{};
        s.a = r->d_hshot;
        s.n = (long long)r->d.nxx * c->nz;
        s.op = 0;
        sd.push_back(s);
    }
    std::vector<double> h;
    double *res;
    for (size_t i0 = 0; i0 < sd.size(); i0 += 64) {
        std::vector<SumDesc> part(sd.begin() + i0, sd.begin() + std::min(sd.size(), i0 + 64));
        TRY(reduce(c, part, h, &res, false));
        std::vector<PrecDesc> pd;
        for (size_t i = 0; i < part.size(); i++) {
            ShotRun *r = rs[i0 + i];
            PrecDesc p;
            p.g = r->d_gshot;
            p.h = r->d_hshot;
            p.n = part[i].n;
            p.sum = res + 2 * i;
            pd.push_back(p);
        }
        PrecDesc *d;
        TRY(put(c, pd, &d, 4096));
        k_shot_precondition<<<dim3(148, (unsigned)pd.size()), 256, 0, c->stream>>>(d);
        c->launches++;
        CK(cudaGetLastError());
    }
    return FWI_OK;
}

// ---------------------------------------------------------------- exchange between ranks
// The hook replaces `count` device doubles by their sum over the ranks, ordered on the
// engine's stream.  Without a hook the context is the whole survey and nothing happens.
static int exchange(fwi_ctx *c, double *dev, size_t count)
{
    if (!c->ar_fn) return FWI_OK;
    const int rc = c->ar_fn(dev, count, (void *)c->stream, c->ar_user);
    if (rc != 0) return fail(FWI_ERR_CUDA, "all-reduce hook failed (%d)", rc);
    CK(cudaGetLastError());
    return FWI_OK;
}

// host scalars summed over the ranks through the hook (a round trip through d_xchg)
static int exchange_scalars(fwi_ctx *c, double *v, int n)
{
    if (!c->ar_fn) return FWI_OK;
    if (n > 8) return fail(FWI_ERR_ARG, "too many scalars for one exchange");
    if (!c->d_xchg) TRY(dmalloc(c, (void **)&c->d_xchg, 8 * sizeof(double)));
    CK(cudaMemcpyAsync(c->d_xchg, v, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    TRY(exchange(c, c->d_xchg, (size_t)n));
    CK(cudaMemcpyAsync(v, c->d_xchg, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FWI_OK;
}

extern "C" int fwi_ctx_set_allreduce(fwi_ctx *c, fwi_allreduce_fn fn, void *user)
{
    if (!c) return fail(FWI_ERR_ARG, "ctx is NULL");
    c->ar_fn = fn;
    c->ar_user = user;
    return FWI_OK;
}

static int stack_and_precondition(fwi_ctx *c, const std::vector<ShotRun *> &rs, int precondition)
{
    const long long m = (long long)c->nz * c->nx;
    CK(cudaMemsetAsync(c->d_gc, 0, m * 8, c->stream));
    CK(cudaMemsetAsync(c->d_hc, 0, m * 8, c->stream));
    std::vector<StackShot> ss;
    for (ShotRun *r : rs) {
        StackShot s;
        s.g = r->d_gshot;
        s.h = r->d_hshot;
        s.ix_min = c->shots[r->shot].s.ix_min;
        s.ix_max = c->shots[r->shot].s.ix_max;
        ss.push_back(s);
    }
    StackShot *d;
    TRY(put(c, ss, &d, 0));
    k_stack<<<592, 256, 0, c->stream>>>(d, (int)ss.size(), c->nz, c->nx, precondition == 1, c->d_gc, c->d_hc);
    c->launches++;
    // the one exchange step of a sharded gradient: both FP64 stacks summed over the ranks
    TRY(exchange(c, c->d_gc, 2 * (size_t)m));
    k_to_float<<<592, 256, 0, c->stream>>>(c->d_gc, c->d_grad, m);
    c->launches++;
    if (precondition == 1) {
        k_to_float<<<592, 256, 0, c->stream>>>(c->d_hc, c->d_prec, m);
        c->launches++;
    }
    if (c->dump.verbose > 0) {  // the stacks before the global preconditioning (propagation.c:996-1005)
        char name[256];
        snprintf(name, sizeof name, "gradient_raw_iter%03d_%d_%d_%.2fm_%.2fm.bin", c->dump.iter, c->nz, c->nx, c->dz,
                 c->dx);
        TRY(dump_device(c, name, c->d_grad, (size_t)m));
        if (precondition == 1) {
            snprintf(name, sizeof name, "precond_iter%03d_%d_%d_%.2fm_%.2fm.bin", c->dump.iter, c->nz, c->nx, c->dz,
                     c->dx);
            TRY(dump_device(c, name, c->d_prec, (size_t)m));
        }
    }
    if (precondition == 1) {
        SumDesc s{};
        s.a = c->d_prec;
        s.n = m;
        s.op = 2;
        std::vector<double> h;
        double *res;
        TRY(reduce(c, {s}, h, &res, false));
        k_global_precondition<<<592, 256, 0, c->stream>>>(c->d_grad, c->d_prec, m, res, 0.005f);
        c->launches++;
    }
    CK(cudaGetLastError());
    return FWI_OK;
}

// zero the frames a pass reads before it has written them
static int zero_initial(fwi_ctx *c, ShotRun *r, bool gradient)
{
    const size_t fb = (size_t)r->d.frame * 4;
    CK(cudaMemsetAsync(frame_ptr(r->d, F_FWD), 0, NROT * fb, c->stream));
    if (gradient) {
        CK(cudaMemsetAsync(frame_ptr(r->d, F_CK), 0, 2 * fb, c->stream));  // u(-1), u(0)
        CK(cudaMemsetAsync(r->d.H, 0, (size_t)r->d.frame * 8, c->stream));
        CK(cudaMemsetAsync(r->d.Gacc, 0, (size_t)r->d.frame * 8, c->stream));
    }
    return FWI_OK;
}

// A(nt) = 0 and A(nt-1) = -injection(nt-1) (propagation.c:676-682 applied to the zero field)
__global__ void k_adj_init(const ShotDesc *__restrict__ shots, int shot_base)
{
    const ShotDesc &S = shots[shot_base + blockIdx.x];
    if (threadIdx.x != 0) return;
    float *A = adj_buf(S, S.nt - 1);
    const float *arow = S.adj_t + (long long)(S.nt - 1) * S.ntr;
    for (int x = 0; x < S.Nx; x++)
        for (int e = S.colptr[x]; e < S.colptr[x + 1]; e++) {
            int2 rr = S.rec[e];
            float a = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(arow[rr.y], S.recK[e]), S.dt), S.dt), S.invdx), S.invdz);
            float *cell = A + (long long)x * S.ld + rr.x;
            *cell = __fsub_rn(*cell, a);
        }
}

static int adj_init(fwi_ctx *c, const std::vector<ShotRun *> &rs, int shot_base)
{
    for (ShotRun *r : rs) {
        const size_t fb = (size_t)r->d.frame * 4;
        CK(cudaMemsetAsync(adj_buf(r->d, c->nt - 1), 0, fb, c->stream));
        CK(cudaMemsetAsync(adj_buf(r->d, c->nt), 0, fb, c->stream));
    }
    k_adj_init<<<(unsigned)rs.size(), 32, 0, c->stream>>>(c->d_desc, shot_base);
    c->launches++;
    CK(cudaGetLastError());
    return FWI_OK;
}

// run a program over a group of shots, through a cached CUDA graph on the batched path
static int run_program(fwi_ctx *c, const std::string &key, const Program *prog, int shot_base, int nshot,
                       const ShotRun *r0, bool batched)
{
    if (c->dump.verbose > 1) {
        // snapshots: direct launches with a copy-out after every snapshot step
        c->snapping = true;
        const int rc = launch_steps(c, prog, shot_base, nshot, r0, batched);
        c->snapping = false;
        return rc;
    }
    if (!batched) return launch_steps(c, prog, shot_base, nshot, r0, false);
    if (!c->use_graphs) return launch_steps(c, prog, shot_base, nshot, r0, true);
    {  // one wavefront launch needs no graph
        int wr = 0, wn = 0;
        if (wave_shape(c, prog, 0, (int)prog->items.size(), nshot, r0, &wr, &wn))
            return launch_steps(c, prog, shot_base, nshot, r0, true);
    }
    const std::string gk = key + "#" + std::to_string(prog->depth);  // graphs of one- and two-step programs differ
    auto it = c->graphs.find(gk);
    if (it == c->graphs.end()) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        long long before = c->launches;
        int rc = launch_steps(c, prog, shot_base, nshot, r0, true);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (rc != FWI_OK) return rc;
        if (e != cudaSuccess) return fail(FWI_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        cudaGraphExec_t ge;
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(FWI_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        c->graph_launches[gk] = c->launches - before;  // the kernels the graph holds
        c->launches = before;
        it = c->graphs.emplace(gk, ge).first;
    }
    CK(cudaGraphLaunch(it->second, c->stream));
    c->stats.graph_launches++;
    c->launches += c->graph_launches[gk];
    return FWI_OK;
}

// run_program between a pair of events of the pass kind's timer; the autotuner, which times
// launch shapes before a new shape's first pass, runs before the first event
static int timed_program(fwi_ctx *c, int kind, const std::string &key, const Program *prog, int shot_base,
                         int nshot, const ShotRun *r0, bool batched)
{
    const char *ke = getenv("FWI_KERNEL");
    const bool tile_kernel = !(ke && strcmp(ke, "step") == 0);
    if (c->tune && tile_kernel && !getenv("FWI_TX") && !getenv("FWI_NST") && !getenv("FWI_CHUNK") && !getenv("FWI_GPT") &&
        !getenv("FWI_OCC"))
        TRY(autotune(c, shot_base, nshot, r0, batched, prog->depth));
    fwi_ctx::PassTimer &t = c->pass[kind];
    if (t.used == t.ev.size()) {
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        t.ev.push_back({a, b});
    }
    const long long l0 = c->launches;
    auto &e = t.ev[t.used++];
    CK(cudaEventRecord(e.first, c->stream));
    TRY(run_program(c, key, prog, shot_base, nshot, r0, batched));
    CK(cudaEventRecord(e.second, c->stream));
    t.launches += c->launches - l0;
    return FWI_OK;
}

// time steps per launch of the step kernel for this run: the context's (two unless FWI_DEPTH=1),
// one for runs that write snapshots and for the cp.async comparison kernel
static int run_depth(const fwi_ctx *c)
{
    const char *ke = getenv("FWI_KERNEL");
    if (c->dump.verbose > 1 || (ke && strcmp(ke, "step") == 0)) return 1;
    return c->depth;
}

static int forward_program(fwi_ctx *c, int kind, Program **out)
{
    const bool two = run_depth(c) == 2;
    const std::string key = std::string(kind == K_FWD1 ? "fwd1" : "fwd0") + (two ? "x2" : "");
    return get_program(c, key, two ? program_forward2(c->nt, kind) : program_forward(c->nt, kind), out);
}

static int adjoint_program(fwi_ctx *c, bool batched, Program **out)
{
    if (run_depth(c) == 2) return get_program(c, "adj/x2", program_adjoint2(c->nt), out);
    return get_program(c, batched ? "adj/overlap" : "adj/plain", program_adjoint(c->nt, batched), out);
}

static int run_forward_group(fwi_ctx *c, std::vector<ShotRun *> &rs, int problem, float freq, int filter, bool batched,
                             const std::string &gkey, int shot_base)
{
    Program *prog;
    TRY(choose_depth(c, shot_base, (int)rs.size(), rs[0], batched));
    TRY(forward_program(c, K_FWD0, &prog));
    for (ShotRun *r : rs) TRY(zero_initial(c, r, false));
    TRY(timed_program(c, 0, "fwd0/" + gkey, prog, shot_base, (int)rs.size(), rs[0], batched));
    if (problem == 2) {
        if (filter < 0 || filter > 2) return fail(FWI_ERR_ARG, "residual filter %d (0 lowpass, 1 bandpass, 2 none)", filter);
        for (ShotRun *r : rs) TRY(prepare_taper(c, r, freq));
    }
    if (problem == 2 && (filter == 0 || filter == 1)) TRY(adjoint_source_filtered(c, rs, filter, false));
    else TRY(gather(c, rs, problem == 2 ? 1 : 0, false));
    return FWI_OK;
}

// forward pass of a gradient (engine mode 1): checkpoints, samples, pseudo-Hessian
static int grad_forward(fwi_ctx *c, std::vector<ShotRun *> &rs, int precondition, bool batched,
                        const std::string &gkey, int shot_base)
{
    Program *pf;
    TRY(choose_depth(c, shot_base, (int)rs.size(), rs[0], batched));
    TRY(forward_program(c, K_FWD1, &pf));
    for (ShotRun *r : rs) TRY(zero_initial(c, r, true));
    TRY(timed_program(c, 0, "fwd1/" + gkey, pf, shot_base, (int)rs.size(), rs[0], batched));
    if (precondition == 1) TRY(finalize(c, rs, 0));
    return FWI_OK;
}

// adjoint pass (engine mode 2) from the adjoint sources in adj_t: replay + adjoint + imaging
static int grad_adjoint(fwi_ctx *c, std::vector<ShotRun *> &rs, bool batched, const std::string &gkey, int shot_base)
{
    Program *pa;
    TRY(adjoint_program(c, batched, &pa));
    TRY(adj_init(c, rs, shot_base));
    TRY(timed_program(c, 1, std::string(batched ? "adjo/" : "adjp/") + gkey, pa, shot_base, (int)rs.size(), rs[0],
                      batched));
    TRY(finalize(c, rs, 1));
    return FWI_OK;
}

static int run_gradient_group(fwi_ctx *c, std::vector<ShotRun *> &rs, float freq, int filter, int precondition,
                              bool batched, const std::string &gkey, int shot_base)
{
    if (filter < 0 || filter > 2) return fail(FWI_ERR_ARG, "residual filter %d (0 lowpass, 1 bandpass, 2 none)", filter);
    TRY(grad_forward(c, rs, precondition, batched, gkey, shot_base));
    for (ShotRun *r : rs) TRY(prepare_taper(c, r, freq));
    bool interp = false;
    for (ShotRun *r : rs) interp = interp || r->d.sr > 1;
    if (filter == 2 && !interp) TRY(gather(c, rs, 1, true));  // residual + tapers straight into adj_t
    else TRY(adjoint_source_filtered(c, rs, filter, true));
    TRY(dump_shot_traces(c, rs));
    TRY(grad_adjoint(c, rs, batched, gkey, shot_base));
    TRY(dump_shot_gradients(c, rs));
    if (precondition == 1) TRY(shot_precondition(c, rs));
    return FWI_OK;
}

// Shots per wave of the batched path: all of them when the frame blocks of every group fit next
// to what is allocated already (the reduction buffer is allocated first) and a reserve for what
// a pass allocates later (descriptor scratch, programs, residual-filter operators): 1/16 of the
// context's budget (at least 4 MiB), else 1/16 of the device.  Otherwise as many shots of the
// largest frame block as fit.  FWI_WAVE caps the wave (the memory-bounded schedule on a small
// survey).
static const int WAVE_POOL = -2;
static int wave_shots(fwi_ctx *c, const std::vector<std::pair<int, int>> &groups, int *out)
{
    TRY(ensure_red(c));
    int ns = 0;
    size_t need = 0, per_max = 0, pooled = 0;
    for (auto &gr : groups) {
        const ShotDesc &d = c->runs[gr.first]->d;
        const size_t per = (size_t)d.nfr * (size_t)d.frame * 4;
        need += per * (size_t)gr.second;
        per_max = std::max(per_max, per);
        ns += gr.second;
    }
    for (auto &kv : c->pools) pooled += kv.second.bytes;
    size_t avail;
    if (c->budget) {
        avail = c->budget > c->used ? c->budget - c->used + pooled : pooled;
        avail -= std::min(avail, std::max<size_t>(c->budget / 16, (size_t)4 << 20));
    } else {
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        avail = fr + pooled;
        avail -= std::min(avail, tot / 16);
    }
    int wave = need <= avail ? ns : (int)std::max<size_t>(1, avail / std::max<size_t>(per_max, 1));
    if (const char *e = getenv("FWI_WAVE")) wave = std::min(wave, std::max(1, atoi(e)));
    *out = std::min(wave, ns);
    return FWI_OK;
}

extern "C" int fwi_ctx_run(fwi_ctx *c, int problem, float freq, int filter, int precondition, int path)
{
    if (!c) return fail(FWI_ERR_ARG, "NULL context");
    if (problem < 0 || problem > 2) return fail(FWI_ERR_ARG, "problem must be 0, 1 or 2 (got %d)", problem);
    if (c->shots.empty()) return fail(FWI_ERR_STATE, "no shots");
    CK(cudaSetDevice(c->device));
    const bool batched = path == FWI_PATH_BATCHED;
    const bool gradient = problem == 1;
    const int ns = (int)c->shots.size();
    long long launches0 = c->launches;
    double cells = 0.0;
    for (auto &t : c->pass) {
        t.used = 0;
        t.ms = 0.0;
        t.launches = 0;
    }
    CK(cudaEventRecord(c->ev0, c->stream));
    if (batched) {
        // one group per plan geometry: shots sharing a window run in the same launches
        if ((int)c->runs.size() != ns) {
            free_runs(c);
            for (int i = 0; i < ns; i++) c->runs.emplace_back(new ShotRun());
        }
        std::vector<ShotDesc> descs(ns);
        for (int i = 0; i < ns; i++) {
            TRY(prepare_run(c, c->runs[i].get(), i, gradient));
            c->runs[i]->d.hessian = gradient && precondition == 1;
        }
        // group consecutive shots with the same plan
        std::vector<std::pair<int, int>> groups;
        for (int i = 0; i < ns; i++) {
            if (groups.empty() || c->runs[i]->plan != c->runs[groups.back().first]->plan) groups.push_back({i, 1});
            else groups.back().second++;
        }
        // Waves: when the frame blocks of the whole survey do not fit in the device memory left,
        // the shots of each group run in waves of as many shots as fit, one after the other
        // through one reused frame pool (a pass zeroes the frames it starts from).  Everything
        // else a shot keeps -- traces, per-shot gradient window, accumulators -- stays allocated
        // for the whole run, so the stack after the last wave sees every shot.
        int wave = ns;
        TRY(wave_shots(c, groups, &wave));
        if (wave >= ns) {
            auto wp = c->pools.find(WAVE_POOL);
            if (wp != c->pools.end()) {
                drop_graphs(c);
                dfree(c, wp->second.p, wp->second.bytes);
                c->pools.erase(wp);
            }
            for (auto &gr : groups) {
                std::vector<ShotRun *> rs;
                for (int i = gr.first; i < gr.first + gr.second; i++) rs.push_back(c->runs[i].get());
                TRY(assign_pool(c, gr.first, rs));
            }
            for (int i = 0; i < ns; i++) descs[i] = c->runs[i]->d;
            TRY(upload_descs(c, descs));
        } else {
            for (auto it = c->pools.begin(); it != c->pools.end();) {
                if (it->first == WAVE_POOL) {
                    ++it;
                    continue;
                }
                drop_graphs(c);  // captured launches hold the released pool's tensor maps
                dfree(c, it->second.p, it->second.bytes);
                it = c->pools.erase(it);
            }
        }
        for (auto &gr : groups)
            for (int w0 = gr.first; w0 < gr.first + gr.second; w0 += wave) {
                const int m = std::min(wave, gr.first + gr.second - w0);
                std::vector<ShotRun *> rs;
                for (int i = w0; i < w0 + m; i++) rs.push_back(c->runs[i].get());
                if (wave < ns) {
                    TRY(assign_pool(c, WAVE_POOL, rs));
                    for (int i = 0; i < ns; i++) descs[i] = c->runs[i]->d;
                    TRY(upload_descs(c, descs));
                }
                std::string gkey = std::to_string(w0) + "+" + std::to_string(m) + "@" +
                                   std::to_string((long long)(intptr_t)rs[0]->plan);
                if (gradient) TRY(run_gradient_group(c, rs, freq, filter, precondition, true, gkey, w0));
                else TRY(run_forward_group(c, rs, problem, freq, filter, true, gkey, w0));
            }
        if (gradient) {
            std::vector<ShotRun *> all;
            for (auto &r : c->runs) all.push_back(r.get());
            TRY(stack_and_precondition(c, all, precondition));
        }
    } else {
        // plain: one shot state, shots in sequence (propagation.c:857, :895)
        if (c->runs.size() != 1) {
            free_runs(c);
            c->runs.emplace_back(new ShotRun());
        }
        ShotRun *r = c->runs[0].get();
        std::vector<float *> gsh, hsh;
        std::vector<std::unique_ptr<ShotRun>> keep;  // per-shot gradient copies for the stack
        std::vector<ShotRun *> stack_list;
        for (int i = 0; i < ns; i++) {
            TRY(prepare_run(c, r, i, gradient));
            r->d.hessian = gradient && precondition == 1;
            TRY(assign_pool(c, -1, {r}));
            TRY(upload_descs(c, {r->d}));
            std::vector<ShotRun *> rs = {r};
            if (gradient) {
                TRY(run_gradient_group(c, rs, freq, filter, precondition, false, "", 0));
                // keep this shot's FP32 gradient / preconditioner for the stack
                std::unique_ptr<ShotRun> k(new ShotRun());
                k->shot = i;
                size_t m = (size_t)c->nz * r->d.nxx * 4;
                void *q;
                TRY(ralloc(c, k.get(), &q, m)); k->d_gshot = (float *)q;
                TRY(ralloc(c, k.get(), &q, m)); k->d_hshot = (float *)q;
                CK(cudaMemcpyAsync(k->d_gshot, r->d_gshot, m, cudaMemcpyDeviceToDevice, c->stream));
                CK(cudaMemcpyAsync(k->d_hshot, r->d_hshot, m, cudaMemcpyDeviceToDevice, c->stream));
                stack_list.push_back(k.get());
                keep.push_back(std::move(k));
            } else {
                TRY(run_forward_group(c, rs, problem, freq, filter, false, "", 0));
            }
            CK(cudaStreamSynchronize(c->stream));
        }
        if (gradient) TRY(stack_and_precondition(c, stack_list, precondition));
        CK(cudaStreamSynchronize(c->stream));
        for (auto &k : keep) free_run(c, k.get());
    }
    TRY(obs_join(c));  // a run that read no observed gathers still returns after their upload
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    TRY(check_kernel_error(c));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    for (auto &t : c->pass)
        for (size_t k = 0; k < t.used; k++) {
            float m = 0.f;
            CK(cudaEventElapsedTime(&m, t.ev[k].first, t.ev[k].second));
            t.ms += m;
        }
    for (int i = 0; i < ns; i++) {
        const fwi_shot &s = c->shots[i].s;
        double cellsz = (double)(c->nz + 2 * c->pml) * (s.ix_max - s.ix_min + 1 + 2 * c->pml);
        int d = fwi_ck_interval(c->nt);
        double steps = gradient ? (double)c->nt * 2 + (c->nt - fwi_ck_count(c->nt)) : (double)c->nt;
        (void)d;
        cells += cellsz * steps;
    }
    c->stats.ms = ms;
    c->stats.cell_updates = cells;
    c->stats.kernel_launches = c->launches - launches0;
    c->stats.device_bytes = c->used;
    return FWI_OK;
}

extern "C" int fwi_ctx_get_traces(fwi_ctx *c, int ishot, float *out)
{
    if (!c || !out || ishot < 0 || ishot >= (int)c->shots.size()) return fail(FWI_ERR_ARG, "bad shot index %d", ishot);
    CK(cudaSetDevice(c->device));
    const fwi_shot &s = c->shots[ishot].s;
    CK(cudaMemcpyAsync(out, c->d_pre[ishot], (size_t)s.ntr * s.ns * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FWI_OK;
}

extern "C" int fwi_ctx_get_gradient(fwi_ctx *c, float *out)
{
    if (!c || !out) return fail(FWI_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(out, c->d_grad, (size_t)c->nz * c->nx * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FWI_OK;
}

extern "C" const float *fwi_ctx_traces_device(fwi_ctx *c, int ishot)
{
    if (!c || ishot < 0 || ishot >= (int)c->shots.size()) return nullptr;
    return c->d_pre[ishot];
}
extern "C" const float *fwi_ctx_gradient_device(fwi_ctx *c) { return c ? c->d_grad : nullptr; }

extern "C" int fwi_ctx_objective(fwi_ctx *c, double *out)
{
    if (!c || !out) return fail(FWI_ERR_ARG, "NULL argument");
    CK(cudaSetDevice(c->device));
    double acc = 0.0;
    std::vector<SumDesc> sd;
    for (size_t i = 0; i < c->shots.size(); i++) {
        SumDesc s{};
        s.a = c->d_pre[i];
        s.n = (long long)c->shots[i].s.ntr * c->shots[i].s.ns;
        s.op = 1;
        sd.push_back(s);
    }
    for (size_t i0 = 0; i0 < sd.size(); i0 += 64) {
        std::vector<SumDesc> part(sd.begin() + i0, sd.begin() + std::min(sd.size(), i0 + 64));
        std::vector<double> h;
        TRY(reduce(c, part, h));
        for (size_t i = 0; i < part.size(); i++) acc += h[2 * i];
    }
    TRY(exchange_scalars(c, &acc, 1));
    *out = 0.5 * acc;
    return FWI_OK;
}

extern "C" int fwi_ctx_set_autotune(fwi_ctx *c, int on)
{
    if (!c) return fail(FWI_ERR_ARG, "ctx is NULL");
    c->tune = on != 0;
    return FWI_OK;
}

extern "C" int fwi_ctx_launch_shape(fwi_ctx *c, int *tile_columns, int *ring_depth, int *shots_per_block)
{
    if (!c) return fail(FWI_ERR_ARG, "ctx is NULL");
    if (tile_columns) *tile_columns = c->last_tx;
    if (ring_depth) *ring_depth = c->last_nst;
    if (shots_per_block) *shots_per_block = c->last_chunk;
    return FWI_OK;
}

extern "C" int fwi_ctx_launch_variant(fwi_ctx *c, int *groups_per_thread, int *blocks_per_sm)
{
    if (!c) return fail(FWI_ERR_ARG, "ctx is NULL");
    if (groups_per_thread) *groups_per_thread = c->last_gpt;
    if (blocks_per_sm) *blocks_per_sm = c->last_minb;
    return FWI_OK;
}

extern "C" int fwi_ctx_launch_persistent(fwi_ctx *c, int *persistent)
{
    if (!c) return fail(FWI_ERR_ARG, "ctx is NULL");
    if (persistent) *persistent = c->last_wave ? 1 : 0;
    return FWI_OK;
}

extern "C" int fwi_ctx_set_graphs(fwi_ctx *c, int on)
{
    if (!c) return fail(FWI_ERR_ARG, "ctx is NULL");
    if (!on) drop_graphs(c);
    c->use_graphs = on != 0;
    return FWI_OK;
}

// Device bytes a context needs for one run of `problem` over these shots: the allocations of
// set_model / set_shots / prepare_run / assign_pool / the FFT stage, with a margin for the
// reduction, descriptor and library workspaces.  A serving loop admits requests by it.
extern "C" size_t fwi_estimate_bytes(const fwi_shot *shots, int nshot, int nz, int nx, int nt, int pml, int problem,
                                     int filter)
{
    if (!shots || nshot <= 0 || nz <= 0 || nx <= 0 || nt <= 0 || pml < 0) return 0;
    const size_t m = (size_t)nz * nx;
    size_t b = 4 * m * 4 + 2 * m * 8;  // vp, rho, grad, prec; FP64 stacks of g and H
    const bool grad = problem == 1;
    const int d = fwi_ck_interval(nt), K = (nt - 1) / d, S5 = d / MST + 2;
    std::set<std::pair<int, int>> windows;
    size_t max_ns = 1, max_ntr = 1;
    for (int i = 0; i < nshot; i++) {
        const fwi_shot &s = shots[i];
        const int nxx = s.ix_max - s.ix_min + 1;
        const size_t Nx = (size_t)nxx + 2 * pml, Nz = (size_t)nz + 2 * pml, ld = (Nz + 3) / 4 * 4;
        const size_t frame = Nx * ld, rec = (size_t)s.ntr * s.ns;
        windows.insert({s.ix_min, s.ix_max});
        b += 3 * rec * 4;                                                // observed, predicted, line-search gathers
        b += (size_t)nt * 12 + (Nx + 1) * 4 + (size_t)s.ntr * 16 + rec * 4;  // source terms, receivers, samples
        b += ((size_t)s.ns + 1 + s.ntr + 1) * 4;                         // taper coefficients
        b += (grad ? (size_t)nframes_gradient(K, S5) : NROT) * frame * 4;  // frame block in the pool
        if (grad) b += 2 * frame * 8 + (size_t)nt * s.ntr * 4 + 2 * (size_t)nz * nxx * 4;
        max_ns = std::max(max_ns, (size_t)s.ns);
        max_ntr = std::max(max_ntr, (size_t)s.ntr);
    }
    for (auto &w : windows) {
        const size_t Nx = (size_t)(w.second - w.first + 1) + 2 * pml, Nz = (size_t)nz + 2 * pml;
        b += 6 * Nx * ((Nz + 3) / 4 * 4) * 4;  // coefficient planes of the window
    }
    // FFT convolution tables: spectra and twiddles of the time and trace filters and of the
    // interpolation (2 M floats each), and the filters' intermediate gather
    const size_t Mt = (size_t)fwi_conv_size((int)std::max(max_ns, (size_t)nt)), Mx = (size_t)fwi_conv_size((int)max_ntr);
    if ((grad || problem == 2) && (filter == 0 || filter == 1)) b += max_ns * max_ntr * 4 + 8 * (Mt + Mx) * 4;
    if (grad) b += 4 * Mt * 4;
    b += (size_t)nshot * sizeof(ShotDesc) + ((size_t)3 * nt + 64) * sizeof(int4) + (8u << 20);
    return b + b / 20 + (96u << 20);  // 5 % and 96 MiB for the library workspaces and graphs
}

extern "C" int fwi_adjoint_program(int nt, int overlap, int *items, int cap)
{
    if (nt <= 0) return 0;
    std::vector<int4> p = overlap == 2 ? program_adjoint2(nt) : program_adjoint(nt, overlap != 0);
    if (items)
        for (int i = 0; i < (int)p.size() && i < cap; i++) {
            items[4 * i] = p[i].x;
            items[4 * i + 1] = p[i].y;
            items[4 * i + 2] = p[i].z;
            items[4 * i + 3] = p[i].w;
        }
    return (int)p.size();
}

extern "C" int fwi_checkpoint_interval(int nt) { return fwi_ck_interval(nt); }

extern "C" int fwi_ctx_stats(fwi_ctx *c, fwi_stats *out)
{
    if (!c || !out) return fail(FWI_ERR_ARG, "NULL argument");
    *out = c->stats;
    return FWI_OK;
}

extern "C" int fwi_ctx_pass_stats(fwi_ctx *c, double *fwd_ms, long long *fwd_launches, double *adj_ms,
                                  long long *adj_launches)
{
    if (!c) return fail(FWI_ERR_ARG, "NULL context");
    if (fwd_ms) *fwd_ms = c->pass[0].ms;
    if (fwd_launches) *fwd_launches = c->pass[0].launches;
    if (adj_ms) *adj_ms = c->pass[1].ms;
    if (adj_launches) *adj_launches = c->pass[1].launches;
    return FWI_OK;
}

// ------------------------------------------------------------------ engine drop-in
// iso_acoustic2d_propagation_engine with the reference's checkpoint object: mode 1 runs
// the forward pass into a context owned by the checkpoint object (its frames stay on
// the device), mode 2 runs the adjoint pass from them.  Mode 0 uses a shared context.
namespace {
struct CkImpl {
    fwi_ctx *ctx = nullptr;
    bool forward_done = false;
};
fwi_ctx *g_engine_ctx = nullptr;

bool rows_contiguous(float **rows, int n1, int n2)
{
    for (int i = 1; i < n2; i++)
        if (rows[i] != rows[0] + (size_t)i * n1) return false;
    return true;
}
}  // namespace

// [ntr][ns] host adjoint source -> adj_t [nt][ntr] on the device (interpolate_traces with r = 1 is a copy)
static __global__ void k_to_time_major(const float *__restrict__ a, float *__restrict__ out, int ntr, int ns, int nt)
{
    long long n = (long long)ntr * nt;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int k = (int)(i / ntr), r = (int)(i % ntr);
        out[i] = k < ns ? a[(long long)r * ns + k] : 0.0f;
    }
}

extern "C" void acoustic2dCheckPoint_init(Acoustic2dCheckPoint *chk)
{
    if (chk) memset(chk, 0, sizeof(*chk));
}

extern "C" void alloc_acoustic2dCheckPoint(Acoustic2dCheckPoint *chk, int NZ, int NX, int nt)
{
    if (!chk) return;
    free_acoustic2dCheckPoint(chk);
    chk->nt = nt;
    chk->dCheckPoint = fwi_ck_interval(nt);
    chk->nCheckPoint = fwi_ck_count(nt);
    chk->ntPoint = chk->nCheckPoint + chk->dCheckPoint - 2;
    chk->memCost = 1.0f * (chk->ntPoint * NZ * NX * (int)sizeof(float)) / powf(1024.0f, 3);
    chk->impl = new CkImpl();
}

extern "C" void free_acoustic2dCheckPoint(Acoustic2dCheckPoint *chk)
{
    if (!chk || !chk->impl) return;
    CkImpl *k = (CkImpl *)chk->impl;
    if (k->ctx) fwi_ctx_destroy(k->ctx);
    delete k;
    chk->impl = nullptr;
}

extern "C" int fwi_iso_acoustic2d_propagation_engine(Record2D *r, Acoustic2dCheckPoint *chk, float **vpm, float **rhom,
                                                     int nx, int nz, float dx, float dz, float dt, int nt, int pml,
                                                     int fs, int precondition, int mode, int iter, int verbose,
                                                     float **grad)
{
    if (!r || !vpm || !rhom || mode < 0 || mode > 2) return fail(FWI_ERR_ARG, "invalid engine arguments");
    if (!rows_contiguous(vpm, nz, nx) || !rows_contiguous(rhom, nz, nx))
        return fail(FWI_ERR_ARG, "vpm/rhom must be one contiguous block (alloc2float layout)");
    if (mode > 0 && (!chk || !chk->impl)) return fail(FWI_ERR_STATE, "modes 1 and 2 need an allocated checkpoint");
    if (mode == 2 && !grad) return fail(FWI_ERR_ARG, "mode 2 writes the gradient: grad is NULL");
    fwi_ctx *c;
    CkImpl *k = mode > 0 ? (CkImpl *)chk->impl : nullptr;
    if (mode == 0) {
        if (!g_engine_ctx) TRY(fwi_ctx_create(&g_engine_ctx, 0, 0));
        c = g_engine_ctx;
    } else {
        if (!k->ctx) TRY(fwi_ctx_create(&k->ctx, 0, 0));
        c = k->ctx;
    }
    // the engine writes only snapshots (verbose > 1); the per-shot files are the driver's
    TRY(fwi_ctx_set_verbose(c, verbose > 1 ? verbose : 0, iter, 0, 0, nullptr));
    fwi_shot s{};
    s.shotID = r->shotID; s.isx = r->isx; s.isz = r->isz; s.ntr = r->ntr; s.ns = r->ns;
    s.sampleRate = r->sampleRate; s.ix_min = 0; s.ix_max = nx - 1;  // vpm is the shot's window already
    s.dt = r->dt; s.dtr = r->dtr; s.fpeak = r->fpeak;
    s.src = r->src; s.igx = r->igx; s.igz = r->igz;
    if (mode == 2) {
        if (!k->forward_done) return fail(FWI_ERR_STATE, "mode 2 before mode 1 on this checkpoint");
        if (r->sampleRate > 1) return fail(FWI_ERR_UNSUPPORTED, "sampleRate > 1 needs FFT trace interpolation (not built)");
        CK(cudaSetDevice(c->device));
        ShotRun *sr = c->runs[0].get();
        const size_t nb = (size_t)r->ntr * r->ns * 4;
        CK(cudaMemcpyAsync(c->d_pre[0], r->traces_p[0], nb, cudaMemcpyHostToDevice, c->stream));
        k_to_time_major<<<296, 256, 0, c->stream>>>(c->d_pre[0], (float *)sr->d.adj_t, r->ntr, r->ns, nt);
        CK(cudaGetLastError());
        std::vector<ShotRun *> rs = {sr};
        TRY(grad_adjoint(c, rs, false, "", 0));
        CK(cudaMemcpyAsync(grad[0], sr->d_gshot, (size_t)nx * nz * 4, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return check_kernel_error(c);
    }
    TRY(fwi_ctx_set_model(c, vpm[0], rhom[0], nz, nx, dx, dz, dt, nt, pml, fs));
    TRY(fwi_ctx_set_shots(c, &s, 1));
    if (mode == 0) {
        TRY(fwi_ctx_run(c, 0, 0.0f, 2, 0, FWI_PATH_PLAIN));
        return fwi_ctx_get_traces(c, 0, r->traces_p[0]);
    }
    // mode 1
    CK(cudaSetDevice(c->device));
    if (c->runs.size() != 1) {
        free_runs(c);
        c->runs.emplace_back(new ShotRun());
    }
    ShotRun *sr = c->runs[0].get();
    TRY(prepare_run(c, sr, 0, true));
    sr->d.hessian = precondition == 1;
    TRY(assign_pool(c, -1, {sr}));
    TRY(upload_descs(c, {sr->d}));
    std::vector<ShotRun *> rs = {sr};
    TRY(grad_forward(c, rs, precondition, false, "", 0));
    TRY(gather(c, rs, 0, false));
    TRY(fwi_ctx_get_traces(c, 0, r->traces_p[0]));
    if (precondition == 1 && grad)
        CK(cudaMemcpyAsync(grad[0], sr->d_hshot, (size_t)nx * nz * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    TRY(check_kernel_error(c));
    k->forward_done = true;
    return FWI_OK;
}

extern "C" void iso_acoustic2d_propagation_engine(Record2D *r, Acoustic2dCheckPoint *chk, float **vpm, float **rhom,
                                                  int nx, int nz, float dx, float dz, float dt, int nt, int pml, int fs,
                                                  int precondition, int mode, int iter, int verbose, float **grad)
{
    int rc = fwi_iso_acoustic2d_propagation_engine(r, chk, vpm, rhom, nx, nz, dx, dz, dt, nt, pml, fs, precondition, mode,
                                                   iter, verbose, grad);
    if (rc != FWI_OK)
        fprintf(stderr, "<error>: iso_acoustic2d_propagation_engine failed (status %d): %s\n", rc, g_err.c_str());
}

// ------------------------------------------------------------------ FWI iteration
extern "C" int fwi_ctx_get_model(fwi_ctx *c, float *vp, float *rho)
{
    if (!c || !vp || !rho || !c->host_model_valid) return fail(FWI_ERR_ARG, "no model");
    memcpy(vp, c->vp.data(), c->vp.size() * 4);
    memcpy(rho, c->rho.data(), c->rho.size() * 4);
    return FWI_OK;
}

static std::vector<float> smooth_weights(int N)
{
    std::vector<float> w(2 * N + 1);
    for (int i = 0; i < 2 * N + 1; i++) {  // common.c:955-961: double cosine, squared in float
        w[i] = (float)cos(3.141592653589793 * (i - N) / (2.0 * N));
        w[i] *= w[i];
    }
    return w;
}

static int sum_gathers(fwi_ctx *c, const std::vector<float *> &a, const std::vector<float *> *b, int op, double *s0,
                       double *s1)
{
    *s0 = 0.0;
    if (s1) *s1 = 0.0;
    std::vector<SumDesc> sd;
    for (size_t i = 0; i < c->shots.size(); i++) {
        SumDesc d{};
        d.a = a[i];
        d.b = b ? (*b)[i] : nullptr;
        d.n = (long long)c->shots[i].s.ntr * c->shots[i].s.ns;
        d.op = op;
        sd.push_back(d);
    }
    for (size_t i0 = 0; i0 < sd.size(); i0 += 64) {
        std::vector<SumDesc> part(sd.begin() + i0, sd.begin() + std::min(sd.size(), i0 + 64));
        std::vector<double> h;
        TRY(reduce(c, part, h));
        for (size_t i = 0; i < part.size(); i++) {  // shots in order, as the reference's outer loop
            *s0 += h[2 * i];
            if (s1) *s1 += h[2 * i + 1];
        }
    }
    return FWI_OK;
}

// one pass of the loop body of acoustic2d_fwi.c:411-465
extern "C" int fwi_ctx_fwi_iteration(fwi_ctx *c, const fwi_iter_params *p, fwi_iter_result *out)
{
    if (!c || !p || !out) return fail(FWI_ERR_ARG, "NULL argument");
    if (!c->host_model_valid || c->shots.empty()) return fail(FWI_ERR_STATE, "set the model, shots and data first");
    if (p->rx < 1 || p->rz < 1) return fail(FWI_ERR_ARG, "smoothing half-widths must be >= 1");
    CK(cudaSetDevice(c->device));
    const int nx = c->nx, nz = c->nz;
    const size_t m = (size_t)nx * nz;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, c->stream));
    long long l0 = c->launches;
    if (c->slow.size() != m) {  // v2slow of the starting model (acoustic2d_fwi.c:365)
        c->slow.resize(m);
        for (size_t i = 0; i < m; i++) c->slow[i] = c->vp[i] != 0.0f ? 1.0f / c->vp[i] : 0.0f;
    }
    // gradient
    TRY(fwi_ctx_run(c, 1, p->freq, p->filter, p->precondition, p->path));
    double cells = c->stats.cell_updates;
    // smoothing along z then x (acoustic2d_fwi.c:418-419), fun1, perturbation, all on the device
    std::vector<float> wz = smooth_weights(p->rz), wx = smooth_weights(p->rx);
    float *d_work;
    const size_t nb = ((m * 4 + 255) / 256) * 256;
    TRY(scratch(c, 3 * nb + 4096 + sizeof(PertState) + 1024, (void **)&d_work));
    float *d_tmp = d_work, *d_slow = (float *)((char *)d_work + nb), *d_pert = (float *)((char *)d_work + 2 * nb);
    float *d_w = (float *)((char *)d_work + 3 * nb);
    PertState *d_st = (PertState *)((char *)d_work + 3 * nb + 4096);
    if ((size_t)(2 * p->rz + 1 + 2 * p->rx + 1) * 4 > 4096) return fail(FWI_ERR_ARG, "smoothing window too wide");
    CK(cudaMemcpyAsync(d_w, wz.data(), wz.size() * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_w + wz.size(), wx.data(), wx.size() * 4, cudaMemcpyHostToDevice, c->stream));
    k_smooth2d<<<592, 256, 0, c->stream>>>(c->d_grad, d_tmp, nx, nz, p->rz, 1, d_w);
    k_smooth2d<<<592, 256, 0, c->stream>>>(d_tmp, c->d_grad, nx, nz, p->rx, 0, d_w + wz.size());
    c->launches += 2;
    double f1;
    TRY(sum_gathers(c, c->d_pre, nullptr, 1, &f1, nullptr));
    TRY(exchange_scalars(c, &f1, 1));
    const float fun1 = (float)(0.5 * f1);
    CK(cudaMemcpyAsync(d_slow, c->slow.data(), m * 4, cudaMemcpyHostToDevice, c->stream));
    SumDesc sd{};
    sd.a = d_slow;
    sd.n = (long long)m;
    sd.op = 0;
    std::vector<double> hs;
    double *d_ssum;
    TRY(reduce(c, {sd}, hs, &d_ssum));
    k_pert_init<<<1, 256, 0, c->stream>>>(d_st);
    k_pert_minmax<<<296, 256, 0, c->stream>>>(c->d_grad, (long long)m, d_st);
    k_pert_hist<<<296, 256, 0, c->stream>>>(c->d_grad, (long long)m, d_st);
    k_pert_scalar<<<1, 32, 0, c->stream>>>(d_st, d_ssum, (long long)m, 0.01f);
    k_pert_apply<<<296, 256, 0, c->stream>>>(c->d_grad, d_pert, (long long)m, d_st);
    c->launches += 5;
    CK(cudaGetLastError());
    std::vector<float> pert(m);
    float scalar = 0.0f;
    CK(cudaMemcpyAsync(pert.data(), d_pert, m * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&scalar, &d_st->scalar, 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    // the output gradient has its water rows zeroed (acoustic2d_fwi.c:425)
    for (int ix = 0; ix < nx && p->waterdepth > 0; ix++)
        CK(cudaMemsetAsync(c->d_grad + (size_t)ix * nz, 0, (size_t)std::min(p->waterdepth, nz) * 4, c->stream));
    // trial model on the host with the C library's powf (Gardner), then the line-search forward
    std::vector<float> vp0 = c->vp, rho0 = c->rho, vpt(m), rhot(m);
    rhot = rho0;
    fwi_model_trial(c->slow.data(), pert.data(), vpt.data(), rhot.data(), nx, nz, p->waterdepth, p->vp_water,
                    p->rho_water, p->vpmin, p->vpmax, p->rhomin, p->rhomax, p->gardner);
    TRY(fwi_ctx_set_model(c, vpt.data(), rhot.data(), nz, nx, c->dx, c->dz, c->dt, c->nt, c->pml, c->fs));
    std::swap(c->d_pre, c->d_pre_alt);  // keep the gradient's residuals: problem 2 writes the other set
    int rc = fwi_ctx_run(c, 2, p->freq, p->filter, p->precondition, p->path);
    if (rc != FWI_OK) {
        std::swap(c->d_pre, c->d_pre_alt);
        return rc;
    }
    cells += c->stats.cell_updates;
    double f2, num, den;
    TRY(sum_gathers(c, c->d_pre, nullptr, 1, &f2, nullptr));
    TRY(sum_gathers(c, c->d_pre_alt, &c->d_pre, 3, &num, &den));
    {
        double v[3] = {f2, num, den};
        TRY(exchange_scalars(c, v, 3));
        f2 = v[0]; num = v[1]; den = v[2];
    }
    const float fun2 = (float)(0.5 * f2);
    const float steplen = den == 0.0 ? 0.0f : (float)(num / den);
    // model update (acoustic2d_fwi.c:452-465)
    std::vector<float> vpn = vp0, rhon = rho0;
    fwi_model_update(c->slow.data(), vpn.data(), rhon.data(), pert.data(), steplen, nx, nz, p->waterdepth,
                     p->vp_water, p->rho_water, p->vpmin, p->vpmax, p->rhomin, p->rhomax, p->gardner);
    TRY(fwi_ctx_set_model(c, vpn.data(), rhon.data(), nz, nx, c->dx, c->dz, c->dt, c->nt, c->pml, c->fs));
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out->fun1 = fun1;
    out->fun2 = fun2;
    out->steplen = steplen;
    out->scalar = scalar;
    out->ms = ms;
    out->cell_updates = cells;
    out->kernel_launches = c->launches - l0;
    return FWI_OK;
}

// ------------------------------------------------------------------ continuous batching
#include "fwi_exec.cuh"
