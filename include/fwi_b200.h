/*
 * fwi_b200.h -- C-ABI of the B200 (sm_100a) 2-D acoustic forward/adjoint engine.
 *
 * Two layers:
 *
 * 1. Drop-in entry points with the names, argument meaning and effects of the
 *    FWI-EDU C implementation (FWILab2dCLangV1.2.6).  A front-end written against
 *    the reference links against this library instead and runs unchanged.  Each
 *    declaration cites the reference declaration it replaces.  Where the reference
 *    calls err() and exits, these print the same kind of message and return; the
 *    matching fwi_* entry point returns the status code instead.
 *
 * 2. The native API (fwi_ctx_*): a device-resident context that keeps the model,
 *    coefficients, wavelets, traces, checkpoints and gradients in HBM, runs shots
 *    one per launch ("plain") or many shots per launch ("batched"), and hands
 *    results back on request.  Plain pointers and sizes only.
 *
 * Array layout everywhere: the reference's alloc2float(n1, n2) layout -- n2 rows of
 * n1 contiguous floats -- so models are [nx][nz] with z fastest and trace gathers are
 * [ntr][ns] with time fastest.  float** arguments must point into ONE contiguous
 * block (rows[i] == rows[0] + i*n1), as alloc2float returns.
 */
#ifndef FWI_B200_H
#define FWI_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FWI_API __attribute__((visibility("default")))
#else
#define FWI_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum {
    FWI_OK = 0,
    FWI_ERR_ARG = 1,        /* invalid argument (sizes, indices, NULL pointers) */
    FWI_ERR_CUDA = 2,       /* a CUDA runtime call failed */
    FWI_ERR_NOMEM = 3,      /* device or host allocation failed / over the context budget */
    FWI_ERR_UNSUPPORTED = 4,/* a reference option this build does not implement */
    FWI_ERR_NODEVICE = 5,   /* no CUDA device: the engine has no CPU fallback */
    FWI_ERR_STATE = 6       /* call order (e.g. adjoint before forward) */
};
/* message of the last failure on the calling thread ("" if none) */
FWI_API const char *fwi_last_error(void);
/* library version string */
FWI_API const char *fwi_version(void);

/* ------------------------------------------------ reference types (drop-in) */

/* shot record; identical layout to Record2D, observation.h:18-48 */
typedef struct {
    int shotID;
    float sx, sz;
    int isx, isz;        /* source grid index: window-local x, global z */
    float fpeak;
    float *src;          /* nt */
    float *gx, *gz;      /* ntr receiver coordinates (m) */
    int *igx, *igz;      /* ntr: window-local x, global z */
    int sampleRate;
    int ntr, ns;
    float dtr, dt;
    int ix_min, ix_max;
    float **traces_vx, **traces_vz, **traces_p; /* traces_p: [ntr][ns] */
    float **precond, **grad;
} Record2D;

/* wavefield checkpoint store of one shot.  Same name and life cycle as
 * Acoustic2dCheckPoint, checkpoint.h:16-26 (init, alloc, engine mode 1 fills it,
 * engine mode 2 consumes it, free); here the frames live in device memory. */
typedef struct {
    int nt, dCheckPoint, nCheckPoint, ntPoint;
    float memCost;        /* GB the reference would hold for the same store */
    void *impl;           /* device-side store, owned by this library */
} Acoustic2dCheckPoint;

/* replaces iso_acoustic2d_propagation, propagation.h:133-142 (propagation.c:777-1036):
 * problem 0 forward modeling into record2d_pre[i].traces_p; problem 1 gradient into
 * grad (and the adjoint source into record2d_pre); problem 2 forward + residual in place. */
FWI_API void iso_acoustic2d_propagation(float **vp, float **rho, Record2D *record2d_obs, int Nshot, int nz, int nx,
                                float dx, float dz, float dt, int nt, int pmlThick, int freesurface,
                                float freq, float filter, int precondition, int problem, int iter,
                                int verbose, Record2D *record2d_pre, float **grad);
/* same contract, returns FWI_OK or an error code instead of exiting */
FWI_API int fwi_iso_acoustic2d_propagation(float **vp, float **rho, Record2D *record2d_obs, int Nshot, int nz, int nx,
                                   float dx, float dz, float dt, int nt, int pmlThick, int freesurface,
                                   float freq, float filter, int precondition, int problem, int iter,
                                   int verbose, Record2D *record2d_pre, float **grad);

/* replaces iso_acoustic2d_propagation_engine, propagation.h:95-101 (propagation.c:356-775):
 * mode 0 forward, mode 1 forward + checkpoints (+ pseudo-Hessian into grad when
 * precondition == 1), mode 2 adjoint from the checkpoints, gradient into grad.
 * vpm/rhom are the shot's window (nz x nx). */
FWI_API void iso_acoustic2d_propagation_engine(Record2D *record2d, Acoustic2dCheckPoint *chkpt, float **vpm,
                                       float **rhom, int nx, int nz, float dx, float dz, float dt, int nt,
                                       int pmlThick, int freesurface, int precondition, int mode, int iter,
                                       int verbose, float **grad);
FWI_API int fwi_iso_acoustic2d_propagation_engine(Record2D *record2d, Acoustic2dCheckPoint *chkpt, float **vpm,
                                          float **rhom, int nx, int nz, float dx, float dz, float dt, int nt,
                                          int pmlThick, int freesurface, int precondition, int mode, int iter,
                                          int verbose, float **grad);

/* replace the checkpoint.h:27-165 life cycle (checkpoint.c:13-128, 267-298) */
FWI_API void acoustic2dCheckPoint_init(Acoustic2dCheckPoint *chkpt);
FWI_API void alloc_acoustic2dCheckPoint(Acoustic2dCheckPoint *chkpt, int NZ, int NX, int nt);
FWI_API void free_acoustic2dCheckPoint(Acoustic2dCheckPoint *chkpt);
FWI_API float calculate_memory_cost_checkpoint(int nt, int NX, int NZ);

/* common.c:584-687 / :689-794 / :482-582 (common.h): the residual filters (FFT, cosine-tapered
 * low/band-pass window, inverse FFT, / nt) of ntr traces of nt samples, and the interpolation
 * of ntr traces from nt to (nt - 1) r + 1 samples (zero-stuffing, rectangular band window).
 * Arrays in the alloc2float layout.  On the GPU as GEMMs with the equivalent operator matrices
 * (FP32 within 1e-6 relative of the transforms). */
FWI_API void apply_traces_lowpass(float **tr, float **trs, int nt, int ntr, float fpass, float fcut, float dt);
FWI_API void apply_traces_bandpass(float **tr, float **trs, int nt, int ntr, float fpass, float fcut, float dt);
FWI_API void interpolate_traces(float **tr, int ntr, int nt, int r, float **trs);

/* common.c:1042-1162 / :1164-1284 (common.h): the 2-D wavenumber low/band-pass of an nz x nx field
 * (s[ix][iz], alloc2float(nz, nx)).  As the reference: the cosine taper of taper_traces with
 * lengths roundf(4 / (kpass d)) is applied to s IN PLACE, the field is padded by 10 x the longer
 * taper with replicated edges, transformed, multiplied by the radial cosine window between kpass
 * and kcut (1/m), transformed back, / (Nz Nx) and cropped into s_filter (which may be s).  On the
 * GPU as FP32 GEMMs with DFT operators that fold the pad and the crop (within 1e-5 relative of
 * the FFTs).  kcut <= kpass or kpass <= 0 prints an error and leaves both arrays unchanged. */
FWI_API void lowpass2d(float **s, int nz, int nx, float dz, float dx, float kpass, float kcut, float **s_filter);
FWI_API void bandpass2d(float **s, int nz, int nx, float dz, float dx, float kpass, float kcut, float **s_filter);

/* replace the optimization.h reductions (optimization.c:13-298), computed on the device */
FWI_API void apply_gradient_precondition(float *grad, const float *precond, int n, float alpha);
FWI_API void apply_gradient_shot_precondition(float *grad, float *precond, int n);
FWI_API float calculate_objective_value(Record2D *record2d, int Nshot);
FWI_API float calculate_step_length(Record2D *record2d_pre0, Record2D *record2d_pre1, int Nshot);
FWI_API float compute_model_perturbation(float fraction, float *slowness, float *gradient, float *out, int len);
/* replaces compute_adjoint_source2d, optimization.h:17-19 (optimization.c:300-419) */
FWI_API void compute_adjoint_source2d(Record2D *record2d_pre, Record2D *record2d_obs, float **vp, float freq,
                              int filter, Record2D *record2d_adjsource);
/* replaces smooth2D, common.h (common.c:927-1040) */
FWI_API void smooth2D(float **in, float **out, int nx, int nz, int N, int iszdirect);

/* ------------------------------------------------------------ native API */

typedef struct fwi_ctx fwi_ctx;

/* one shot in flat form (the Record2D fields the engine reads) */
typedef struct {
    int shotID;          /* 1-based */
    int isx, isz;        /* window-local x, global z */
    int ntr, ns, sampleRate;
    int ix_min, ix_max;  /* model window, inclusive */
    float dt;            /* record sample interval */
    float dtr;           /* receiver interval (m) */
    float fpeak;         /* wavelet peak frequency (Hz) */
    const float *src;    /* nt samples */
    const int *igx;      /* ntr, window-local */
    const int *igz;      /* ntr, global */
} fwi_shot;

/* execution paths of fwi_ctx_run */
enum {
    FWI_PATH_PLAIN = 0,   /* one shot per launch, one launch per time step (the straight port) */
    FWI_PATH_BATCHED = 1  /* all shots of a batch per launch, time loop captured as CUDA graphs */
};

/* device_budget_bytes: 0 = no cap; otherwise allocations beyond it fail with FWI_ERR_NOMEM */
FWI_API int fwi_ctx_create(fwi_ctx **ctx, int device, size_t device_budget_bytes);
FWI_API int fwi_ctx_destroy(fwi_ctx *ctx);
/* model on the global grid (host arrays [nx][nz]) and the run constants */
FWI_API int fwi_ctx_set_model(fwi_ctx *ctx, const float *vp, const float *rho, int nz, int nx, float dx, float dz,
                      float dt, int nt, int pmlThick, int freesurface);
/* same, from device pointers (no host copy) */
FWI_API int fwi_ctx_set_model_device(fwi_ctx *ctx, const float *d_vp, const float *d_rho, int nz, int nx, float dx,
                             float dz, float dt, int nt, int pmlThick, int freesurface);
FWI_API int fwi_ctx_set_shots(fwi_ctx *ctx, const fwi_shot *shots, int nshot);
/* observed gathers: one host array [ntr][ns] per shot.  The upload runs on a stream of its own,
 * overlapping the next run's forward pass: page-locked arrays are read after the call returns, so
 * keep them unchanged until the next fwi_ctx_run (or fwi_ctx_destroy) returns; pageable arrays
 * are staged before the call returns. */
FWI_API int fwi_ctx_set_observed(fwi_ctx *ctx, const float *const *obs);
/* problem 0/1/2 as iso_acoustic2d_propagation; results stay on the device */
FWI_API int fwi_ctx_run(fwi_ctx *ctx, int problem, float freq, int filter, int precondition, int path);
/* copy results back: predicted / residual gathers of one shot, gradient [nx][nz] */
FWI_API int fwi_ctx_get_traces(fwi_ctx *ctx, int ishot, float *out);
FWI_API int fwi_ctx_get_gradient(fwi_ctx *ctx, float *out);
/* device pointers of the results (valid until the next run / set call) */
FWI_API const float *fwi_ctx_traces_device(fwi_ctx *ctx, int ishot);
FWI_API const float *fwi_ctx_gradient_device(fwi_ctx *ctx);
/* device-side FP64 misfit 0.5*sum(r^2) over the current residual gathers */
FWI_API int fwi_ctx_objective(fwi_ctx *ctx, double *out);
/* statistics of the last run */
typedef struct {
    double ms;               /* device time of the run (CUDA events) */
    double cell_updates;     /* stencil applications (padded cells x steps) */
    long long kernel_launches;
    long long graph_launches;
    size_t device_bytes;     /* device memory held by the context */
} fwi_stats;
FWI_API int fwi_ctx_stats(fwi_ctx *ctx, fwi_stats *out);
/* device time and step-kernel launches of the last run's passes: the forward passes (modeling,
 * or the checkpointing forward of a gradient) and the adjoint passes (each launch a replay step
 * and an adjoint step of every shot of the group), summed over shot groups and waves; the
 * autotuner's probes are not included */
FWI_API int fwi_ctx_pass_stats(fwi_ctx *ctx, double *fwd_ms, long long *fwd_launches, double *adj_ms,
                               long long *adj_launches);

/* The step kernel's launch shape (tile width 8/16 columns, z-groups per thread, blocks per SM it
 * is compiled for, shared-memory ring depth 2..4 shots, shots per block) is picked by an
 * autotuner: the first run of a launch shape (padded grid, shots per launch, arithmetic, path)
 * times the candidates on the run's own scratch frames and keeps the fastest for the process; on
 * the batched path it also tunes the halo depth (one time step per launch, or two with the
 * temporal-blocking kernel) and the context keeps the faster (FWI_DEPTH=1|2 pins it).
 * Off (or FWI_TUNE=0; or any of FWI_TX / FWI_NST / FWI_CHUNK / FWI_GPT / FWI_OCC set): a built-in
 * heuristic with those overrides.  fwi_ctx_launch_shape and fwi_ctx_launch_variant report the
 * shape of the last launch. */
FWI_API int fwi_ctx_set_autotune(fwi_ctx *ctx, int on);
FWI_API int fwi_ctx_launch_shape(fwi_ctx *ctx, int *tile_columns, int *ring_depth, int *shots_per_block);
/* the rest of the last launch's shape: z-groups per consumer thread (1 or 2) and the blocks per SM
 * the step kernel was compiled for (1: no minimum, coefficients in registers; 3: coefficients
 * read from shared memory).  No counterpart in the reference. */
FWI_API int fwi_ctx_launch_variant(fwi_ctx *ctx, int *groups_per_thread, int *blocks_per_sm);
/* 1 when the last pass ran as one persistent wavefront launch.  With FWI_PERSIST=1 in the
 * environment (default off), a forward pass on the batched path (modeling, or the checkpointing
 * forward of a gradient) whose 16-column tiles times shot ranges of 2..32 shots fit the GPU's
 * resident blocks runs as a single cooperative launch in which every block owns one tile and shot
 * range for all steps and waits only for its neighbouring tiles' previous step; results are the
 * step launches' bit for bit.  Off by default because it is slower on the benchmark survey (57.8
 * against 43.6 us per step, 60 shots on 221 x 601): its tiles are assigned once, so the tiles with
 * the free surface and the sources pace the whole grid, where the step launches' blocks balance
 * them.  The shape functions then report that launch.  No counterpart in the reference. */
FWI_API int fwi_ctx_launch_persistent(fwi_ctx *ctx, int *persistent);

/* CUDA graphs on the batched path (default on; FWI_GRAPH=0 in the environment turns them off):
 * off, every step is launched directly -- cheaper for a launch sequence run only once. */
FWI_API int fwi_ctx_set_graphs(fwi_ctx *ctx, int on);

/* The reference's verbose output (replaces the `verbose`/`iter` arguments and the shotInterval /
 * snapInterval environment variables of iso_acoustic2d_propagation, propagation.c:423-441,
 * 846-852).  verbose >= 1: a gradient run (problem 1) writes, for every shot_interval-th shot,
 * predicted_iter*_shot*.bin, adjsource_iter*_shot*.bin and gradient_raw_iter*_shot*.bin, and
 * per gradient gradient_raw_iter*.bin and precond_iter*.bin (propagation.c:917-944, 996-1005);
 * verbose > 1: also wavefield snapshots every snap_interval steps of the shots whose
 * (shotID - 1) % shot_interval == 0 (wavefield_forward*, wavefield_forward_reconstruction*,
 * wavefield_backward*, propagation.c:597-601, 717-723; the reconstructed field is written at
 * imaging steps, multiples of 5).  Raw float32 files with the reference's names, in `dir` (NULL:
 * the working directory, as the reference).  shot_interval / snap_interval <= 0: read from the
 * environment variables shotInterval / snapInterval, defaults 20 / 1000.  Snapshot runs launch
 * the step kernel directly (no CUDA graphs) and copy every snapshot out as it is produced. */
FWI_API int fwi_ctx_set_verbose(fwi_ctx *ctx, int verbose, int iter, int shot_interval, int snap_interval,
                                const char *dir);

/* Device bytes a context needs for one run of `problem` (0 modeling, 1 gradient, 2 line-search
 * residual) over these shots of an nz x nx model: what a serving loop admits requests by.
 * No counterpart in the reference. */
FWI_API size_t fwi_estimate_bytes(const fwi_shot *shots, int nshot, int nz, int nx, int nt, int pml, int problem,
                                  int filter);

/* ---------------------------------------------------------------- serving
 * A request loop on one GPU (no counterpart in the reference, which runs one job per process).
 * Requests of any grid size arrive through fwi_server_submit from any thread; the server admits
 * the oldest one as soon as one of `max_active` workers is free and its footprint
 * (fwi_request_bytes) fits into `hbm_budget` (0: 90 % of the free device memory) beside the
 * requests already running, and runs admitted requests concurrently, each on its own stream.
 * Results are written into the caller's buffers, which must stay valid until fwi_server_wait
 * reports the request done.  fwi_server_destroy finishes every submitted request first. */
typedef struct fwi_server fwi_server;
enum { FWI_REQ_MODEL = 0, FWI_REQ_GRADIENT = 1 };
enum { FWI_REQ_QUEUED = 0, FWI_REQ_RUNNING = 1, FWI_REQ_DONE = 2, FWI_REQ_FAILED = 3 };
typedef struct fwi_request {
    int kind;                     /* FWI_REQ_MODEL (modeling, problem 0) or FWI_REQ_GRADIENT (problem 1) */
    int nz, nx;                   /* model grid; vp and rho are [nx][nz] host arrays */
    float dx, dz, dt;
    int nt, pml, fs;
    const float *vp, *rho;
    const fwi_shot *shots;
    int nshot;
    const float *const *obs;      /* gradient: observed traces per shot, [ntr][ns] */
    float freq;                   /* residual filter frequency (0: the shot's fpeak) */
    int filter, precondition;     /* as iso_acoustic2d_propagation */
    float *const *traces;         /* out, per shot [ntr][ns] or NULL: seismograms / adjoint sources */
    float *grad;                  /* out, gradient [nx][nz] (gradient requests) or NULL */
} fwi_request;
typedef struct fwi_request_info {
    int state, status;            /* FWI_REQ_*; FWI_OK or the engine's error code */
    size_t bytes;                 /* admitted footprint */
    double queue_ms, run_ms, total_ms;
    double objective;             /* misfit of a gradient request */
    double cell_updates;
    char error[256];
} fwi_request_info;
typedef struct fwi_server_stats {
    long long submitted, completed, failed, rejected;
    double p50_ms, p99_ms, max_ms;          /* submission to completion */
    double p50_queue_ms, p99_queue_ms;      /* submission to admission */
    double wall_s;                          /* first submission to last completion */
    double cell_updates, shots_modeled, shot_gradients;
    size_t budget, peak_bytes;
    int max_active, peak_active;
} fwi_server_report;
FWI_API int fwi_server_create(fwi_server **out, int device, size_t hbm_budget, int max_active);
FWI_API size_t fwi_request_bytes(const fwi_request *req);
FWI_API int fwi_server_submit(fwi_server *s, const fwi_request *req, long long *id);
FWI_API int fwi_server_wait(fwi_server *s, long long id, double timeout_s, fwi_request_info *info);
FWI_API int fwi_server_stats(fwi_server *s, fwi_server_report *out);
FWI_API int fwi_server_destroy(fwi_server *s);

/* Shot-sharded runs (one context per GPU, each holding a share of the survey's shots and the
 * whole model).  The path has one exchange step per gradient: the FP64 stacks of the gradient
 * and of the pseudo-Hessian (propagation.c:953-976 stacks them over shots) and the
 * scalar sums of the FWI loop (misfit, step-length numerator and denominator,
 * optimization.c:13-76).  With a hook installed, the engine calls it at each exchange point
 * with `count` device doubles that the hook must replace, in place, by their sum over all
 * ranks, enqueued on (or synchronised with) `stream`, the engine's CUDA stream; it returns 0 on
 * success.  Every rank reaches the same exchange points in the same order.  The global
 * preconditioning and everything after it then run redundantly on each rank, as in the
 * reference after its stack.  No counterpart in the reference (it runs on one host). */
typedef int (*fwi_allreduce_fn)(double *dev, size_t count, void *stream, void *user);
FWI_API int fwi_ctx_set_allreduce(fwi_ctx *ctx, fwi_allreduce_fn fn, void *user);

/* one iteration of the FWI loop of acoustic2d_fwi.c:411-465 on the context's model, shots and
 * observed data, everything between the two propagations on the device:
 * gradient (problem 1) -> cos^2 smoothing along z (rz) then x (rx) -> fun1 = misfit ->
 * histogram-scaled perturbation of the slowness -> trial model -> forward + residual
 * (problem 2) -> fun2 -> step length -> model update.  The updated model stays in the
 * context (fwi_ctx_get_model).  The slowness is carried between iterations as the
 * reference carries it; the first call derives it from the model. */
typedef struct {
    int rx, rz;                 /* smoothing half-widths (x, z) */
    int precondition;           /* pseudo-Hessian preconditioning */
    int filter;                 /* residual filter: 2 (tapers only) */
    float freq;                 /* taper reference frequency (0: wavelet peak) */
    int waterdepth;             /* rows kept at the water values */
    float vp_water, rho_water;
    float vpmin, vpmax, rhomin, rhomax;
    int gardner;                /* 1: rho from vp by Gardner after each update */
    int path;                   /* FWI_PATH_PLAIN or FWI_PATH_BATCHED */
} fwi_iter_params;
typedef struct {
    float fun1, fun2, steplen, scalar;
    double ms;                  /* device time of the iteration (CUDA events) */
    double cell_updates;
    long long kernel_launches;
} fwi_iter_result;
FWI_API int fwi_ctx_fwi_iteration(fwi_ctx *ctx, const fwi_iter_params *p, fwi_iter_result *out);
/* current model and gradient of the context (host arrays [nx][nz]) */
FWI_API int fwi_ctx_get_model(fwi_ctx *ctx, float *vp, float *rho);

/* Two-pass cos^2 smoothing of a device-resident [nx][nz] field -- a z pass with half-width rz, then
 * an x pass with rx, each computed as smooth2D computes it -- that allocates no memory.  It has no
 * counterpart in the reference.  It is meant for callers that cannot call cudaMalloc: a serving
 * loop that has reserved its whole device budget up front, host code that runs between the
 * segments of a captured CUDA graph, or a latency-critical loop where an allocation would
 * synchronise the device.  d_in and d_out are the caller's device arrays (the same array smooths
 * in place; partly overlapping arrays are not allowed); the intermediate field lives in a file-scope device array of 4194304 floats (16 MiB) that every
 * GPU loading this library holds until the process exits.  nx*nz above 4194304 or half-widths
 * outside [1, 32] are rejected with FWI_ERR_ARG and a message.  The first call on a device looks up
 * the array's address on that device (with that device current): make that first call before any
 * stream capture.  The address found then belongs to that CUDA context: after a cudaDeviceReset
 * the process must not call this entry point again.  All calls share the array, so calls that
 * overlap on the GPU race on it.
 * stream is a cudaStream_t (NULL: the legacy default stream); the call only enqueues work. */
FWI_API int fwi_smooth2d_noalloc(const float *d_in, float *d_out, int nx, int nz, int rz, int rx, void *stream);

/* Continuous batching (no counterpart in the reference, whose runs go one at a time): an executor
 * advances several independent runs -- each a context with its own model, grid size, record
 * length and shots -- by the same step launches.  fwi_exec_add prepares a run of `problem`
 * (0 modeling, 1 gradient, 2 line-search residual; freq, filter, precondition as for
 * fwi_ctx_run) on a context whose model, shots and (problems 1, 2) observed data are set, and
 * adds it to the batch: it joins at the next step launch, whatever the others' progress.
 * fwi_exec_step issues up to `launches` step launches (<= 0: until the batch is empty), each
 * advancing every run in the batch by one item of its own program, plus each run's work
 * between its passes; *active = runs still in the batch.  A run whose last work is issued is
 * handed back to its context (its stream ordered after that work): fwi_exec_poll then sets
 * *done = 1 and *status, and the context's results are read as after fwi_ctx_run.  While a run
 * is in the batch its context must not be used otherwise.  Results are bit-identical to
 * fwi_ctx_run's batched path.  One thread may call fwi_exec_step while others call
 * fwi_exec_add; the executor's arithmetic is FWI_MATH at creation and runs must match it.
 * Snapshot output (verbose > 1) is not available here. */
typedef struct fwi_exec fwi_exec;
FWI_API int fwi_exec_create(fwi_exec **out, int device);
FWI_API int fwi_exec_add(fwi_exec *ex, fwi_ctx *ctx, int problem, float freq, int filter, int precondition);
FWI_API int fwi_exec_step(fwi_exec *ex, int launches, int *active);
FWI_API int fwi_exec_poll(fwi_exec *ex, fwi_ctx *ctx, int *done, int *status);
FWI_API int fwi_exec_launches(fwi_exec *ex, long long *launches);
FWI_API int fwi_exec_destroy(fwi_exec *ex);

/* Self-test of the failure path of the step kernel's waits (no counterpart in the reference): a
 * one-block kernel waits, with the step kernel's bounded wait and a limit of limit_ms (1..2000),
 * on an mbarrier phase that nothing completes; it gives up, sets the context's error word and
 * returns.  Returns FWI_ERR_CUDA with the message a stalled tile copy produces (the expected
 * outcome); the context stays usable. */
FWI_API int fwi_ctx_selftest_wait(fwi_ctx *ctx, int limit_ms);

/* Measurement helper (no counterpart in the reference): the L2 bandwidth figure that bounds the
 * plain one-shot-per-launch path, whose per-shot state stays in L2.  Copies `bytes` between the
 * device buffers d_a and d_b (each `bytes` long, 16-byte aligned, small enough that both stay in
 * L2) `passes` times inside one kernel launch, alternating direction; *ms_out = device time of
 * that launch (CUDA events on `stream`).  Bytes moved = 2 * bytes * passes. */
FWI_API int fwi_l2_copy_probe(void *d_a, void *d_b, long long bytes, int passes, void *stream, float *ms_out);

/* the launch program of one shot's adjoint pass (host-only, no device needed): four ints per
 * launch {kindA, stepA, kindB, stepB} with kinds 0 none, 3 replay step, 4 adjoint step.
 * overlap 0 is the reference's order (a segment is replayed when the reverse loop reaches it,
 * propagation.c:641-673); overlap 1 replays segment k-1 alongside the adjoint steps of segment k;
 * overlap 2 is the two-step kernel's program: as 1, with up to two replay and two adjoint steps
 * per launch (a kind | 0x100 advances two steps from the step given).
 * Returns the number of launches; writes at most cap launches when items is not NULL. */
FWI_API int fwi_adjoint_program(int nt, int overlap, int *items, int cap);
/* checkpoint interval d = max(round(sqrt(2(nt-1))), 3) of checkpoint.c:47 */
FWI_API int fwi_checkpoint_interval(int nt);

#ifdef __cplusplus
}
#endif
#endif
