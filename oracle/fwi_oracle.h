/*
 * fwi_oracle.h -- CPU restatement of the FWI-EDU 2-D acoustic forward/adjoint
 * engine.  TEST INFRASTRUCTURE ONLY: the checker that tests/, smoke() and the
 * bench's CPU-baseline leg use.  The product library never links it.
 *
 * Built twice by oracle/Makefile: ORACLE_REAL=float (bit-for-bit the strict
 * IEEE build of the reference: same expression order, same float/double
 * promotions, no contraction) and ORACLE_REAL=double (the FP64 build of the
 * same algorithm, used as the error reference).
 *
 * Arrays are flat and column-major like the reference's alloc2float(nz, nx):
 * a[ix][iz] lives at a[ix*nz + iz] (z fastest).
 */
#ifndef FWI_ORACLE_H
#define FWI_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* one shot record; mirrors the fields of Record2D (observation.h:18-48) the engine reads */
typedef struct {
    int shotID;          /* 1-based */
    int isx, isz;        /* source grid index: x window-local, z global (no pml) */
    int ntr;             /* receivers */
    int ns;              /* samples per trace */
    int sampleRate;      /* engine steps per recorded sample */
    int ix_min, ix_max;  /* model window (inclusive) */
    float dt;            /* record sample interval (dt * sampleRate) */
    float dtr;           /* receiver interval */
    float fpeak;         /* wavelet peak frequency */
    const float *src;    /* nt */
    const int *igx;      /* ntr, window-local */
    const int *igz;      /* ntr, global */
} OrcShot;

/* padded coefficient fields for one model window (Nz x Nx, z fastest), in the oracle precision */
int orc_real_size(void);

/* K20: pad + MEAL + coefficient prep + rgfd (propagation.c:508-532). Outputs are Nz*Nx each. */
void orc_setup(const float *vpm, const float *rhom, int nz, int nx, int pml,
               float dx, float dz, float dt, float fpeak,
               void *coef1, void *coef2, void *coef3, void *K,
               void *invrho, void *invrhox, void *invrhoz);

/* forward modeling of one shot (engine mode 0): traces[ntr*ns] */
int orc_forward(const OrcShot *shot, const float *vpm, const float *rhom, int nz, int nx,
                float dx, float dz, float dt, int nt, int pml, int freesurface, float *traces);

/* one shot gradient: engine mode 1 (+H), adjoint source, engine mode 2, per-shot
 * preconditioning.  traces_pre (in/out): predicted traces, overwritten with the adjoint
 * source as in the reference; grad_shot/precond_shot: nz*(ix_max-ix_min+1) */
int orc_shot_gradient(const OrcShot *shot, const float *vp_global, const float *rho_global,
                      int nz, int nx_global, float dx, float dz, float dt, int nt, int pml,
                      int freesurface, float freq, int filter, int precondition,
                      const float *traces_obs, float *traces_pre,
                      float *grad_shot, float *precond_shot);

/* mirrors iso_acoustic2d_propagation (propagation.c:777-1036) for Nshot shots.
 * obs/pre: per-shot trace buffers (pointer arrays).  grad: nz*nx (problem 1), else NULL. */
int orc_propagation(const float *vp, const float *rho, const OrcShot *shots, int Nshot,
                    int nz, int nx, float dx, float dz, float dt, int nt, int pml,
                    int freesurface, float freq, float filter, int precondition, int problem,
                    float *const *obs, float *const *pre, float *grad);

/* the reductions and model operations of the FWI loop (optimization.c, common.c) */
float orc_objective(float *const *traces, const int *ntr, const int *ns, int Nshot);
float orc_step_length(float *const *pre0, float *const *pre1, const int *ntr, const int *ns, int Nshot);
float orc_model_perturbation(float fraction, const float *slowness, const float *gradient, float *out, int len);
void orc_smooth2d(const float *in, float *out, int nx, int nz, int N, int iszdirect);
void orc_taper_traces(float *tr, int nt, int ntr, int taperLenTime, int taperLenTrace);
void orc_adjoint_source(const OrcShot *shot, const float *vp_global, int nz, float freq, int filter,
                        const float *pre, const float *obs, float *adj);
void orc_shot_precondition(float *grad, float *precond, int n);
/* checkpoint snapshots stored as 0: oracle precision, 1: FP16 with max-abs scaling, 2: BF16 */
void orc_set_checkpoint_precision(int mode);
void orc_global_precondition(float *grad, const float *precond, int n, float alpha);
/* model update of acoustic2d_fwi.c:425-465 after the step length is known */
void orc_vp2density(const float *vp, float *rho, int n);
void orc_fwi_update(float *slow, float *vp, float *rho, const float *perturb, float steplen,
                    int nx, int nz, int waterdepth, float vp_water, float rho_water,
                    float vpmin, float vpmax, float rhomin, float rhomax, int gardner);
void orc_fwi_trial(const float *slow, const float *perturb, float *vp, float *rho, int nx, int nz,
                   int waterdepth, float vp_water, float rho_water, float vpmin, float vpmax,
                   float rhomin, float rhomax, int gardner);

/* checkpoint bookkeeping of checkpoint.c:29-99 */
int orc_checkpoint_interval(int nt);
int orc_checkpoint_count(int nt);

#ifdef __cplusplus
}
#endif
#endif
