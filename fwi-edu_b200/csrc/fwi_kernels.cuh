// fwi_kernels.cuh -- shared definitions of the engine's device code: the per-shot
// descriptor the step kernel reads, the work-item kinds of the launch programs,
// and the mapping from a time index to the frame buffer that holds that field.
//
// Fields are [Nx][ld] floats, z fastest, ld = Nz rounded up to 4 (16-byte rows).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fwi {

// item kinds of the per-launch work programs
enum StepKind : int {
    K_NONE = 0,
    K_FWD0 = 1,  // forward modeling (engine mode 0)
    K_FWD1 = 2,  // forward with checkpoints and pseudo-Hessian (engine mode 1)
    K_REP = 3,   // forward reconstruction from a checkpoint (replay)
    K_ADJ = 4    // adjoint step with injection and imaging (engine mode 2)
};

constexpr int MST = 5;     // imaging / pseudo-Hessian interval (propagation.h:21)
constexpr int LX_MAX = 64; // longest x strip of one block

struct ShotDesc {
    // geometry of the padded window
    int Nx, Nz, ld, G, pml, nz, nxx, fs, izStart;
    int nt, d, K, ns, sr, ntr, S5, hessian;
    int isx, isz;  // padded source cell
    float invdx, invdz, invdxdx, invdzdz, invdtdt, dt;
    float negzero;  // -0.0f, for the step kernels' packed products (fma(a, b, -0) rounds as a*b)
    // coefficients [Nx][ld]
    const float *c1, *c2, *ck, *irx, *irz, *ir;
    // source terms per step: forward (double, propagation.c:558) and replay (float, :662)
    const double *srcd;
    const float *srcf;
    // receivers as a per-column list: colptr[Nx+1] into rec (padded z, trace index) and recK
    const int *colptr;
    const int2 *rec;
    const float *recK;
    const int *rec_off;    // per receiver (trace order): padded cell offset X*ld + Z
    float *traces_t;       // [ns][ntr] samples of the forward pass
    const float *adj_t;    // [nt][ntr] adjoint source
    // wavefield storage: one block of nfr frames of Nx*ld floats per shot (the blocks of a
    // shot group are consecutive in one pool, so one tensor map covers the group), laid out as
    // F_FWD (NROT forward frames), F_ADJ (NROT adjoint), F_REP (NROT replay), F_CK (2(K+1) checkpoint
    // slots: slot 0 = u(-1), 2k+1 = u(kd), 2k = u(kd-1)), then 2*S5 replayed frames kept for
    // imaging (t % 5 == 0), double-buffered by segment.  A forward-only run has nfr = 3.
    float *frames;
    int nfr;
    double *H, *Gacc;      // [Nx][ld] FP64 accumulators (pseudo-Hessian, gradient)
    long long frame;       // Nx*ld
    int rz0, rz1;          // padded depth range of this shot's receivers
    int snap;              // > 0: steps whose output time is a multiple of snap mirror every free-surface
                           // row (pml-1 .. 0), as the reference's snapshots hold them; 0: only the
                           // three rows the stencil reads again
};

// ------------------------------------------------------------ buffer selection
// Slot of a stored forward time index t (checkpoint.c:130-159 keeps (u(c-1), u(c))
// for every c = k*d < nt), -1 when the step is not stored.
__host__ __device__ inline int stored_slot(const ShotDesc &S, int t)
{
    if (t == -1) return 0;
    if (t < 0 || t >= S.nt) return -1;
    if (t % S.d == 0) return 2 * (t / S.d) + 1;
    if ((t + 1) % S.d == 0 && t + 1 < S.nt) return 2 * ((t + 1) / S.d);
    return -1;
}
// Fields that are not kept rotate through NROT frames by time index.  Four, not three: a launch
// that advances two steps (temporal blocking) reads u(t) and u(t-1) and writes u(t+1) and u(t+2),
// and its blocks read halos of u(t-1) while others already write u(t+2): four distinct frames.
constexpr int NROT = 4;
constexpr int F_FWD = 0, F_ADJ = NROT, F_REP = 2 * NROT, F_CK = 3 * NROT;
__host__ __device__ inline int nframes_gradient(int K, int S5) { return F_CK + 2 * (K + 1) + 2 * S5; }
__host__ __device__ inline float *frame_ptr(const ShotDesc &S, int i) { return S.frames + (long long)i * S.frame; }

// frame of the forward field u(t) in a pass that keeps checkpoints (mode 1) or not (mode 0)
__host__ __device__ inline int fwd_idx(const ShotDesc &S, int t, bool keep)
{
    if (keep) {
        int s = stored_slot(S, t);
        if (s >= 0) return F_CK + s;
    }
    return F_FWD + (t + NROT) % NROT;
}
// replayed frame of segment k (checkpoint c = k*d), t > c, t % 5 == 0
__host__ __device__ inline int seg_idx(const ShotDesc &S, int t)
{
    int k = t / S.d, c = k * S.d;
    int j = t / MST - (c + MST) / MST;
    return F_CK + 2 * (S.K + 1) + (k & 1) * S.S5 + j;
}
// u(t) during the replay of the segment containing t
__host__ __device__ inline int rep_idx(const ShotDesc &S, int t)
{
    int s = stored_slot(S, t);
    if (s >= 0) return F_CK + s;
    if (t % MST == 0) return seg_idx(S, t);
    return F_REP + t % NROT;
}
// adjoint field A(t): p1 of adjoint step t (with the injection of step t applied)
__host__ __device__ inline int adj_idx(const ShotDesc &, int t) { return F_ADJ + (t + NROT) % NROT; }
// forward field used by the imaging condition at adjoint step it (it % 5 == 0)
__host__ __device__ inline int img_idx(const ShotDesc &S, int it)
{
    int s = stored_slot(S, it);
    if (s >= 0) return F_CK + s;
    return seg_idx(S, it);
}
__host__ __device__ inline float *fwd_buf(const ShotDesc &S, int t, bool keep) { return frame_ptr(S, fwd_idx(S, t, keep)); }
__host__ __device__ inline float *rep_buf(const ShotDesc &S, int t) { return frame_ptr(S, rep_idx(S, t)); }
__host__ __device__ inline float *adj_buf(const ShotDesc &S, int t) { return frame_ptr(S, adj_idx(S, t)); }
__host__ __device__ inline float *img_buf(const ShotDesc &S, int it) { return frame_ptr(S, img_idx(S, it)); }

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float comp(const float4 &v, int j) { return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w; }
__device__ __forceinline__ void setc(float4 &v, int j, float a)
{
    if (j == 0) v.x = a;
    else if (j == 1) v.y = a;
    else if (j == 2) v.z = a;
    else v.w = a;
}
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs_(float a, float b) { return __fsub_rn(a, b); }

}  // namespace fwi
