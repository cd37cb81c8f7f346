// fwi_aux.cuh -- the per-shot and per-survey kernels around the time loop:
// trace transposition and adjoint source, finalisation of the FP64 accumulators,
// preconditioning, the shot stack and the FP64 reductions (misfit, RMS, means).
// Reductions are two-pass and deterministic (fixed tree per block, partials summed
// in block order), so a run is reproducible bit for bit.
#pragma once
#include <cuda_runtime.h>
#include "fwi_kernels.cuh"

namespace fwi {

struct GatherDesc {
    const float *traces_t;  // [ns][ntr] forward samples
    float *pre;             // [ntr][ns] predicted gather / residual (in place, as the reference)
    const float *obs;       // [ntr][ns] observed gather (residual modes)
    float *adj_t;           // [nt][ntr] adjoint source for injection (may be null)
    const float *tct;       // time taper coefficients (Lt+1), null when Lt == 0
    const float *tcr;       // trace taper coefficients (Lr+1), null when Lr == 0
    int ns, ntr, Lt, Lr;
    int adj_rows;           // rows of adj_t (the engine's nt): samples beyond it are not injected
};

// 0: copy samples out; 1: residual + tapers (filter 2 adjoint source, optimization.c:335-418).
// The taper multiplies the time factor first, then the trace factor (taper_traces, common.c:796-895).
// block (32, 8): a 32x32 tile of samples x traces
static __global__ void k_gather(const GatherDesc *__restrict__ gd, int mode)
{
    __shared__ float tile[32][33];
    __shared__ float tile2[32][33];
    const GatherDesc &D = gd[blockIdx.z];
    const int k0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    if (k0 >= D.ns || r0 >= D.ntr) return;
    const int tx = threadIdx.x;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {  // [k][itr], coalesced along itr
        int k = k0 + i, r = r0 + tx;
        tile[i][tx] = (k < D.ns && r < D.ntr) ? D.traces_t[(long long)k * D.ntr + r] : 0.0f;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {  // [itr][k], coalesced along k
        int r = r0 + i, k = k0 + tx;
        float v = tile[tx][i];
        if (r < D.ntr && k < D.ns) {
            long long o = (long long)r * D.ns + k;
            if (mode == 1) {
                v = __fsub_rn(v, D.obs[o]);
                if (D.Lt > 0) {
                    if (k <= D.Lt) v = __fmul_rn(v, D.tct[D.Lt - k]);
                    int kb = D.ns - D.Lt - 1;
                    if (k >= kb) v = __fmul_rn(v, D.tct[k - kb]);
                }
                if (D.Lr > 0) {
                    if (r <= D.Lr) v = __fmul_rn(v, D.tcr[D.Lr - r]);
                    int rb = D.ntr - D.Lr - 1;
                    if (r >= rb) v = __fmul_rn(v, D.tcr[r - rb]);
                }
            }
            D.pre[o] = v;
        }
        tile2[i][tx] = v;
    }
    if (mode != 1 || D.adj_t == nullptr) return;
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {  // back to [k][itr] for the injection
        int k = k0 + i, r = r0 + tx;
        if (k < D.ns && k < D.adj_rows && r < D.ntr) D.adj_t[(long long)k * D.ntr + r] = tile2[tx][i];
    }
}

// taper_traces (common.c:796-895) in place on one [ntr][ns] gather per blockIdx.y: the time
// factor first, then the trace factor, as k_gather applies them
struct TaperDesc {
    float *a;
    const float *tct, *tcr;
    int ns, ntr, Lt, Lr;
};
static __global__ void k_taper(const TaperDesc *__restrict__ td)
{
    const TaperDesc &D = td[blockIdx.y];
    const long long n = (long long)D.ns * D.ntr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / D.ns), k = (int)(i % D.ns);
        float v = D.a[i];
        if (D.Lt > 0) {
            if (k <= D.Lt) v = __fmul_rn(v, D.tct[D.Lt - k]);
            const int kb = D.ns - D.Lt - 1;
            if (k >= kb) v = __fmul_rn(v, D.tct[k - kb]);
        }
        if (D.Lr > 0) {
            if (r <= D.Lr) v = __fmul_rn(v, D.tcr[D.Lr - r]);
            const int rb = D.ntr - D.Lr - 1;
            if (r >= rb) v = __fmul_rn(v, D.tcr[r - rb]);
        }
        D.a[i] = v;
    }
}

struct FinDesc {
    const double *acc;    // [Nx][ld] accumulator
    float *out;           // [nxx][nz] window, FP32 as the reference keeps per-shot fields
    const float *vp, *rho;  // global model [nx][nz] (unpadded, without the layer scaling)
    int ix_min, nxx, nz, pml, ld;
};

// which = 0: pseudo-Hessian 4 H / (rho v)^2 (propagation.c:610-623); 1: gradient 2 G / (rho v) (:733-743)
static __global__ void k_finalize(const FinDesc *__restrict__ fd, int which)
{
    const FinDesc &D = fd[blockIdx.y];
    long long n = (long long)D.nxx * D.nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int ix = (int)(i / D.nz), iz = (int)(i % D.nz);
        long long gi = (long long)(ix + D.ix_min) * D.nz + iz;
        float rv = __fmul_rn(D.rho[gi], D.vp[gi]);
        double a = D.acc[(long long)(ix + D.pml) * D.ld + iz + D.pml];
        double r = which == 0 ? __ddiv_rn(__dmul_rn(4.0, a), (double)__fmul_rn(rv, rv)) : __ddiv_rn(__dmul_rn(2.0, a), (double)rv);
        D.out[i] = (float)r;
    }
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
template <int NT>
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double ws[NT / 32];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < NT / 32 ? ws[threadIdx.x] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

struct SumDesc {
    const float *a;        // first operand
    const float *b;        // second operand or null
    long long n;
    int op;                // 0: sum a; 1: sum a*a (float product); 2: sum (double)a*(double)a;
                           // 3: sum a*(a-b) and (a-b)^2 (two results, float products)
    double *partial;       // gridDim.x (x2 for op 3) partial sums
};

template <int NT>
__global__ void __launch_bounds__(NT) k_sum_partial(const SumDesc *__restrict__ sd)
{
    const SumDesc &D = sd[blockIdx.y];
    double s0 = 0.0, s1 = 0.0;
    for (long long i = blockIdx.x * (long long)NT + threadIdx.x; i < D.n; i += (long long)gridDim.x * NT) {
        float a = D.a[i];
        if (D.op == 0) s0 += (double)a;
        else if (D.op == 1) s0 += (double)__fmul_rn(a, a);
        else if (D.op == 2) s0 += (double)a * (double)a;
        else {
            float dl = __fsub_rn(a, D.b[i]);
            s0 += (double)__fmul_rn(a, dl);
            s1 += (double)__fmul_rn(dl, dl);
        }
    }
    s0 = block_sum<NT>(s0);
    if (D.op == 3) s1 = block_sum<NT>(s1);
    if (threadIdx.x == 0) {
        D.partial[blockIdx.x] = s0;
        if (D.op == 3) D.partial[gridDim.x + blockIdx.x] = s1;
    }
}

// sums nparts partials per descriptor in fixed order into out[2*y], out[2*y+1]
static __global__ void k_sum_final(const SumDesc *__restrict__ sd, int nparts, double *out)
{
    const SumDesc &D = sd[blockIdx.x];
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int i = 0; i < nparts; ++i) s0 += D.partial[i];
        if (D.op == 3)
            for (int i = 0; i < nparts; ++i) s1 += D.partial[nparts + i];
        out[2 * blockIdx.x] = s0;
        out[2 * blockIdx.x + 1] = s1;
    }
}

// per-shot preconditioning (optimization.c:58-97): avg = (float)(sum/n); f = 1 + H/(7 avg); g /= f; H /= f
struct PrecDesc {
    float *g, *h;
    long long n;
    const double *sum;  // sum of h (FP64)
};
static __global__ void k_shot_precondition(const PrecDesc *__restrict__ pd)
{
    const PrecDesc &D = pd[blockIdx.y];
    const float avg = (float)(*D.sum / (double)D.n);
    const float s7 = __fmul_rn(7.0f, avg);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < D.n; i += (long long)gridDim.x * blockDim.x) {
        float h = D.h[i];
        float f = __fadd_rn(1.0f, __fdiv_rn(h, s7));
        D.g[i] = __fdiv_rn(D.g[i], f);
        D.h[i] = __fdiv_rn(h, f);
    }
}

// shot stack in shot order (propagation.c:953-976): one thread per global cell
struct StackShot {
    const float *g, *h;
    int ix_min, ix_max;
};
static __global__ void k_stack(const StackShot *__restrict__ ss, int nshot, int nz, int nx, int with_h, double *gc, double *hc)
{
    long long n = (long long)nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int ix = (int)(i / nz), iz = (int)(i % nz);
        double a = gc[i], b = with_h ? hc[i] : 0.0;
        for (int s = 0; s < nshot; ++s) {
            const StackShot &S = ss[s];
            if (ix < S.ix_min || ix > S.ix_max) continue;
            long long j = (long long)(ix - S.ix_min) * nz + iz;
            a = __dadd_rn(a, (double)S.g[j]);
            if (with_h) b = __dadd_rn(b, (double)S.h[j]);
        }
        gc[i] = a;
        if (with_h) hc[i] = b;
    }
}

// FP64 stacks to FP32, then global preconditioning g /= (H + alpha*rms) (optimization.c:13-56)
static __global__ void k_to_float(const double *a, float *out, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)a[i];
}
static __global__ void k_global_precondition(float *grad, const float *prec, long long n, const double *sumsq, float alpha)
{
    const float rms = (float)sqrt(*sumsq / (double)n);
    const float ar = __fmul_rn(alpha, rms);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        grad[i] = __fdiv_rn(grad[i], __fadd_rn(prec[i], ar));
}

}  // namespace fwi
