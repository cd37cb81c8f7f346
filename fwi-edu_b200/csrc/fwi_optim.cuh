// fwi_optim.cuh -- device kernels of the FWI loop around the gradient: cos^2 smoothing
// (smooth2D, common.c:927-1040), the histogram-scaled model perturbation
// (compute_model_perturbation, optimization.c:178-298), the residual with its tapers
// (compute_adjoint_source2d with filter 2, optimization.c:300-419) and the water-layer
// reset.  Each keeps the reference's per-element operation order.
#pragma once
#include <cfloat>
#include <cuda_runtime.h>

#include "fwi_smooth.cuh"

namespace fwi {

// one smoothing pass with the window weights w[0..2N] in device memory
static __global__ void k_smooth2d(const float *__restrict__ in, float *__restrict__ out, int nx, int nz, int N,
                                  int zdir, const float *__restrict__ w)
{
    smooth_pass(in, out, nx, nz, N, zdir, w);
}

// ------------------------------------------------------------ perturbation
struct PertState {
    float mx, mn;         // max(0, max g), min(0, min g)
    float interval;       // (float)((mx - mn) / 1000.0): float difference, double quotient
    float scalar;         // result
    int hist[1001];
    double avg_slow;      // sum of slowness (FP64)
};

__device__ __forceinline__ float atomic_max_f(float *a, float v)
{
    return v >= 0.f ? __int_as_float(atomicMax((int *)a, __float_as_int(v)))
                    : __uint_as_float(atomicMin((unsigned int *)a, __float_as_uint(v)));
}
__device__ __forceinline__ float atomic_min_f(float *a, float v)
{
    return v >= 0.f ? __int_as_float(atomicMin((int *)a, __float_as_int(v)))
                    : __uint_as_float(atomicMax((unsigned int *)a, __float_as_uint(v)));
}

static __global__ void k_pert_init(PertState *st)
{
    for (int i = threadIdx.x; i < 1001; i += blockDim.x) st->hist[i] = 0;
    if (threadIdx.x == 0) {
        st->mx = 0.0f;
        st->mn = 0.0f;
        st->avg_slow = 0.0;
    }
}

static __global__ void k_pert_minmax(const float *__restrict__ g, long long n, PertState *st)
{
    float mx = 0.0f, mn = 0.0f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        mx = fmaxf(mx, g[i]);
        mn = fminf(mn, g[i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, o));
        mn = fminf(mn, __shfl_down_sync(0xffffffffu, mn, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomic_max_f(&st->mx, mx);
        atomic_min_f(&st->mn, mn);
    }
}

// pos = (int)((g - Min) / interval + 0.5): float quotient, double add, truncation
static __global__ void k_pert_hist(const float *__restrict__ g, long long n, PertState *st)
{
    __shared__ int h[1001];
    for (int i = threadIdx.x; i < 1001; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const float mn = st->mn;
    const float interval = (float)((double)__fsub_rn(st->mx, mn) / 1000.0);  // float difference, double quotient
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float q = __fdiv_rn(__fsub_rn(g[i], mn), interval);
        int pos = (int)((double)q + 0.5);
        pos = pos < 0 ? 0 : (pos > 1000 ? 1000 : pos);  // the reference indexes unchecked; valid gradients stay in [0, 1000]
        atomicAdd(&h[pos], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 1001; i += blockDim.x)
        if (h[i]) atomicAdd(&st->hist[i], h[i]);
    if (blockIdx.x == 0 && threadIdx.x == 0) st->interval = interval;
}

// peak, widen to 99 % of the mass, scale = mean(slowness) * fraction / max|edge| (optimization.c:238-285)
static __global__ void k_pert_scalar(PertState *st, const double *slow_sum, long long len, float fraction)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int peak = 0, pos = 0;
    for (int i = 0; i < 1001; i++)
        if (st->hist[i] > peak) {
            peak = st->hist[i];
            pos = i;
        }
    int hi = pos, lo = pos;
    const float flen = (float)len;
    float acc = __fdiv_rn((float)st->hist[hi], flen);
    int guard = 0;
    while (acc < 0.99f && guard++ < 4096) {  // at most 1000 widenings can change acc
        if (hi < 1000) {
            hi++;
            acc = __fadd_rn(acc, __fdiv_rn((float)st->hist[hi], flen));
        }
        if (lo > 0) {
            lo--;
            acc = __fadd_rn(acc, __fdiv_rn((float)st->hist[lo], flen));
        }
    }
    const float a = fabsf(__fadd_rn(st->mn, __fmul_rn((float)lo, st->interval)));
    const float b = fabsf(__fadd_rn(st->mn, __fmul_rn((float)hi, st->interval)));
    const float edge = a > b ? a : b;
    st->scalar = (float)__ddiv_rn(__dmul_rn(__ddiv_rn(*slow_sum, (double)len), (double)fraction), (double)edge);
}

static __global__ void k_pert_apply(const float *__restrict__ g, float *__restrict__ out, long long n, const PertState *st)
{
    const float ms = -st->scalar;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = __fmul_rn(ms, g[i]);
}

// residual + tapers of one gather [ntr][ns] (time factor first, then trace factor)
static __global__ void k_residual_taper(const float *__restrict__ pre, const float *__restrict__ obs, float *__restrict__ out,
                                        int ns, int ntr, int Lt, int Lr, const float *__restrict__ tct,
                                        const float *__restrict__ tcr)
{
    const long long n = (long long)ns * ntr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / ns), k = (int)(i % ns);
        float v = __fsub_rn(pre[i], obs[i]);
        if (Lt > 0) {
            if (k <= Lt) v = __fmul_rn(v, tct[Lt - k]);
            if (k >= ns - Lt - 1) v = __fmul_rn(v, tct[k - (ns - Lt - 1)]);
        }
        if (Lr > 0) {
            if (r <= Lr) v = __fmul_rn(v, tcr[Lr - r]);
            if (r >= ntr - Lr - 1) v = __fmul_rn(v, tcr[r - (ntr - Lr - 1)]);
        }
        out[i] = v;
    }
}

}  // namespace fwi
