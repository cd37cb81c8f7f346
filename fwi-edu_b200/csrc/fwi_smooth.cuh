// fwi_smooth.cuh -- one pass of the cos^2 gradient smoothing (smooth2D, common.c:927-1040),
// shared by the engine's kernel (weights in device memory) and the no-allocation entry
// point (weights passed by value with the kernel arguments).
//
// out[ix][iz] = sum_k w[k] in[..] / (sum_k w[k] + FLT_MIN) over the window of half-width N
// clipped to the axis, FP64 accumulation in window order as the reference accumulates; z
// direction when zdir, x otherwise.  Arrays are [nx][nz], z fastest.
#pragma once
#include <cfloat>
#include <cuda_runtime.h>

namespace fwi {

// W: anything indexable by the window position k = 0..2N (a device pointer, or a struct
// holding the weights)
template <class W>
__device__ __forceinline__ void smooth_pass(const float *__restrict__ in, float *__restrict__ out, int nx, int nz,
                                            int N, int zdir, const W &w)
{
    const long long n = (long long)nx * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / nz), iz = (int)(i % nz);
        const int j = zdir ? iz : ix, n1 = zdir ? nz : nx;
        const int ws = j >= N ? 0 : N - j, ds = j >= N ? j - N : 0;
        const int we = (n1 - 1 - j < N) ? 2 * N - (N - (n1 - 1 - j)) : 2 * N;
        double a1 = 0.0, a2 = 0.0;
        for (int k = ws, k2 = ds; k <= we; ++k, ++k2) {
            const float v = zdir ? in[(long long)ix * nz + k2] : in[(long long)k2 * nz + iz];
            a1 = __dadd_rn(a1, (double)__fmul_rn(w[k], v));
            a2 = __dadd_rn(a2, (double)w[k]);
        }
        out[i] = (float)__ddiv_rn(a1, __dadd_rn(a2, (double)FLT_MIN));
    }
}

}  // namespace fwi
