// fwi_probe.cu -- the L2 bandwidth figure behind the plain path's roofline.
//
// A one-shot step of the 221 x 601 survey keeps its whole state (three fields and the
// coefficient planes, about 6.6 MB) in the 126 MB L2, so the plain path is bounded by L2
// bandwidth, not HBM.  No measured L2 figure exists for this GPU, so the bench measures one
// with this kernel: a STREAM-style copy between two device buffers small enough to stay
// L2-resident, swept `passes` times inside one launch (so that launch gaps do not count),
// alternating direction each pass.  Bytes moved = 2 * n * 16 * passes.
#include <cuda_runtime.h>

#include "../../include/fwi_b200.h"

namespace {

__global__ void k_l2_copy(float4 *__restrict__ a, float4 *__restrict__ b, long long n, int passes)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int p = 0; p < passes; ++p) {
        const float4 *src = (p & 1) ? b : a;
        float4 *dst = (p & 1) ? a : b;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[i];
        // each thread copies the same indices in every pass: no pass reads another thread's writes
    }
}

}  // namespace

extern "C" int fwi_l2_copy_probe(void *d_a, void *d_b, long long bytes, int passes, void *stream, float *ms_out)
{
    if (!d_a || !d_b || bytes < 16 || passes < 1 || !ms_out) return FWI_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const long long n = bytes / 16;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
        return FWI_ERR_CUDA;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return FWI_ERR_CUDA;
    const dim3 grid(4 * sms), block(512);
    k_l2_copy<<<grid, block, 0, st>>>((float4 *)d_a, (float4 *)d_b, n, 2);  // warm: both buffers into L2
    cudaEventRecord(e0, st);
    k_l2_copy<<<grid, block, 0, st>>>((float4 *)d_a, (float4 *)d_b, n, passes);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return FWI_ERR_CUDA;
    *ms_out = ms;
    return FWI_OK;
}
