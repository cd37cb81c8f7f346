// fwi_noalloc.cu -- the gradient smoothing of the FWI loop for callers that cannot
// allocate device memory.
//
// Some callers must not call cudaMalloc: a serving loop that has reserved its whole
// device-memory budget up front and admits work against it, a host that runs between
// the segments of a captured CUDA graph, or a latency-critical loop where an
// allocation would synchronise the device and stall the other streams.  For them,
// fwi_smooth2d_noalloc smooths a gradient in place of the two smooth2D calls of the
// FWI loop (z pass, then x pass) using only memory that already exists: the caller's
// input and output arrays, the window weights passed by value with the kernel
// arguments, and one file-scope device array for the intermediate field.
//
// That array (FWI_NOALLOC_MAX_CELLS floats, 16 MiB) is reserved by every GPU that
// loads this library for as long as the process lives.  All calls share it: two
// calls whose work overlaps on the GPU (different streams, no ordering between them)
// race on it.  Each call writes every intermediate cell before reading it, so no part
// of it needs clearing between calls.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/fwi_b200.h"
#include "fwi_smooth.cuh"

#define FWI_NOALLOC_MAX_CELLS (1 << 22)  // nx * nz limit of fwi_smooth2d_noalloc
#define FWI_NOALLOC_MAX_HALF 32          // largest smoothing half-width

namespace {

static __device__ __align__(256) float g_smooth_scratch[FWI_NOALLOC_MAX_CELLS];

struct Window {
    float w[2 * FWI_NOALLOC_MAX_HALF + 1];
    __device__ float operator[](int k) const { return w[k]; }
};

// one cos^2 pass (smooth2D, common.c:927-1040) with the weights passed by value: the
// engine's smoothing pass (fwi_smooth.cuh), reading nothing but its arguments
__global__ void k_smooth_pass(const float *__restrict__ in, float *__restrict__ out, int nx, int nz, int N, int zdir,
                              Window w)
{
    fwi::smooth_pass(in, out, nx, nz, N, zdir, w);
}

Window weights(int N)
{
    Window w;
    memset(&w, 0, sizeof(w));
    for (int i = 0; i < 2 * N + 1; i++) {  // double cosine, squared in float (common.c:955-961)
        w.w[i] = (float)cos(3.141592653589793 * (i - N) / (2.0 * N));
        w.w[i] *= w.w[i];
    }
    return w;
}

// device address of the scratch array, resolved once per device with that device current
// (on the first call made on that device).  The address belongs to the CUDA context of that
// first call: a process that resets the device (cudaDeviceReset) and goes on calling this
// entry point gets a stale address, so such a process must not use it after a reset.
std::mutex g_mu;
float *g_addr[64];
bool g_ready[64];

int scratch_for_current_device(float **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FWI_ERR_NODEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ready[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_smooth_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "<error>: fwi_smooth2d_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                    cudaGetErrorString(e));
            return FWI_ERR_CUDA;
        }
        g_addr[dev] = (float *)p;
        g_ready[dev] = true;
    }
    *out = g_addr[dev];
    return FWI_OK;
}

}  // namespace

extern "C" int fwi_smooth2d_noalloc(const float *d_in, float *d_out, int nx, int nz, int rz, int rx, void *stream)
{
    if (!d_in || !d_out || nx <= 0 || nz <= 0) {
        fprintf(stderr, "<error>: fwi_smooth2d_noalloc: NULL array or empty grid (nx=%d, nz=%d)\n", nx, nz);
        return FWI_ERR_ARG;
    }
    if ((long long)nx * nz > FWI_NOALLOC_MAX_CELLS) {
        fprintf(stderr,
                "<error>: fwi_smooth2d_noalloc: %d x %d = %lld cells exceeds the %d-cell scratch array; "
                "use smooth2D for larger models\n",
                nx, nz, (long long)nx * nz, FWI_NOALLOC_MAX_CELLS);
        return FWI_ERR_ARG;
    }
    if (rz < 1 || rx < 1 || rz > FWI_NOALLOC_MAX_HALF || rx > FWI_NOALLOC_MAX_HALF) {
        fprintf(stderr, "<error>: fwi_smooth2d_noalloc: half-widths rz=%d rx=%d must lie in [1, %d]\n", rz, rx,
                FWI_NOALLOC_MAX_HALF);
        return FWI_ERR_ARG;
    }
    float *tmp = nullptr;
    int rc = scratch_for_current_device(&tmp);
    if (rc != FWI_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    k_smooth_pass<<<592, 256, 0, st>>>(d_in, tmp, nx, nz, rz, 1, weights(rz));
    k_smooth_pass<<<592, 256, 0, st>>>(tmp, d_out, nx, nz, rx, 0, weights(rx));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "<error>: fwi_smooth2d_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        return FWI_ERR_CUDA;
    }
    return FWI_OK;
}
