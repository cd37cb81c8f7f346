// fwi_fft.cuh -- batched circular convolution of real sequences by FFT, in shared memory.
//
// The residual filters of compute_adjoint_source2d (apply_traces_lowpass / _bandpass,
// common.c:584-794: forward FFT, a real cosine-tapered window on the non-negative
// frequencies, inverse FFT, / n) and interpolate_traces (common.c:482-582: zero-stuffing by
// r, a rectangular band window, inverse FFT, real part / N) are, for real input, circular
// convolutions with a fixed real kernel h of the sequence length n:
//     y[i] = sum_j h[(i - j) mod n] x[j]        (interpolation: x zero-stuffed first).
// n is the trace length or the trace count (4001 and 601 on the benchmark survey: primes),
// so the kernel computes it as an M-point circular convolution, M the power of two >= 2n - 1:
// the zero-padded sequence times the spectrum G of the kernel wrapped onto M points (built
// once on the host in FP64, G = FFT_M(h wrapped) / M), which equals the n-point result on
// [0, n).  Two real sequences share one complex transform (x1 + i x2, the kernel is real).
//
// One block holds P such pairs in shared memory (P * M complex floats): the sequences are
// loaded bit-reversed, transformed by radix-2 decimation in time (natural order out),
// multiplied by G, transformed back by decimation in frequency with conjugate twiddles
// (bit-reversed order out) and written from the bit-reversed positions.  FP64 transforms where
// a block holds them (M <= 8192), FP32 above; agreement with the reference is to floating-point
// tolerance, not bitwise (its result carries its own FFT's rounding).
#pragma once
#include <cuda_runtime.h>

namespace fwi {

struct ConvDesc {
    const float *in;            // input sequences: element e of sequence s at in[s * in_ss + e * in_es]
    long long in_es, in_ss;
    int n_in;                   // input samples per sequence
    int stuff;                  // zero-stuffing factor: input sample j lands on position j * stuff
    float *out;                 // output: position i of sequence s at out[s * out_ss + i * out_es]
    long long out_es, out_ss;
    int n_out;                  // positions written per sequence; positions >= N are written as 0
    int N;                      // convolution length
    int nseq;                   // sequences
    int M, logM;                // FFT size, a power of two >= 2N - 1
    int P;                      // sequence pairs per block
    int dbl;                    // 1: transforms in FP64 (G and tw double2), 0: FP32 (float2)
    const void *G;              // FFT_M of the wrapped kernel, / M
    const void *tw;             // exp(-2 pi i k / M), k < M / 2
};

template <class R> struct Cplx;
template <> struct Cplx<float> {
    typedef float2 T;
    static __device__ __forceinline__ T make(float a, float b) { return make_float2(a, b); }
};
template <> struct Cplx<double> {
    typedef double2 T;
    static __device__ __forceinline__ T make(double a, double b) { return make_double2(a, b); }
};

template <class T>
__device__ __forceinline__ T cmulc(T a, T b)
{
    T r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// grid: ceil(nseq / (2 P)) blocks; dynamic shared memory P * M complex values of type R
template <class R>
static __global__ void __launch_bounds__(512) k_fft_conv(const ConvDesc d)
{
    typedef typename Cplx<R>::T C;
    extern __shared__ __align__(16) unsigned char fsm[];
    C *fbuf = reinterpret_cast<C *>(fsm);
    const C *G = static_cast<const C *>(d.G), *tw = static_cast<const C *>(d.tw);
    const int M = d.M, P = d.P, half_M = M >> 1;
    const int s0 = blockIdx.x * 2 * P;  // first sequence of the block
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int i = tid; i < P * M; i += nth) fbuf[i] = Cplx<R>::make(0, 0);
    __syncthreads();
    // load: pair q holds sequences s0 + 2q (real part) and s0 + 2q + 1 (imaginary part); the
    // sequence index runs fastest so that neighbouring threads read neighbouring addresses when
    // the sequences interleave (in_ss == 1)
    const int nsb = min(2 * P, d.nseq - s0);
    for (int t = tid; t < d.n_in * nsb; t += nth) {
        const int j = t / nsb, sl = t % nsb;
        const float v = d.in[(long long)(s0 + sl) * d.in_ss + (long long)j * d.in_es];
        const unsigned pos = __brev((unsigned)(j * d.stuff)) >> (32 - d.logM);
        R *c = reinterpret_cast<R *>(&fbuf[(sl >> 1) * M + pos]);
        c[sl & 1] = (R)v;
    }
    __syncthreads();
    // forward: decimation in time, bit-reversed in, natural order out
    for (int len = 2, lg = 1; len <= M; len <<= 1, ++lg) {
        const int half = len >> 1, tstep = M >> lg;
        for (int b = tid; b < P * half_M; b += nth) {
            const int q = b / half_M, bb = b - q * half_M;
            const int p = bb & (half - 1), i = ((bb >> (lg - 1)) << lg) + p, j = i + half;
            C *f = fbuf + q * M;
            const C t = cmulc(tw[p * tstep], f[j]), a = f[i];
            f[i] = Cplx<R>::make(a.x + t.x, a.y + t.y);
            f[j] = Cplx<R>::make(a.x - t.x, a.y - t.y);
        }
        __syncthreads();
    }
    for (int i = tid; i < P * M; i += nth) fbuf[i] = cmulc(fbuf[i], G[i & (M - 1)]);
    __syncthreads();
    // inverse: decimation in frequency with conjugate twiddles, natural in, bit-reversed out
    for (int len = M, lg = d.logM; len >= 2; len >>= 1, --lg) {
        const int half = len >> 1, tstep = M >> lg;
        for (int b = tid; b < P * half_M; b += nth) {
            const int q = b / half_M, bb = b - q * half_M;
            const int p = bb & (half - 1), i = ((bb >> (lg - 1)) << lg) + p, j = i + half;
            C *f = fbuf + q * M;
            const C w = tw[p * tstep], a = f[i], c = f[j];
            f[i] = Cplx<R>::make(a.x + c.x, a.y + c.y);
            f[j] = cmulc(Cplx<R>::make(a.x - c.x, a.y - c.y), Cplx<R>::make(w.x, -w.y));
        }
        __syncthreads();
    }
    for (int t = tid; t < d.n_out * nsb; t += nth) {
        const int i = t / nsb, sl = t % nsb;
        float v = 0.f;
        if (i < d.N) {
            const unsigned pos = __brev((unsigned)i) >> (32 - d.logM);
            const R *c = reinterpret_cast<const R *>(&fbuf[(sl >> 1) * M + pos]);
            v = (float)c[sl & 1];
        }
        d.out[(long long)(s0 + sl) * d.out_ss + (long long)i * d.out_es] = v;
    }
}

constexpr int FFT_CONV_MAX = 16384;      // largest M one block holds in FP32 (128 KB of shared memory)
constexpr int FFT_CONV_MAX_F64 = 8192;   // largest M one block holds in FP64 (128 KB)

// The transforms run in FP64 where the block holds them (M <= 8192): the filtered residual can
// be much smaller than the residual (a low-pass far below the source's band), and an FP32
// transform's rounding, relative to the input, then shows in the output.
static inline bool conv_in_f64(int M) { return M <= FFT_CONV_MAX_F64; }

// fills M, logM and P of d (M from d.N, as fwi_conv_size) and launches; cudaErrorInvalidValue when
// M > FFT_CONV_MAX, the sizes do not fit, or d.dbl does not match conv_in_f64(M)
static inline cudaError_t launch_fft_conv(ConvDesc d, cudaStream_t st)
{
    int M = 2, lg = 1;  // the size fwi_conv_size gives, for which G and tw were built
    while (M < 2 * d.N - 1) M <<= 1, ++lg;
    if (M > FFT_CONV_MAX || d.N < 1 || d.nseq < 1 || d.n_in < 1 || (d.n_in - 1) * d.stuff >= d.N ||
        (d.dbl != 0) != conv_in_f64(M))
        return cudaErrorInvalidValue;
    d.M = M;
    d.logM = lg;
    const size_t csize = d.dbl ? 16 : 8;
    d.P = M >= 8192 ? 1 : 8192 / M;  // up to 64 KB (FP32) / 128 KB (FP64) of pairs per block
    d.P = d.P < (d.nseq + 1) / 2 ? d.P : (d.nseq + 1) / 2;
    const size_t smem = (size_t)d.P * M * csize;
    const void *fn = d.dbl ? (const void *)k_fft_conv<double> : (const void *)k_fft_conv<float>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int blocks = (d.nseq + 2 * d.P - 1) / (2 * d.P);
    if (d.dbl) k_fft_conv<double><<<blocks, 512, smem, st>>>(d);
    else k_fft_conv<float><<<blocks, 512, smem, st>>>(d);
    return cudaGetLastError();
}

}  // namespace fwi
