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

// The core of an M-point circular convolution of the P sequences in fbuf (each loaded at its
// bit-reversed positions): radix-2 decimation in time (natural order out), multiplication by the
// spectrum G (which carries the 1 / M), and the inverse by decimation in frequency with conjugate
// twiddles (bit-reversed order out).  Every thread of the block takes part.
template <class R>
__device__ __forceinline__ void fft_conv_core(typename Cplx<R>::T *fbuf, int P, int M, int logM,
                                              const typename Cplx<R>::T *G, const typename Cplx<R>::T *tw)
{
    typedef typename Cplx<R>::T C;
    const int tid = threadIdx.x, nth = blockDim.x, half_M = M >> 1;
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
    for (int len = M, lg = logM; len >= 2; len >>= 1, --lg) {
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
}

// grid: ceil(nseq / (2 P)) blocks; dynamic shared memory P * M complex values of type R
template <class R>
static __global__ void __launch_bounds__(512) k_fft_conv(const ConvDesc d)
{
    typedef typename Cplx<R>::T C;
    extern __shared__ __align__(16) unsigned char fsm[];
    C *fbuf = reinterpret_cast<C *>(fsm);
    const C *G = static_cast<const C *>(d.G), *tw = static_cast<const C *>(d.tw);
    const int M = d.M, P = d.P;
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
    fft_conv_core<R>(fbuf, P, M, d.logM, G, tw);
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

// ---------------------------------------------------------------- DFTs of any length (Bluestein)
// An N-point DFT X_k = sum_j x_j e^{-2 pi i jk / N} is conj(b_k) times the convolution of
// u_j = x_j conj(b_j) with b, b_m = e^{i pi m^2 / N} (jk = (j^2 + k^2 - (k - j)^2) / 2); the inverse
// direction (e^{+2 pi i jk / N}) uses the conjugate chirps.  The convolution runs as the M-point
// one above (M the power of two >= 2N - 1) with the spectrum of b wrapped onto M points.
// With a window, the first DFT's result is multiplied by a real window and transformed again in
// the opposite direction in the same block: the chirp that ends the first DFT and the one that
// starts the second multiply to |b_j|^2 = 1, so the window multiplies the convolution's output.
struct BlueDesc {
    const void *in;             // input: element j of sequence s at in[s * in_ss + j * in_es]
    long long in_es, in_ss;
    int in_cplx;                // 1: float2 values, 0: float (imaginary part 0)
    void *out;                  // output position k (o0 <= k < o0 + no) of sequence s at
    long long out_es, out_ss;   //   out[s * out_ss + (k - o0) * out_es]
    int out_real;               // 1: the real part as float, divided by `divisor`; 0: float2
    float divisor;
    int o0, no;
    int N, nseq, M, logM, P;
    int dir;                    // direction of the first DFT: -1 forward, +1 inverse
    const float *win;           // null, or the window: position k of sequence s at win[k * win_es + s * win_ss]
    long long win_es, win_ss;
    const void *tables;         // fwi_bluestein_tables: chirp (N), spectrum of b (M), of conj(b) (M)
    const void *tw;             // exp(-2 pi i k / M), k < M / 2
    int dbl;                    // tables and transforms in FP64
};

// grid: ceil(nseq / P) blocks; dynamic shared memory P * M complex values of type R
template <class R>
static __global__ void __launch_bounds__(512) k_bluestein(const BlueDesc d)
{
    typedef typename Cplx<R>::T C;
    extern __shared__ __align__(16) unsigned char fsm[];
    C *fbuf = reinterpret_cast<C *>(fsm);
    const C *chirp = static_cast<const C *>(d.tables), *Bf = chirp + d.N, *Bi = Bf + d.M;
    const C *tw = static_cast<const C *>(d.tw);
    const int M = d.M, P = d.P, N = d.N, sh = 32 - d.logM;
    const int s0 = blockIdx.x * P, nsb = min(P, d.nseq - s0);
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int i = tid; i < P * M; i += nth) fbuf[i] = Cplx<R>::make(0, 0);
    __syncthreads();
    for (int t = tid; t < N * nsb; t += nth) {
        const int j = t / nsb, sl = t - j * nsb;
        const long long a = (long long)(s0 + sl) * d.in_ss + (long long)j * d.in_es;
        C v;
        if (d.in_cplx) {
            const float2 f = static_cast<const float2 *>(d.in)[a];
            v = Cplx<R>::make(f.x, f.y);
        } else {
            v = Cplx<R>::make(static_cast<const float *>(d.in)[a], 0);
        }
        const C b = chirp[j];
        fbuf[sl * M + (__brev((unsigned)j) >> sh)] = cmulc(v, Cplx<R>::make(b.x, d.dir < 0 ? -b.y : b.y));
    }
    __syncthreads();
    fft_conv_core<R>(fbuf, P, M, d.logM, d.dir < 0 ? Bf : Bi, tw);
    int dir = d.dir;
    if (d.win) {
        for (int i = tid; i < P * M; i += nth) {
            const int sl = i / M, p = i - sl * M, j = (int)(__brev((unsigned)p) >> sh);
            if (sl < nsb && j < N) {
                const R w = (R)d.win[(long long)j * d.win_es + (long long)(s0 + sl) * d.win_ss];
                fbuf[i] = Cplx<R>::make(fbuf[i].x * w, fbuf[i].y * w);
            } else {
                fbuf[i] = Cplx<R>::make(0, 0);
            }
        }
        __syncthreads();
        dir = -dir;
        fft_conv_core<R>(fbuf, P, M, d.logM, dir < 0 ? Bf : Bi, tw);
    }
    for (int t = tid; t < d.no * nsb; t += nth) {
        const int kk = t / nsb, sl = t - kk * nsb, k = d.o0 + kk;
        const C b = chirp[k];
        const C v = cmulc(fbuf[sl * M + (__brev((unsigned)k) >> sh)], Cplx<R>::make(b.x, dir < 0 ? -b.y : b.y));
        const long long a = (long long)(s0 + sl) * d.out_ss + (long long)kk * d.out_es;
        if (d.out_real) static_cast<float *>(d.out)[a] = (float)v.x / d.divisor;
        else static_cast<float2 *>(d.out)[a] = make_float2((float)v.x, (float)v.y);
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

// fills M, logM and P of d (M = the power of two >= 2N - 1, for which the tables were built) and
// launches; cudaErrorInvalidValue when M > FFT_CONV_MAX, the output range leaves [0, N), or d.dbl
// does not match conv_in_f64(M)
static inline cudaError_t launch_bluestein(BlueDesc d, cudaStream_t st)
{
    int M = 2, lg = 1;
    while (M < 2 * d.N - 1) M <<= 1, ++lg;
    if (M > FFT_CONV_MAX || d.N < 1 || d.nseq < 1 || d.o0 < 0 || d.no < 1 || d.o0 + d.no > d.N ||
        (d.dbl != 0) != conv_in_f64(M))
        return cudaErrorInvalidValue;
    d.M = M;
    d.logM = lg;
    const size_t csize = d.dbl ? 16 : 8;
    d.P = M >= 8192 ? 1 : 8192 / M;
    d.P = d.P < d.nseq ? d.P : d.nseq;
    const size_t smem = (size_t)d.P * M * csize;
    const void *fn = d.dbl ? (const void *)k_bluestein<double> : (const void *)k_bluestein<float>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int blocks = (d.nseq + d.P - 1) / d.P;
    if (d.dbl) k_bluestein<double><<<blocks, 512, smem, st>>>(d);
    else k_bluestein<float><<<blocks, 512, smem, st>>>(d);
    return cudaGetLastError();
}

}  // namespace fwi
