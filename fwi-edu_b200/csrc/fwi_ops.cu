// fwi_ops.cu -- the reference-named FWI-loop operations (optimization.c, common.c),
// computed on the device.  These keep the reference's host-array interfaces so a
// front-end written against FWI-EDU links unchanged; each call stages its arrays
// through one process-wide device workspace.  The device-resident FWI iteration of
// fwi_engine.cu runs the same kernels without the host round trips.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fwi_b200.h"
#include "fwi_aux.cuh"
#include "fwi_optim.cuh"
#include "fwi_fft.cuh"
#include "fwi_setup.h"

using namespace fwi;

namespace {

struct Ops {
    int dev = -1;
    cudaStream_t st = nullptr;
    char *buf = nullptr;
    size_t cap = 0;
};
Ops g_ops;
std::mutex g_ops_mu;

bool report(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return true;
    fprintf(stderr, "<error>: %s: %s\n", what, cudaGetErrorString(e));
    return false;
}

// workspace of at least `bytes`, 256-byte aligned sub-buffers handed out by offset
bool ops_ready(size_t bytes)
{
    int dev = 0;
    if (const char *p = getenv("FWI_DEVICE")) dev = atoi(p);
    if (g_ops.dev != dev) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= dev) {
            fprintf(stderr, "<error>: no CUDA device %d: the FWI operations run on the GPU only\n", dev);
            return false;
        }
        if (!report(cudaSetDevice(dev), "cudaSetDevice")) return false;
        if (!report(cudaStreamCreateWithFlags(&g_ops.st, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
        g_ops.dev = dev;
    }
    if (!report(cudaSetDevice(dev), "cudaSetDevice")) return false;
    if (bytes > g_ops.cap) {
        if (g_ops.buf) cudaFree(g_ops.buf);
        g_ops.buf = nullptr;
        g_ops.cap = 0;
        if (!report(cudaMalloc(&g_ops.buf, bytes), "cudaMalloc")) return false;
        g_ops.cap = bytes;
    }
    return true;
}

size_t al(size_t b) { return (b + 255) & ~size_t(255); }

// ---- device tables built once on the host per (kind, size, parameters) and kept
std::map<std::string, float *> g_opmats;

std::string fbits(float v)
{
    unsigned u;
    memcpy(&u, &v, 4);
    return std::to_string(u);
}

const float *op_matrix(const std::string &key, size_t count, void (*build)(float *, const int *, const float *),
                       const int *ip, const float *fp)
{
    auto it = g_opmats.find(key);
    if (it != g_opmats.end()) return it->second;
    std::vector<float> h(count);
    build(h.data(), ip, fp);
    float *d = nullptr;
    if (!report(cudaMalloc(&d, count * 4), "cudaMalloc")) return nullptr;
    if (!report(cudaMemcpy(d, h.data(), count * 4, cudaMemcpyHostToDevice), "copy")) return nullptr;
    g_opmats[key] = d;
    return d;
}

// ---- residual filters and interpolation: FFT convolutions (fwi_fft.cuh) with the kernel's
// spectrum and the twiddles built once on the host (FP64) and kept on the device
struct Kernel1d {
    int kind;  // 0 / 1: apply_traces_lowpass / _bandpass of length n; 2: interpolate_traces from ns by r
    int n, r;
    float fpass, fcut, dt;
};

void build_spectrum(float *out, const int *ip, const float *fp)
{
    const int kind = ip[0], n = ip[1], r = ip[2], N = ip[3], M = fwi_conv_size(N);
    std::vector<double> h(N);
    if (kind == 2) fwi_interp_kernel(n, r, h.data());
    else fwi_filter_kernel(kind, n, fp[0], fp[1], fp[2], h.data());
    if (conv_in_f64(M)) fwi_conv_spectrum_f64(h.data(), N, M, reinterpret_cast<double *>(out));
    else fwi_conv_spectrum(h.data(), N, M, out);
}
void build_twiddles(float *out, const int *ip, const float *)
{
    if (conv_in_f64(ip[0])) fwi_fft_twiddles_f64(ip[0], reinterpret_cast<double *>(out));
    else fwi_fft_twiddles(ip[0], out);
}

// the tables of a convolution of length N into d; false (with a message) when N is too long
bool conv_tables(const Kernel1d &k, int N, ConvDesc *d)
{
    const int M = fwi_conv_size(N);
    if (M > FFT_CONV_MAX) {
        fprintf(stderr, "<error>: FFT convolution of length %d needs %d points (at most %d)\n", N, M, FFT_CONV_MAX);
        return false;
    }
    const bool f64 = conv_in_f64(M);
    const int ip[4] = {k.kind, k.n, k.r, N};
    const float fp[3] = {k.fpass, k.fcut, k.dt};
    const float *G = op_matrix("s" + std::to_string(k.kind) + "/" + std::to_string(k.n) + "/" + std::to_string(k.r) +
                                   "/" + fbits(k.fpass) + "/" + fbits(k.fcut) + "/" + fbits(k.dt),
                               (size_t)(f64 ? 4 : 2) * M, build_spectrum, ip, fp);
    const int ipt[1] = {M};
    const float *tw = op_matrix("tw/" + std::to_string(M), (size_t)(f64 ? 2 : 1) * M, build_twiddles, ipt, nullptr);
    if (!G || !tw) return false;
    d->G = G;
    d->tw = tw;
    d->dbl = f64 ? 1 : 0;
    d->N = N;
    return true;
}

bool run_conv(const ConvDesc &d, const char *what)
{
    return report(launch_fft_conv(d, g_ops.st), what);
}

// y (nvec sequences of n samples at element stride es, sequence stride ss) = filter applied to x
bool filter_vectors(const float *x, float *y, int n, int nvec, long long es, long long ss, int filter, float fpass,
                    float fcut, float dt)
{
    ConvDesc d{};
    if (!conv_tables({filter, n, 1, fpass, fcut, dt}, n, &d)) return false;
    d.in = x; d.in_es = es; d.in_ss = ss; d.n_in = n; d.stuff = 1;
    d.out = y; d.out_es = es; d.out_ss = ss; d.n_out = n; d.nseq = nvec;
    return run_conv(d, "FFT convolution");
}

// the taper of taper_traces (common.c:796-895) on a [ntr][ns] device gather
bool taper_device(float *a, int ns, int ntr, int Lt, int Lr, const float *tct, const float *tcr, TaperDesc *d)
{
    TaperDesc t{a, tct, tcr, ns, ntr, Lt, Lr};
    if (!report(cudaMemcpyAsync(d, &t, sizeof(t), cudaMemcpyHostToDevice, g_ops.st), "copy")) return false;
    k_taper<<<dim3(148, 1), 256, 0, g_ops.st>>>(d);
    return report(cudaGetLastError(), "k_taper");
}

// FP64 sums of one or two operand arrays already on the device
bool dsum(const float *a, const float *b, long long n, int op, double out[2])
{
    const int NP = 592;
    char *base = g_ops.buf + g_ops.cap - al(sizeof(SumDesc)) - al(2 * NP * 8 + 16);
    SumDesc h{};
    h.a = a;
    h.b = b;
    h.n = n;
    h.op = op;
    h.partial = (double *)(base + al(sizeof(SumDesc)));
    double *res = h.partial + 2 * NP;
    if (!report(cudaMemcpyAsync(base, &h, sizeof(h), cudaMemcpyHostToDevice, g_ops.st), "copy")) return false;
    k_sum_partial<256><<<dim3(NP, 1), 256, 0, g_ops.st>>>((const SumDesc *)base);
    k_sum_final<<<1, 32, 0, g_ops.st>>>((const SumDesc *)base, NP, res);
    if (!report(cudaMemcpyAsync(out, res, 16, cudaMemcpyDeviceToHost, g_ops.st), "copy")) return false;
    return report(cudaStreamSynchronize(g_ops.st), "reduction");
}
const size_t RED_BYTES = 2 * 592 * 8 + 4096;

}  // namespace

// calculate_objective_value, optimization.c:99-132: 0.5 * sum over shots of traces^2 (FP64)
extern "C" float calculate_objective_value(Record2D *r, int Nshot)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    long long n = 0;
    for (int i = 0; i < Nshot; i++) n += (long long)r[i].ntr * r[i].ns;
    if (!ops_ready(al(n * 4) + RED_BYTES)) return NAN;
    float *d = (float *)g_ops.buf;
    long long off = 0;
    for (int i = 0; i < Nshot; i++) {
        size_t b = (size_t)r[i].ntr * r[i].ns * 4;
        if (!report(cudaMemcpyAsync(d + off, r[i].traces_p[0], b, cudaMemcpyHostToDevice, g_ops.st), "copy")) return NAN;
        off += (long long)r[i].ntr * r[i].ns;
    }
    double s[2];
    if (!dsum(d, nullptr, n, 1, s)) return NAN;
    return (float)(0.5 * s[0]);
}

// calculate_step_length, optimization.c:134-176: sum r0 (r0 - r1) / sum (r0 - r1)^2
extern "C" float calculate_step_length(Record2D *p0, Record2D *p1, int Nshot)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    long long n = 0;
    for (int i = 0; i < Nshot; i++) n += (long long)p0[i].ntr * p0[i].ns;
    if (!ops_ready(2 * al(n * 4) + RED_BYTES)) return NAN;
    float *a = (float *)g_ops.buf, *b = (float *)(g_ops.buf + al(n * 4));
    long long off = 0;
    for (int i = 0; i < Nshot; i++) {
        size_t nb = (size_t)p0[i].ntr * p0[i].ns * 4;
        cudaMemcpyAsync(a + off, p0[i].traces_p[0], nb, cudaMemcpyHostToDevice, g_ops.st);
        cudaMemcpyAsync(b + off, p1[i].traces_p[0], nb, cudaMemcpyHostToDevice, g_ops.st);
        off += (long long)p0[i].ntr * p0[i].ns;
    }
    double s[2];
    if (!dsum(a, b, n, 3, s)) return NAN;
    if (s[1] == 0.0) {
        fprintf(stderr, "<warning>: denominator is zero in step length calculation, returning 0.\n");
        return 0.0f;
    }
    return (float)(s[0] / s[1]);
}

// compute_model_perturbation, optimization.c:178-298
extern "C" float compute_model_perturbation(float fraction, float *slowness, float *gradient, float *out, int len)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    if (len <= 0) return 0.0f;
    size_t nb = al((size_t)len * 4);
    if (!ops_ready(3 * nb + al(sizeof(PertState)) + RED_BYTES)) return NAN;
    float *g = (float *)g_ops.buf, *sl = (float *)(g_ops.buf + nb), *o = (float *)(g_ops.buf + 2 * nb);
    PertState *st = (PertState *)(g_ops.buf + 3 * nb);
    cudaMemcpyAsync(g, gradient, (size_t)len * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(sl, slowness, (size_t)len * 4, cudaMemcpyHostToDevice, g_ops.st);
    double s[2];
    if (!dsum(sl, nullptr, len, 0, s)) return NAN;
    double *ssum = (double *)((char *)st + offsetof(PertState, avg_slow));
    k_pert_init<<<1, 256, 0, g_ops.st>>>(st);
    cudaMemcpyAsync(ssum, &s[0], 8, cudaMemcpyHostToDevice, g_ops.st);
    k_pert_minmax<<<296, 256, 0, g_ops.st>>>(g, len, st);
    k_pert_hist<<<296, 256, 0, g_ops.st>>>(g, len, st);
    k_pert_scalar<<<1, 32, 0, g_ops.st>>>(st, ssum, len, fraction);
    k_pert_apply<<<296, 256, 0, g_ops.st>>>(g, o, len, st);
    float scalar = NAN;
    cudaMemcpyAsync(&scalar, (char *)st + offsetof(PertState, scalar), 4, cudaMemcpyDeviceToHost, g_ops.st);
    cudaMemcpyAsync(out, o, (size_t)len * 4, cudaMemcpyDeviceToHost, g_ops.st);
    if (!report(cudaStreamSynchronize(g_ops.st), "compute_model_perturbation")) return NAN;
    return scalar;
}

// smooth2D, common.c:927-1040: one cos^2 pass along z (iszdirect == 1) or x
extern "C" void smooth2D(float **in, float **out, int nx, int nz, int N, int iszdirect)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    size_t m = (size_t)nx * nz;
    size_t nb = al(m * 4);
    if (!ops_ready(2 * nb + al((2 * N + 1) * 4))) return;
    std::vector<float> w(2 * N + 1);
    for (int i = 0; i < 2 * N + 1; i++) {
        w[i] = (float)cos(3.141592653589793 * (i - N) / (2.0 * N));
        w[i] *= w[i];
    }
    float *a = (float *)g_ops.buf, *b = (float *)(g_ops.buf + nb), *dw = (float *)(g_ops.buf + 2 * nb);
    cudaMemcpyAsync(a, in[0], m * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(dw, w.data(), w.size() * 4, cudaMemcpyHostToDevice, g_ops.st);
    k_smooth2d<<<592, 256, 0, g_ops.st>>>(a, b, nx, nz, N, iszdirect == 1, dw);
    cudaMemcpyAsync(out[0], b, m * 4, cudaMemcpyDeviceToHost, g_ops.st);
    report(cudaStreamSynchronize(g_ops.st), "smooth2D");
}

// compute_adjoint_source2d, optimization.c:300-419: residual; for filters 0/1 the time taper, time
// filter, trace taper and trace filter (FFT convolutions); both tapers
extern "C" void compute_adjoint_source2d(Record2D *pre, Record2D *obs, float **vp, float freq, int filter,
                                         Record2D *adj)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    if (filter < 0 || filter > 2) {
        fprintf(stderr, "<error>: compute_adjoint_source2d: residual filter %d (0 lowpass, 1 bandpass, 2 none)\n",
                filter);
        return;
    }
    const int ns = adj->ns, ntr = adj->ntr;
    double vp_sum = 0.0;
    for (int i = 0; i < ntr; i++) vp_sum += vp[adj->igx[i]][adj->igz[i]];  // window-local igx, global vp
    float vp_avg = (float)(vp_sum / ntr);
    if (freq == 0.0f) freq = adj->fpeak;
    float kpass = freq / vp_avg;
    int Lt = (int)roundf((2.0f / freq) / adj->dt) + 1;
    int Lr = (int)roundf((2.0f / kpass) / adj->dtr) + 1;
    if (Lt > 0 && Lt > ns / 3) Lt = ns / 3;
    if (Lr > 0 && Lr > ntr / 3) Lr = ntr / 3;
    if (Lt < 0) Lt = 0;
    if (Lr < 0) Lr = 0;
    std::vector<float> tct(Lt + 1), tcr(Lr + 1);
    if (Lt > 0) fwi_taper_coefs(Lt, tct.data());
    if (Lr > 0) fwi_taper_coefs(Lr, tcr.data());
    size_t m = (size_t)ns * ntr, nb = al(m * 4);
    const size_t tb = al((Lt + 1) * 4) + al((Lr + 1) * 4);
    if (!ops_ready(3 * nb + tb + al(sizeof(TaperDesc)) + 256)) return;
    float *dp = (float *)g_ops.buf, *dob = (float *)(g_ops.buf + nb), *da = (float *)(g_ops.buf + 2 * nb);
    float *dt_ = (float *)(g_ops.buf + 3 * nb), *dr = (float *)(g_ops.buf + 3 * nb + al((Lt + 1) * 4));
    TaperDesc *td = (TaperDesc *)(g_ops.buf + 3 * nb + tb);
    cudaMemcpyAsync(dp, pre->traces_p[0], m * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(dob, obs->traces_p[0], m * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(dt_, tct.data(), (Lt + 1) * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(dr, tcr.data(), (Lr + 1) * 4, cudaMemcpyHostToDevice, g_ops.st);
    if (filter == 2) {
        k_residual_taper<<<296, 256, 0, g_ops.st>>>(dp, dob, da, ns, ntr, Lt, Lr, dt_, dr);
    } else {
        k_residual_taper<<<296, 256, 0, g_ops.st>>>(dp, dob, da, ns, ntr, Lt, 0, dt_, dr);
        // time filter of every trace, trace taper, filter along the traces of every sample, tapers
        if (!filter_vectors(da, dp, ns, ntr, 1, ns, filter, freq, 2.0f * freq, adj->dt)) {
            fprintf(stderr, "<error>: compute_adjoint_source2d: time filter failed\n");
            return;
        }
        if (!taper_device(dp, ns, ntr, 0, Lr, dt_, dr, td)) return;
        if (!filter_vectors(dp, dp, ntr, ns, ns, 1, filter, kpass, 2.0f * kpass, adj->dtr)) {
            fprintf(stderr, "<error>: compute_adjoint_source2d: trace filter failed\n");
            return;
        }
        cudaStreamSynchronize(g_ops.st);  // the taper descriptor is reused
        if (!taper_device(dp, ns, ntr, Lt, Lr, dt_, dr, td)) return;
        da = dp;
    }
    cudaMemcpyAsync(adj->traces_p[0], da, m * 4, cudaMemcpyDeviceToHost, g_ops.st);
    report(cudaStreamSynchronize(g_ops.st), "compute_adjoint_source2d");
}

// apply_traces_lowpass / apply_traces_bandpass (common.c:584-794): ntr traces of nt samples,
// tr and trs in the alloc2float(nt, ntr) layout (one contiguous block); tr == trs is allowed
static void traces_filter(float **tr, float **trs, int nt, int ntr, float fpass, float fcut, float dt, int filter,
                          const char *name)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    if (!tr || !trs || nt <= 0 || ntr <= 0) {
        fprintf(stderr, "<error>: %s: invalid input (nt=%d, ntr=%d)\n", name, nt, ntr);
        return;
    }
    if (fcut <= fpass) {
        fprintf(stderr, "<error>: %s: fcut must be greater than fpass!\n", name);
        return;
    }
    const size_t m = (size_t)nt * ntr, nb = al(m * 4);
    if (!ops_ready(2 * nb)) return;
    float *x = (float *)g_ops.buf, *y = (float *)(g_ops.buf + nb);
    cudaMemcpyAsync(x, tr[0], m * 4, cudaMemcpyHostToDevice, g_ops.st);
    if (!filter_vectors(x, y, nt, ntr, 1, nt, filter, fpass, fcut, dt)) {
        fprintf(stderr, "<error>: %s: FFT convolution failed\n", name);
        return;
    }
    cudaMemcpyAsync(trs[0], y, m * 4, cudaMemcpyDeviceToHost, g_ops.st);
    report(cudaStreamSynchronize(g_ops.st), name);
}

extern "C" void apply_traces_lowpass(float **tr, float **trs, int nt, int ntr, float fpass, float fcut, float dt)
{
    traces_filter(tr, trs, nt, ntr, fpass, fcut, dt, 0, "apply_traces_lowpass");
}

extern "C" void apply_traces_bandpass(float **tr, float **trs, int nt, int ntr, float fpass, float fcut, float dt)
{
    traces_filter(tr, trs, nt, ntr, fpass, fcut, dt, 1, "apply_traces_bandpass");
}

// interpolate_traces (common.c:482-582): ntr traces of nt samples -> ns = (nt - 1) r + 1 samples
extern "C" void interpolate_traces(float **tr, int ntr, int nt, int r, float **trs)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    if (ntr <= 0 || nt <= 0 || !tr || !trs) {
        fprintf(stderr, "<error>: invalid input (ntr=%d, nt=%d) in function interpolate_traces!\n", ntr, nt);
        return;
    }
    if (r <= 1) {
        memcpy(trs[0], tr[0], sizeof(float) * (size_t)ntr * nt);
        return;
    }
    const int ns = (nt - 1) * r + 1;
    const size_t nb = al((size_t)nt * ntr * 4);
    if (!ops_ready(nb + al((size_t)ns * ntr * 4))) return;
    float *x = (float *)g_ops.buf, *y = (float *)(g_ops.buf + nb);
    ConvDesc d{};
    if (!conv_tables({2, nt, r, 0.f, 0.f, 0.f}, ns, &d)) return;
    cudaMemcpyAsync(x, tr[0], sizeof(float) * (size_t)nt * ntr, cudaMemcpyHostToDevice, g_ops.st);
    // each trace zero-stuffed by r and convolved with the band window's kernel
    d.in = x; d.in_es = 1; d.in_ss = nt; d.n_in = nt; d.stuff = r;
    d.out = y; d.out_es = 1; d.out_ss = ns; d.n_out = ns; d.nseq = ntr;
    if (!run_conv(d, "interpolate_traces")) return;
    cudaMemcpyAsync(trs[0], y, sizeof(float) * (size_t)ns * ntr, cudaMemcpyDeviceToHost, g_ops.st);
    report(cudaStreamSynchronize(g_ops.st), "interpolate_traces");
}

// ---- 2-D wavenumber filters: Y = crop(IDFT2(W . DFT2(pad(X)))) / (Nz Nx) as five FP32 GEMMs
namespace {

void build_wn_window(float *h, const int *ip, const float *fp)
{
    fwi_wavenumber_window(ip[0], ip[1], ip[2], fp[0], fp[1], fp[2], fp[3], h);
}
void build_bluestein(float *h, const int *ip, const float *)
{
    fwi_bluestein_tables(ip[0], fwi_conv_size(ip[0]), conv_in_f64(fwi_conv_size(ip[0])) ? 1 : 0, h);
}

// the chirp and spectra of an N-point DFT, and the twiddles of its convolution size, into d
bool dft_tables(int N, BlueDesc *d)
{
    const int M = fwi_conv_size(N);
    if (M > FFT_CONV_MAX) {
        fprintf(stderr, "<error>: a DFT of length %d needs %d-point transforms (at most %d)\n", N, M, FFT_CONV_MAX);
        return false;
    }
    const bool f64 = conv_in_f64(M);
    const int ip[1] = {N}, ipt[1] = {M};
    const float *t = op_matrix("bl/" + std::to_string(N), (size_t)(f64 ? 2 : 1) * 2 * (N + 2 * (size_t)M),
                               build_bluestein, ip, nullptr);
    const float *tw = op_matrix("tw/" + std::to_string(M), (size_t)(f64 ? 2 : 1) * M, build_twiddles, ipt, nullptr);
    if (!t || !tw) return false;
    d->tables = t;
    d->tw = tw;
    d->dbl = f64 ? 1 : 0;
    d->N = N;
    return true;
}

// the edge-replicating pad of pad_model2d (common.c:110-170): padded sample (z, x) takes the
// model's sample at the clamped position
__global__ void k_pad_replicate(const float *__restrict__ x, int nz, int nx, int pad, float *__restrict__ y, int Nz,
                                long long plane)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
         i += (long long)gridDim.x * blockDim.x) {
        const int X = (int)(i / Nz), Z = (int)(i - (long long)X * Nz);
        const int xs = min(max(X - pad, 0), nx - 1), zs = min(max(Z - pad, 0), nz - 1);
        y[i] = x[(long long)xs * nz + zs];
    }
}

// lowpass2d / bandpass2d: taper, edge-replicating pad, 2-D DFT of the padded field, the
// reference's float window, inverse 2-D DFT, / (Nz Nx), crop (common.c:1042-1284).  The DFTs have
// the padded field's own sizes (the window is defined on that grid) and run as Bluestein
// transforms on the device in three launches: the z transforms of every padded column; for every
// z wavenumber the x transform, the window and the inverse x transform, kept at the model's
// columns only; the inverse z transforms of those columns, kept at the model's rows.
void wavenumber_filter(float **s, int nz, int nx, float dz, float dx, float kpass, float kcut, float **s_filter,
                       int filter, const char *name)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    if (!s || !s_filter || nz <= 0 || nx <= 0) {
        fprintf(stderr, "<error>: %s: invalid input (nz=%d, nx=%d)\n", name, nz, nx);
        return;
    }
    if (!(kpass > 0.0f) || kcut <= kpass) {
        fprintf(stderr, "<error>: %s: need 0 < kpass < kcut (kpass=%g, kcut=%g)\n", name, kpass, kcut);
        return;
    }
    // taper lengths and pad as lowpass2d (common.c:1079-1091); taper_traces clamps to a third
    const int Lx = (int)roundf(4 / (kpass * dx)), Lz = (int)roundf(4 / (kpass * dz));
    const int pad = 10 * (Lx > Lz ? Lx : Lz);
    const int Lt = Lz > nz / 3 ? nz / 3 : Lz, Lr = Lx > nx / 3 ? nx / 3 : Lx;
    const long long Nz = nz + 2LL * pad, Nx = nx + 2LL * pad;
    if (Nz * Nx > (1LL << 31) / 2) {
        fprintf(stderr, "<error>: %s: padded field %lld x %lld too large\n", name, Nz, Nx);
        return;
    }
    BlueDesc dz_{}, dx_{};
    if (!dft_tables((int)Nz, &dz_) || !dft_tables((int)Nx, &dx_)) return;
    std::vector<float> tct(Lt + 1), tcr(Lr + 1);
    if (Lt > 0) fwi_taper_coefs(Lt, tct.data());
    if (Lr > 0) fwi_taper_coefs(Lr, tcr.data());
    const size_t m = (size_t)nz * nx, plane = (size_t)(Nz * Nx);
    const size_t bx = al(m * 4), bP = al(plane * 4), bA = al(plane * 8), bG = al((size_t)nx * Nz * 8);
    const size_t bt = al((Lt + 1) * 4) + al((Lr + 1) * 4);
    if (!ops_ready(2 * bx + bP + bA + bG + bt + al(sizeof(TaperDesc)) + 256)) return;
    char *b = g_ops.buf;
    float *x = (float *)b, *P = (float *)(b + bx);
    float2 *A = (float2 *)(b + bx + bP), *Gc = (float2 *)(b + bx + bP + bA);
    float *Y = (float *)(b + bx + bP + bA + bG);
    float *dct = (float *)(b + 2 * bx + bP + bA + bG), *dcr = (float *)((char *)dct + al((Lt + 1) * 4));
    TaperDesc *td = (TaperDesc *)(b + 2 * bx + bP + bA + bG + bt);

    const int iNx = (int)Nx, iNz = (int)Nz;
    const int wi[3] = {filter, iNx, iNz};
    const float wf[4] = {dx, dz, kpass, kcut};
    const float *W = op_matrix("w2/" + std::to_string(filter) + "/" + std::to_string(iNx) + "/" +
                                   std::to_string(iNz) + "/" + fbits(dx) + "/" + fbits(dz) + "/" + fbits(kpass) +
                                   "/" + fbits(kcut),
                               plane, build_wn_window, wi, wf);
    if (!W) return;

    cudaMemcpyAsync(x, s[0], m * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(dct, tct.data(), (Lt + 1) * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(dcr, tcr.data(), (Lr + 1) * 4, cudaMemcpyHostToDevice, g_ops.st);
    if (!taper_device(x, nz, nx, Lt, Lr, dct, dcr, td)) return;
    cudaMemcpyAsync(s[0], x, m * 4, cudaMemcpyDeviceToHost, g_ops.st);  // the reference tapers its input
    k_pad_replicate<<<592, 256, 0, g_ops.st>>>(x, nz, nx, pad, P, iNz, (long long)plane);
    bool ok = report(cudaGetLastError(), "k_pad_replicate");
    // z transforms of the padded columns: A[x][kz]
    BlueDesc d1 = dz_;
    d1.in = P; d1.in_es = 1; d1.in_ss = Nz; d1.in_cplx = 0;
    d1.out = A; d1.out_es = 1; d1.out_ss = Nz; d1.out_real = 0; d1.o0 = 0; d1.no = iNz;
    d1.nseq = iNx; d1.dir = -1;
    ok = ok && report(launch_bluestein(d1, g_ops.st), name);
    // per z wavenumber: x transform, window W[kx][kz], inverse x transform at the model's columns
    BlueDesc d2 = dx_;
    d2.in = A; d2.in_es = Nz; d2.in_ss = 1; d2.in_cplx = 1;
    d2.win = W; d2.win_es = Nz; d2.win_ss = 1;
    d2.out = Gc; d2.out_es = Nz; d2.out_ss = 1; d2.out_real = 0; d2.o0 = pad; d2.no = nx;
    d2.nseq = iNz; d2.dir = -1;
    ok = ok && report(launch_bluestein(d2, g_ops.st), name);
    // inverse z transforms of the model's columns at the model's rows, real part / (Nz Nx)
    BlueDesc d3 = dz_;
    d3.in = Gc; d3.in_es = 1; d3.in_ss = Nz; d3.in_cplx = 1;
    d3.out = Y; d3.out_es = 1; d3.out_ss = nz; d3.out_real = 1; d3.divisor = (float)(iNz * iNx);
    d3.o0 = pad; d3.no = nz; d3.nseq = nx; d3.dir = 1;
    ok = ok && report(launch_bluestein(d3, g_ops.st), name);
    if (!ok) {
        cudaStreamSynchronize(g_ops.st);
        return;
    }
    cudaMemcpyAsync(s_filter[0], Y, m * 4, cudaMemcpyDeviceToHost, g_ops.st);
    report(cudaStreamSynchronize(g_ops.st), name);
}

}  // namespace

extern "C" void lowpass2d(float **s, int nz, int nx, float dz, float dx, float kpass, float kcut, float **s_filter)
{
    wavenumber_filter(s, nz, nx, dz, dx, kpass, kcut, s_filter, 0, "lowpass2d");
}

extern "C" void bandpass2d(float **s, int nz, int nx, float dz, float dx, float kpass, float kcut, float **s_filter)
{
    wavenumber_filter(s, nz, nx, dz, dx, kpass, kcut, s_filter, 1, "bandpass2d");
}

// apply_gradient_shot_precondition, optimization.c:58-97
extern "C" void apply_gradient_shot_precondition(float *grad, float *precond, int n)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    size_t nb = al((size_t)n * 4);
    if (!ops_ready(2 * nb + al(sizeof(PrecDesc)) + 256 + RED_BYTES)) return;
    float *g = (float *)g_ops.buf, *h = (float *)(g_ops.buf + nb);
    PrecDesc *pd = (PrecDesc *)(g_ops.buf + 2 * nb);
    double *sum = (double *)(g_ops.buf + 2 * nb + al(sizeof(PrecDesc)));
    cudaMemcpyAsync(g, grad, (size_t)n * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(h, precond, (size_t)n * 4, cudaMemcpyHostToDevice, g_ops.st);
    double s[2];
    if (!dsum(h, nullptr, n, 0, s)) return;
    PrecDesc p{g, h, n, sum};
    cudaMemcpyAsync(sum, &s[0], 8, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(pd, &p, sizeof(p), cudaMemcpyHostToDevice, g_ops.st);
    k_shot_precondition<<<dim3(148, 1), 256, 0, g_ops.st>>>(pd);
    cudaMemcpyAsync(grad, g, (size_t)n * 4, cudaMemcpyDeviceToHost, g_ops.st);
    cudaMemcpyAsync(precond, h, (size_t)n * 4, cudaMemcpyDeviceToHost, g_ops.st);
    report(cudaStreamSynchronize(g_ops.st), "apply_gradient_shot_precondition");
}

// apply_gradient_precondition, optimization.c:13-56: g /= (H + alpha * rms(H))
extern "C" void apply_gradient_precondition(float *grad, const float *precond, int n, float alpha)
{
    std::lock_guard<std::mutex> lk(g_ops_mu);
    if (alpha <= 0.0f) alpha = 0.005f;
    size_t nb = al((size_t)n * 4);
    if (!ops_ready(2 * nb + 256 + RED_BYTES)) return;
    float *g = (float *)g_ops.buf, *h = (float *)(g_ops.buf + nb);
    double *sum = (double *)(g_ops.buf + 2 * nb);
    cudaMemcpyAsync(g, grad, (size_t)n * 4, cudaMemcpyHostToDevice, g_ops.st);
    cudaMemcpyAsync(h, precond, (size_t)n * 4, cudaMemcpyHostToDevice, g_ops.st);
    double s[2];
    if (!dsum(h, nullptr, n, 2, s)) return;
    cudaMemcpyAsync(sum, &s[0], 8, cudaMemcpyHostToDevice, g_ops.st);
    k_global_precondition<<<296, 256, 0, g_ops.st>>>(g, h, n, sum, alpha);
    cudaMemcpyAsync(grad, g, (size_t)n * 4, cudaMemcpyDeviceToHost, g_ops.st);
    report(cudaStreamSynchronize(g_ops.st), "apply_gradient_precondition");
}

// calculate_memory_cost_checkpoint, checkpoint.c:267-298: GB of the (nCheckPoint + d - 2)-frame store
extern "C" float calculate_memory_cost_checkpoint(int nt, int NX, int NZ)
{
    int d = fwi_ck_interval(nt), n = fwi_ck_count(nt);
    int ntPoint = n + d - 2;
    return 1.0f * (ntPoint * NZ * NX * (int)sizeof(float)) / powf(1024.0f, 3);
}
