// fwi_kernels.cuh -- sm_100a kernels of the 2-D acoustic forward/adjoint engine.
//
// The hot kernel is k_step: one application of the 6th-order variable-density
// stencil (acoustic_iso2d_fd_it_6order, propagation.c:13-74) to a whole padded
// grid, fused with everything the reference does around it in the same time
// step: point source (propagation.c:558 / :662), mirror free surface (:76-101),
// receiver sampling (:567-576), adjoint injection (:676-682), pseudo-Hessian
// (:579-594) and the zero-lag imaging condition (:700-714).
//
// Thread layout.  Fields are [Nx][ld] floats, z fastest, ld = Nz rounded up to 4.
// A lane owns one float4 z-group (4 cells); the warps of a block stack along z and
// cover one whole column; the block then marches along x over a strip of LX
// columns, keeping p1 of columns x-3..x+3 in a 7-deep register queue, so every
// p1 element is loaded from memory once per strip.  The z-neighbours come from the
// adjacent lanes by warp shuffles; the two lanes at a warp edge fetch their halo
// group themselves.
//
// Arithmetic.  Every product and sum uses __fmul_rn/__fadd_rn/__fsub_rn in the
// reference's association order, so no multiply-add is contracted and each cell
// is rounded exactly as the reference's strict IEEE build rounds it.
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
    // coefficients [Nx][ld]
    const float *c1, *c2, *ck, *irx, *irz, *ir;
    // source terms per step: forward (double, propagation.c:558) and replay (float, :662)
    const double *srcd;
    const float *srcf;
    // receivers as a per-column list: colptr[Nx+1] into rec (padded z, trace index) and recK
    const int *colptr;
    const int2 *rec;
    const float *recK;
    float *traces_t;       // [ns][ntr] samples of the forward pass
    const float *adj_t;    // [nt][ntr] adjoint source
    // wavefield storage, each a sequence of frames of Nx*ld floats
    float *ckslots;        // 2*(K+1) checkpoint frames: slot 0 = u(-1), 2k+1 = u(kd), 2k = u(kd-1)
    float *fscr;           // 3 forward scratch frames
    float *rscr;           // 3 replay scratch frames
    float *seg;            // 2*S5 replayed frames kept for imaging (t % 5 == 0), double-buffered by segment
    float *ascr;           // 3 adjoint frames
    double *H, *Gacc;      // [Nx][ld] FP64 accumulators (pseudo-Hessian, gradient)
    long long frame;       // Nx*ld
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
__host__ __device__ inline float *frame_at(float *base, long long frame, int i) { return base + (long long)i * frame; }

// forward field u(t) in a pass that keeps checkpoints (mode 1) or not (mode 0)
__host__ __device__ inline float *fwd_buf(const ShotDesc &S, int t, bool keep)
{
    if (keep) {
        int s = stored_slot(S, t);
        if (s >= 0) return frame_at(S.ckslots, S.frame, s);
    }
    return frame_at(S.fscr, S.frame, (t + 3) % 3);
}
// replayed frame of segment k (checkpoint c = k*d), t > c, t % 5 == 0
__host__ __device__ inline float *seg_buf(const ShotDesc &S, int t)
{
    int k = t / S.d, c = k * S.d;
    int j = t / MST - (c + MST) / MST;
    return frame_at(S.seg, S.frame, (k & 1) * S.S5 + j);
}
// u(t) during the replay of the segment containing t
__host__ __device__ inline float *rep_buf(const ShotDesc &S, int t)
{
    int s = stored_slot(S, t);
    if (s >= 0) return frame_at(S.ckslots, S.frame, s);
    if (t % MST == 0) return seg_buf(S, t);
    return frame_at(S.rscr, S.frame, t % 3);
}
// adjoint field A(t): p1 of adjoint step t (with the injection of step t applied)
__host__ __device__ inline float *adj_buf(const ShotDesc &S, int t) { return frame_at(S.ascr, S.frame, (t + 3) % 3); }
// forward field used by the imaging condition at adjoint step it (it % 5 == 0)
__host__ __device__ inline float *img_buf(const ShotDesc &S, int it)
{
    int s = stored_slot(S, it);
    if (s >= 0) return frame_at(S.ckslots, S.frame, s);
    return seg_buf(S, it);
}

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

// stencil of one cell: c[] holds p1[x][z-3..z+3] (index 0..6), xm/xp p1[x-k][z], p1[x+k][z]
struct Cell {
    float zm3, zm2, zm1, z0, zp1, zp2, zp3;
    float xm3, xm2, xm1, xp1, xp2, xp3;
};
__device__ __forceinline__ float stencil(const Cell &c, float c1, float c2, float ck, float irx, float irz,
                                         float ir, float p0, float invdx, float invdz, float invdxdx,
                                         float invdzdz)
{
    const float C1 = 0.77793115f, C2 = -0.17388691f, C3 = 0.02338713f;
    const float D0 = -2.8215452f, D1 = 1.57663238f, D2 = -0.18347238f, D3 = 0.01761260f;
    float dpdz = fm(fa(fa(fm(C1, fs_(c.zp1, c.zm1)), fm(C2, fs_(c.zp2, c.zm2))), fm(C3, fs_(c.zp3, c.zm3))), invdz);
    float dpdx = fm(fa(fa(fm(C1, fs_(c.xp1, c.xm1)), fm(C2, fs_(c.xp2, c.xm2))), fm(C3, fs_(c.xp3, c.xm3))), invdx);
    float dzz = fm(fa(fa(fa(fm(D0, c.z0), fm(D1, fa(c.zp1, c.zm1))), fm(D2, fa(c.zp2, c.zm2))), fm(D3, fa(c.zp3, c.zm3))),
                   invdzdz);
    float dxx = fm(fa(fa(fa(fm(D0, c.z0), fm(D1, fa(c.xp1, c.xm1))), fm(D2, fa(c.xp2, c.xm2))), fm(D3, fa(c.xp3, c.xm3))),
                   invdxdx);
    float lap = fa(fa(fm(irx, dpdx), fm(irz, dpdz)), fm(ir, fa(dxx, dzz)));
    return fa(fa(fm(c1, c.z0), fm(c2, p0)), fm(ck, lap));
}

// ------------------------------------------------------------------ k_step
// grid: x = strip of LX columns, y = 2*shot + sub-item; block = 32*W lanes (W warps along z)
// prog[shot*prog_stride + L] = {kindA, itA, kindB, itB}
template <int LX>
__global__ void __launch_bounds__(256) k_step(const ShotDesc *__restrict__ shots, const int4 *__restrict__ prog,
                                              int prog_stride, int L, int shot_base)
{
    const int s = shot_base + (blockIdx.y >> 1);
    const int4 pw = prog[(long long)s * prog_stride + L];
    const int kind = (blockIdx.y & 1) ? pw.z : pw.x;
    const int it = (blockIdx.y & 1) ? pw.w : pw.y;
    if (kind == K_NONE) return;
    const ShotDesc &S = shots[s];
    const int X0 = blockIdx.x * LX;
    if (X0 >= S.Nx) return;
    const int Nx = S.Nx, ld = S.ld, pml = S.pml;
    const int g = threadIdx.x;
    const bool gv = g < S.G;
    const int z0 = 4 * g;
    const int lane = threadIdx.x & 31;

    // buffers of this item
    const float *p1, *p0;
    float *out;
    const float *u = nullptr;
    if (kind == K_FWD0 || kind == K_FWD1) {
        const bool keep = kind == K_FWD1;
        p1 = fwd_buf(S, it, keep);
        p0 = fwd_buf(S, it - 1, keep);
        out = fwd_buf(S, it + 1, keep);
    } else if (kind == K_REP) {
        p1 = rep_buf(S, it);
        p0 = rep_buf(S, it - 1);
        out = rep_buf(S, it + 1);
    } else {
        p1 = adj_buf(S, it);
        p0 = adj_buf(S, it + 1);
        out = adj_buf(S, it - 1);
        if (it % MST == 0) u = img_buf(S, it);
    }
    const bool fwd = kind == K_FWD0 || kind == K_FWD1;
    const bool sample = fwd && (it % S.sr == 0);
    const bool inject = kind == K_ADJ && it >= 1;
    const bool hess = kind == K_FWD1 && S.hessian && (it % MST == 0);
    const bool image = u != nullptr;
    const int kk = it / S.sr;

    // source term of this step, applied by the lane that owns the source cell
    float srcf = 0.0f;
    double srcd = 0.0;
    if (fwd) srcd = S.srcd[it];
    if (kind == K_REP) srcf = S.srcf[it];

    const float invdx = S.invdx, invdz = S.invdz, invdxdx = S.invdxdx, invdzdz = S.invdzdz;
    const int xlo = 3, xhi = Nx - 4, zlo = S.izStart, zhi = S.Nz - 4;

    float4 q[7];
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        int x = X0 - 3 + k;
        q[k] = (gv && x >= 0 && x < Nx) ? ldg4(p1 + (long long)x * ld + z0) : zero4;
    }
    const int xend = min(X0 + LX, Nx);
    for (int x = X0; x < xend; ++x) {
        {
            int xn = x + 3;
            q[6] = (gv && xn < Nx) ? ldg4(p1 + (long long)xn * ld + z0) : zero4;
        }
        const long long col = (long long)x * ld;
        // z-halo of the centre column: 3 cells below from lane-1, 3 above from lane+1
        float l1 = __shfl_up_sync(0xffffffffu, q[3].w, 1);
        float l2 = __shfl_up_sync(0xffffffffu, q[3].z, 1);
        float l3 = __shfl_up_sync(0xffffffffu, q[3].y, 1);
        float r1 = __shfl_down_sync(0xffffffffu, q[3].x, 1);
        float r2 = __shfl_down_sync(0xffffffffu, q[3].y, 1);
        float r3 = __shfl_down_sync(0xffffffffu, q[3].z, 1);
        if (lane == 0 && gv && g > 0) {
            float4 h = ld4(p1 + col + z0 - 4);
            l1 = h.w; l2 = h.z; l3 = h.y;
        }
        if (lane == 31 && g + 1 < S.G) {
            float4 h = ld4(p1 + col + z0 + 4);
            r1 = h.x; r2 = h.y; r3 = h.z;
        }
        const bool xin = x >= xlo && x <= xhi;
        const bool any = gv && xin && z0 + 3 >= zlo && z0 <= zhi;
        float4 v = zero4;
        if (any) {
            const bool damp = !(x >= pml && x < Nx - pml && z0 >= pml && z0 + 3 < S.Nz - pml);
            float4 c1 = damp ? ldg4(S.c1 + col + z0) : make_float4(2.f, 2.f, 2.f, 2.f);
            float4 c2 = damp ? ldg4(S.c2 + col + z0) : make_float4(-1.f, -1.f, -1.f, -1.f);
            float4 ck = ldg4(S.ck + col + z0), irx = ldg4(S.irx + col + z0), irz = ldg4(S.irz + col + z0);
            float4 ir = ldg4(S.ir + col + z0);
            float4 pz = ldg4(p0 + col + z0);
            const float zz[10] = {l3, l2, l1, q[3].x, q[3].y, q[3].z, q[3].w, r1, r2, r3};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int z = z0 + j;
                if (z < zlo || z > zhi) continue;
                Cell c;
                c.zm3 = zz[j]; c.zm2 = zz[j + 1]; c.zm1 = zz[j + 2]; c.z0 = zz[j + 3];
                c.zp1 = zz[j + 4]; c.zp2 = zz[j + 5]; c.zp3 = zz[j + 6];
                c.xm3 = comp(q[0], j); c.xm2 = comp(q[1], j); c.xm1 = comp(q[2], j);
                c.xp1 = comp(q[4], j); c.xp2 = comp(q[5], j); c.xp3 = comp(q[6], j);
                setc(v, j, stencil(c, comp(c1, j), comp(c2, j), comp(ck, j), comp(irx, j), comp(irz, j), comp(ir, j),
                                   comp(pz, j), invdx, invdz, invdxdx, invdzdz));
            }
        }
        if (gv) {
            const bool src_here = x == S.isx && S.isz >= z0 && S.isz < z0 + 4;
            const int js = S.isz - z0;
            // forward: the source enters before the free surface, in double (propagation.c:558-564)
            if (fwd && src_here) setc(v, js, (float)__dadd_rn((double)comp(v, js), srcd));
            float4 mir = zero4;  // values mirrored above the free surface
            if (S.fs) {
                if (pml >= z0 && pml < z0 + 4) setc(v, pml - z0, -0.0f);
#pragma unroll
                for (int j = 0; j < 4; ++j) setc(mir, j, -comp(v, j));
            }
            // replay: free surface first, then the float source (propagation.c:656-662)
            if (kind == K_REP && src_here) setc(v, js, fa(comp(v, js), srcf));
            // receivers of this column
            if (sample || inject) {
                const int e0 = __ldg(S.colptr + x), e1 = __ldg(S.colptr + x + 1);
                for (int e = e0; e < e1; ++e) {
                    const int2 r = __ldg(S.rec + e);
                    if (r.x < z0 || r.x >= z0 + 4) continue;
                    const int j = r.x - z0;
                    if (sample) S.traces_t[(long long)kk * S.ntr + r.y] = comp(q[3], j);
                }
            }
            // pseudo-Hessian / imaging on the model interior, FP64 accumulation
            if ((hess || image) && x >= pml && x < pml + S.nxx && z0 + 3 >= pml && z0 < pml + S.nz) {
                float4 pz = ldg4(p0 + col + z0);
                float4 uu = image ? ldg4(u + col + z0) : zero4;
                double2 *acc = reinterpret_cast<double2 *>((image ? S.Gacc : S.H) + col + z0);
                double2 a0 = acc[0], a1 = acc[1];
                double a[4] = {a0.x, a0.y, a1.x, a1.y};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int z = z0 + j;
                    if (z < pml || z >= pml + S.nz) continue;
                    float t = fm(fa(fs_(comp(v, j), fm(2.0f, comp(q[3], j))), comp(pz, j)), S.invdtdt);
                    float w = image ? fm(t, comp(uu, j)) : fm(t, t);
                    a[j] = __dadd_rn(a[j], (double)w);
                }
                acc[0] = make_double2(a[0], a[1]);
                acc[1] = make_double2(a[2], a[3]);
            }
            // adjoint: the injection of step it-1 goes into this output (propagation.c:676-682)
            if (inject) {
                const int e0 = __ldg(S.colptr + x), e1 = __ldg(S.colptr + x + 1);
                const float *arow = S.adj_t + (long long)(it - 1) * S.ntr;
                for (int e = e0; e < e1; ++e) {
                    const int2 r = __ldg(S.rec + e);
                    if (r.x < z0 || r.x >= z0 + 4) continue;
                    const int j = r.x - z0;
                    float a = fm(fm(fm(fm(fm(__ldg(arow + r.y), __ldg(S.recK + e)), S.dt), S.dt), invdx), invdz);
                    setc(v, j, fs_(comp(v, j), a));
                }
            }
            // store: the owner writes rows >= pml (all rows without a free surface); the
            // rows above are written by the mirror of rows pml+1..2*pml
            float *o = out + col + z0;
            if (!S.fs || z0 >= pml) {
                *reinterpret_cast<float4 *>(o) = v;
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (z0 + j >= pml) o[j] = comp(v, j);
            }
            if (S.fs) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int z = z0 + j;
                    if (z > pml && z <= 2 * pml) out[col + 2 * pml - z] = comp(mir, j);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) q[k] = q[k + 1];
    }
}

}  // namespace fwi
