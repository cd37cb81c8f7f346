// fwi_step.cuh -- the fused time-step kernel.
//
// One block advances S shots that share a model window (one coefficient set) by
// one time step over a tile of 16 float4 z-groups (64 cells) by TX columns.  The
// block first stages in shared memory with cp.async, before one wait, everything
// it reads: for every shot the p1 tile with its halo (one group above and below,
// three columns left and right) and the p0 tile, and once for all S shots the six
// coefficient tiles (out-of-range parts are zero-filled by the copy itself).  Each
// thread then computes the float4 groups of its columns from shared memory.  Lanes map to 16 z-groups x 8 columns, so a short column
// leaves few lanes idle, and no state is carried from column to column.
//
// Fused per step, as the reference does around acoustic_iso2d_fd_it_6order
// (propagation.c:13-74): point source (:558 forward, double, before the free
// surface; :662 replay, float, after it), mirror free surface (:76-101), pseudo-
// Hessian (:579-594), imaging (:700-714) and the adjoint injection (:676-682),
// which goes into this step's output so the next step reads it as p1.  Receiver
// sampling (:567-576) is done by one extra block per shot group.
//
// MATH 0 evaluates every product and sum with __fmul_rn/__fadd_rn/__fsub_rn in the
// reference's order (bit-identical to its strict IEEE build); MATH 1 lets the
// compiler contract multiply-adds (within the stated FP32 tolerance, not bitwise).
#pragma once
#include "fwi_kernels.cuh"

namespace fwi {

constexpr int TG = 16;             // z-groups per tile (64 cells)
constexpr int TYX = 8;             // thread columns per block
constexpr int STEP_THREADS = TG * TYX;

template <int MATH>
__device__ __forceinline__ float cell(float zm3, float zm2, float zm1, float z0, float zp1, float zp2, float zp3,
                                      float xm3, float xm2, float xm1, float xp1, float xp2, float xp3, float c1,
                                      float c2, float ck, float irx, float irz, float ir, float p0, float invdx,
                                      float invdz, float invdxdx, float invdzdz)
{
    const float C1 = 0.77793115f, C2 = -0.17388691f, C3 = 0.02338713f;
    const float D0 = -2.8215452f, D1 = 1.57663238f, D2 = -0.18347238f, D3 = 0.01761260f;
    if (MATH == 0) {
        float dpdz = fm(fa(fa(fm(C1, fs_(zp1, zm1)), fm(C2, fs_(zp2, zm2))), fm(C3, fs_(zp3, zm3))), invdz);
        float dpdx = fm(fa(fa(fm(C1, fs_(xp1, xm1)), fm(C2, fs_(xp2, xm2))), fm(C3, fs_(xp3, xm3))), invdx);
        float dzz = fm(fa(fa(fa(fm(D0, z0), fm(D1, fa(zp1, zm1))), fm(D2, fa(zp2, zm2))), fm(D3, fa(zp3, zm3))), invdzdz);
        float dxx = fm(fa(fa(fa(fm(D0, z0), fm(D1, fa(xp1, xm1))), fm(D2, fa(xp2, xm2))), fm(D3, fa(xp3, xm3))), invdxdx);
        float lap = fa(fa(fm(irx, dpdx), fm(irz, dpdz)), fm(ir, fa(dxx, dzz)));
        return fa(fa(fm(c1, z0), fm(c2, p0)), fm(ck, lap));
    } else {
        float dpdz = (C1 * (zp1 - zm1) + C2 * (zp2 - zm2) + C3 * (zp3 - zm3)) * invdz;
        float dpdx = (C1 * (xp1 - xm1) + C2 * (xp2 - xm2) + C3 * (xp3 - xm3)) * invdx;
        float dzz = (D0 * z0 + D1 * (zp1 + zm1) + D2 * (zp2 + zm2) + D3 * (zp3 + zm3)) * invdzdz;
        float dxx = (D0 * z0 + D1 * (xp1 + xm1) + D2 * (xp2 + xm2) + D3 * (xp3 + xm3)) * invdxdx;
        return c1 * z0 + c2 * p0 + ck * (irx * dpdx + irz * dpdz + ir * (dxx + dzz));
    }
}

// four cells of a z-group; zz[0..9] = p1[x][z0-3 .. z0+6]; a..h: columns x-3..x-1, x+1..x+3
template <int MATH>
__device__ __forceinline__ float4 group(const float (&zz)[10], const float4 &a, const float4 &b, const float4 &c,
                                        const float4 &e, const float4 &f, const float4 &h, const float4 &c1,
                                        const float4 &c2, const float4 &ck, const float4 &irx, const float4 &irz,
                                        const float4 &ir, const float4 &p0, float invdx, float invdz, float invdxdx,
                                        float invdzdz)
{
    float4 v;
    v.x = cell<MATH>(zz[0], zz[1], zz[2], zz[3], zz[4], zz[5], zz[6], a.x, b.x, c.x, e.x, f.x, h.x, c1.x, c2.x, ck.x,
                     irx.x, irz.x, ir.x, p0.x, invdx, invdz, invdxdx, invdzdz);
    v.y = cell<MATH>(zz[1], zz[2], zz[3], zz[4], zz[5], zz[6], zz[7], a.y, b.y, c.y, e.y, f.y, h.y, c1.y, c2.y, ck.y,
                     irx.y, irz.y, ir.y, p0.y, invdx, invdz, invdxdx, invdzdz);
    v.z = cell<MATH>(zz[2], zz[3], zz[4], zz[5], zz[6], zz[7], zz[8], a.z, b.z, c.z, e.z, f.z, h.z, c1.z, c2.z, ck.z,
                     irx.z, irz.z, ir.z, p0.z, invdx, invdz, invdxdx, invdzdz);
    v.w = cell<MATH>(zz[3], zz[4], zz[5], zz[6], zz[7], zz[8], zz[9], a.w, b.w, c.w, e.w, f.w, h.w, c1.w, c2.w, ck.w,
                     irx.w, irz.w, ir.w, p0.w, invdx, invdz, invdxdx, invdzdz);
    return v;
}

// 16-byte global -> shared copy that zero-fills when src_bytes == 0 (cp.async, no register staging)
__device__ __forceinline__ void cp16(void *smem, const void *gmem, int src_bytes)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_commit_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <int S>
struct Bufs {
    const float *p1[S], *p0[S], *u[S];
    float *out[S];
    int isx[S], isz[S];  // padded source cell
    double srcd[S];      // this step's forward source term (double, propagation.c:558)
    float srcf[S];       // this step's replay source term (float, :662)
};

// grid: x = column tile of TX columns (one extra x index: the receiver-sampling block),
//       y = 2 * group-of-S + sub-item, z = tile of TG z-groups.  block = TG x TYX threads.
// Everything the block reads (p1 tile with halo, p0 and the six coefficient fields of
// its cells) is staged in shared memory by cp.async before a single wait.
template <int TX, int S, int MATH>
__global__ void __launch_bounds__(STEP_THREADS) k_step(const ShotDesc *__restrict__ shots, const int4 *__restrict__ prog,
                                                       int L, int shot_base, int nshot)
{
    constexpr int TCOL = TX + 6, TROW = TG + 2;  // p1 tile: columns x-3..x+TX+2, groups g-1..g+TG
    __shared__ float4 sp1[S][TCOL][TROW];
    __shared__ float4 sp0[S][TX][TG];
    __shared__ float4 scf[6][TX][TG];  // c1, c2, coef3*K, d(1/rho)/dx, d(1/rho)/dz, 1/rho
    __shared__ Bufs<S> B;
    const int4 pw = prog[L];
    const int kind = (blockIdx.y & 1) ? pw.z : pw.x;
    const int it = (blockIdx.y & 1) ? pw.w : pw.y;
    if (kind == K_NONE) return;
    const int s0 = shot_base + (blockIdx.y >> 1) * S;
    const int nsh = min(S, shot_base + nshot - s0);  // shots of this block (the last group may be short)
    const ShotDesc &A = shots[s0];                   // geometry and coefficients of the group
    const int Nx = A.Nx, ld = A.ld, pml = A.pml, G = A.G, Nz = A.Nz;
    const int nxt = (Nx + TX - 1) / TX;
    const bool fwd = kind == K_FWD0 || kind == K_FWD1;
    const int tid = threadIdx.y * TG + threadIdx.x;

    // ---- the receiver-sampling block: p1 is read-only during this launch
    if ((int)blockIdx.x >= nxt) {
        if (!fwd || it % A.sr != 0 || (int)blockIdx.x > nxt || blockIdx.z != 0) return;
        for (int s = 0; s < nsh; ++s) {
            const ShotDesc &D = shots[s0 + s];
            const float *p1 = fwd_buf(D, it, kind == K_FWD1);
            float *tr = D.traces_t + (long long)(it / D.sr) * D.ntr;
            for (int r = tid; r < D.ntr; r += STEP_THREADS) tr[r] = p1[D.rec_off[r]];
        }
        return;
    }

    // ---- one thread resolves which frames this step reads and writes (divisions by d, 3, 5)
    if (tid < S) {
        const int s = tid;
        const ShotDesc &D = shots[s0 + (s < nsh ? s : 0)];
        B.u[s] = nullptr;
        if (fwd) {
            const bool keep = kind == K_FWD1;
            B.p1[s] = fwd_buf(D, it, keep);
            B.p0[s] = fwd_buf(D, it - 1, keep);
            B.out[s] = fwd_buf(D, it + 1, keep);
        } else if (kind == K_REP) {
            B.p1[s] = rep_buf(D, it);
            B.p0[s] = rep_buf(D, it - 1);
            B.out[s] = rep_buf(D, it + 1);
        } else {
            B.p1[s] = adj_buf(D, it);
            B.p0[s] = adj_buf(D, it + 1);
            B.out[s] = adj_buf(D, it - 1);
            if (it % MST == 0) B.u[s] = img_buf(D, it);
        }
        B.isx[s] = s < nsh ? D.isx : -1;
        B.isz[s] = D.isz;
        B.srcd[s] = fwd ? D.srcd[it] : 0.0;
        B.srcf[s] = kind == K_REP ? D.srcf[it] : 0.0f;
    }
    __syncthreads();

    // ---- stage p1 tiles, p0 and the coefficients of this tile
    const int X0 = blockIdx.x * TX, G0 = blockIdx.z * TG;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const float *p1 = B.p1[s];
        for (int r = tid; r < TCOL * TROW; r += STEP_THREADS) {
            const int cx = r / TROW, cg = r % TROW;
            const int x = X0 - 3 + cx, gg = G0 - 1 + cg;
            const bool in = s < nsh && x >= 0 && x < Nx && gg >= 0 && gg < G;
            cp16(&sp1[s][cx][cg], p1 + (in ? (long long)x * ld + 4 * gg : 0), in ? 16 : 0);
        }
    }
    {
        const float *cf[6] = {A.c1, A.c2, A.ck, A.irx, A.irz, A.ir};
        for (int r = tid; r < TX * TG; r += STEP_THREADS) {
            const int cx = r / TG, cg = r % TG;
            const int x = X0 + cx, gg = G0 + cg;
            const bool in = x < Nx && gg < G;
            const long long off = in ? (long long)x * ld + 4 * gg : 0;
#pragma unroll
            for (int f = 0; f < 6; ++f) cp16(&scf[f][cx][cg], cf[f] + off, in ? 16 : 0);
#pragma unroll
            for (int s = 0; s < S; ++s) cp16(&sp0[s][cx][cg], B.p0[s] + off, (in && s < nsh) ? 16 : 0);
        }
    }
    cp_commit_wait_all();
    __syncthreads();

    const bool inject = kind == K_ADJ && it >= 1;
    const bool hess = kind == K_FWD1 && A.hessian && (it % MST == 0);
    const bool image = kind == K_ADJ && (it % MST == 0);
    const bool accum = hess || image;

    // per-lane constants
    const int g = G0 + threadIdx.x;
    const bool gv = g < G;
    const int z0 = 4 * g;
    const int zlo = A.izStart, zhi = Nz - 4;
    const bool zfd = gv && z0 + 3 >= zlo && z0 <= zhi;
    const bool zpart = z0 < zlo || z0 + 3 > zhi;  // group straddles the edge of the updated rows
    const bool zint = gv && z0 + 3 >= pml && z0 < pml + A.nz;
    const bool fs_top = A.fs && gv && z0 <= 2 * pml;  // the free-surface row or the rows it mirrors
    const int jpml = (pml >= z0 && pml < z0 + 4) ? pml - z0 : -1;
    const float invdx = A.invdx, invdz = A.invdz, invdxdx = A.invdxdx, invdzdz = A.invdzdz, invdtdt = A.invdtdt;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!gv) return;  // no barrier follows
    const int cg = threadIdx.x + 1;

#pragma unroll 1
    for (int k = threadIdx.y; k < TX; k += TYX) {
        const int x = X0 + k;
        if (x >= Nx) break;
        const int cx = k + 3;  // p1 tile column of x
        const long long colx = (long long)x * ld;
        const long long col = colx + z0;
        const bool any = zfd && x >= 3 && x <= Nx - 4;
        const bool acc_here = accum && zint && x >= pml && x < pml + A.nxx;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (s >= nsh) break;
            const float4 cq = sp1[s][cx][cg];
            const float4 p0 = sp0[s][k][threadIdx.x];
            float4 v = zero4;
            if (any) {
                const float4 lo = sp1[s][cx][cg - 1], hi = sp1[s][cx][cg + 1];
                const float zz[10] = {lo.y, lo.z, lo.w, cq.x, cq.y, cq.z, cq.w, hi.x, hi.y, hi.z};
                v = group<MATH>(zz, sp1[s][cx - 3][cg], sp1[s][cx - 2][cg], sp1[s][cx - 1][cg], sp1[s][cx + 1][cg],
                                sp1[s][cx + 2][cg], sp1[s][cx + 3][cg], scf[0][k][threadIdx.x], scf[1][k][threadIdx.x],
                                scf[2][k][threadIdx.x], scf[3][k][threadIdx.x], scf[4][k][threadIdx.x],
                                scf[5][k][threadIdx.x], p0, invdx, invdz, invdxdx, invdzdz);
                if (zpart) {
                    if (z0 < zlo || z0 > zhi) v.x = 0.f;
                    if (z0 + 1 < zlo || z0 + 1 > zhi) v.y = 0.f;
                    if (z0 + 2 < zlo || z0 + 2 > zhi) v.z = 0.f;
                    if (z0 + 3 < zlo || z0 + 3 > zhi) v.w = 0.f;
                }
            }
            const bool src_here = x == B.isx[s] && B.isz[s] >= z0 && B.isz[s] < z0 + 4;
            // forward: the source enters before the free surface, in double (propagation.c:558-564)
            if (fwd && src_here) setc(v, B.isz[s] - z0, (float)__dadd_rn((double)comp(v, B.isz[s] - z0), B.srcd[s]));
            float4 mir = zero4;
            if (fs_top) {
                if (jpml >= 0) setc(v, jpml, -0.0f);
                mir = make_float4(-v.x, -v.y, -v.z, -v.w);
            }
            // replay: free surface first, then the float source (propagation.c:656-662)
            if (kind == K_REP && src_here) setc(v, B.isz[s] - z0, fa(comp(v, B.isz[s] - z0), B.srcf[s]));
            if (acc_here) {
                const ShotDesc &D = shots[s0 + s];
                const float4 uu = image ? ldg4(B.u[s] + col) : zero4;
                double2 *acc = reinterpret_cast<double2 *>((image ? D.Gacc : D.H) + col);
                double2 a0 = acc[0], a1 = acc[1];
                double a[4] = {a0.x, a0.y, a1.x, a1.y};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int z = z0 + j;
                    if (z < pml || z >= pml + D.nz) continue;
                    float t = fm(fa(fs_(comp(v, j), fm(2.0f, comp(cq, j))), comp(p0, j)), invdtdt);
                    float w = image ? fm(t, comp(uu, j)) : fm(t, t);
                    a[j] = __dadd_rn(a[j], (double)w);
                }
                acc[0] = make_double2(a[0], a[1]);
                acc[1] = make_double2(a[2], a[3]);
            }
            if (inject) {
                const ShotDesc &D = shots[s0 + s];
                const int e0 = __ldg(D.colptr + x), e1 = __ldg(D.colptr + x + 1);
                const float *arow = D.adj_t + (long long)(it - 1) * D.ntr;
                for (int e = e0; e < e1; ++e) {
                    const int2 r = __ldg(D.rec + e);
                    if (r.x < z0 || r.x >= z0 + 4) continue;
                    const int j = r.x - z0;
                    float a = fm(fm(fm(fm(fm(__ldg(arow + r.y), __ldg(D.recK + e)), D.dt), D.dt), invdx), invdz);
                    setc(v, j, fs_(comp(v, j), a));
                }
            }
            float *o = B.out[s] + col;
            if (!fs_top || z0 >= pml) {
                *reinterpret_cast<float4 *>(o) = v;
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (z0 + j >= pml) o[j] = comp(v, j);
            }
            if (fs_top) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int z = z0 + j;
                    if (z > pml && z <= 2 * pml) B.out[s][colx + 2 * pml - z] = comp(mir, j);
                }
            }
        }
    }
}

}  // namespace fwi
