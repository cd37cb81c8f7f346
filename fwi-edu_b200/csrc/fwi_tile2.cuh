// fwi_tile2.cuh -- two time steps per launch (temporal blocking with a halo of depth two).
//
// The one-step kernel (fwi_tile.cuh) moves 12 bytes of fields per cell-update through HBM: p1
// and p0 in, p2 out.  This kernel advances a shot by two steps per launch: a block loads u(t)
// with a halo of two stencil radii (6 cells) and u(t-1) with a halo of one, computes u(t+1) on
// its tile grown by one stencil radius (3 cells) into shared memory, then u(t+2) on its tile
// from there, and writes u(t+1) and u(t+2) of its tile.  Per two cell-updates that is 8 bytes in
// and 8 out (8 bytes per cell-update instead of 12), half the launches, and 1.27 times the
// stencil arithmetic (the grown region of the first step is recomputed by the neighbours).
//
// Everything the one-step kernel fuses around the stencil is applied to each of the two steps
// in the reference's order, bit for bit: forward source (double, before the free surface),
// mirror free surface, replay source (float, after it), pseudo-Hessian and imaging on the tile
// (every 5th step), adjoint injection (on the grown region too, since the second step reads it)
// and receiver sampling of u(t) and u(t+1) on the tile.  The free-surface mirror rows of u(t+1)
// that the second step reads come from the threads that own the mirrored rows, written into the
// shared copy before a barrier of the consumer warps.
//
// A program item of depth two (kind | K_DEPTH2) names the first of its two steps; items of depth
// one (an odd number of steps, a segment's last replay step) run the first step only.  Fields
// that are not kept rotate through four frames (NROT), so the two outputs of a launch never land
// in a frame that another block of the same launch still reads.
#pragma once
#include "fwi_tile.cuh"

namespace fwi {

constexpr int K_DEPTH2 = 0x100;  // program-item flag: the item advances two steps

template <int TX>
struct Tile2Geom {
    static constexpr int AG = TG + 4;   // u(t) box: groups G0-2 .. G0+TG+1
    static constexpr int AX = TX + 12;  // u(t) box: columns X0-6 .. X0+TX+5
    static constexpr int CG = TG + 2;   // grown region: groups G0-1 .. G0+TG
    static constexpr int CX = TX + 6;   // grown region: columns X0-3 .. X0+TX+2
    static constexpr int A_BYTES = AG * AX * 16;
    static constexpr int B_BYTES = CG * CX * 16;  // u(t-1) box: the grown region
    static constexpr int CF_BYTES = 6 * CG * CX * 16;
    static constexpr int C_BYTES = CG * CX * 16;  // u(t+1) on the grown region
    static constexpr int B_OFF = round128(A_BYTES);
    static constexpr int STAGE = B_OFF + round128(B_BYTES);
    static constexpr int C_OFF = round128(CF_BYTES);  // two u(t+1) buffers (shot parity)
    static constexpr int ST_OFF = C_OFF + 2 * round128(C_BYTES);
    static constexpr int smem(int nst) { return ST_OFF + nst * STAGE; }
    static constexpr int TASKS1 = CG * CX;  // groups of the first step
};

// named barrier of the consumer warps only (the producer warp does not take part)
__device__ __forceinline__ void consumers_sync(int nthreads)
{
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}
__device__ __forceinline__ void sts4(unsigned a, const float4 &v)
{
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}
__device__ __forceinline__ void sts1(unsigned a, float v) { asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory"); }

// grid: x = column tile, y = 2 * shot chunk + program item half, z = tile of TG z-groups.
// block = (TG, TX + 32 / TG) threads: rows 0..TX-1 are the consumers, the last row the producer.
// Tensor maps: tm_a {ld, Nx, nfr, nshot} box {4 AG, AX, 1, 1}; tm_b the same with box
// {4 CG, CX, 1, 1}; tm_cf {ld, Nx, 6} box {4 CG, CX, 6}.  Dynamic shared memory Tile2Geom::smem(NST).
template <int TX, int NST, int MATH>
__global__ void __launch_bounds__(TG * TX + 32, 2)
    k_tile2(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
            const __grid_constant__ CUtensorMap tm_cf, const ShotDesc *__restrict__ shots,
            const int4 *__restrict__ prog, int L, int shot_base, int nshot, int chunk, int *err)
{
    using Geo = Tile2Geom<TX>;
    constexpr int NC = TG * TX;  // consumer threads
    constexpr int NW = NC / 32;  // consumer warps
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long full[NST], empty[NST], cfbar;
    __shared__ float *s_out[2][TILE_CH_MAX];
    __shared__ const float *s_u[2][TILE_CH_MAX];
    __shared__ float *s_tr[2][TILE_CH_MAX];  // trace row of u(t) / u(t+1), or null
    __shared__ double s_srcd[2][TILE_CH_MAX];
    __shared__ float s_srcf[2][TILE_CH_MAX];
    __shared__ int s_isx[TILE_CH_MAX], s_isz[TILE_CH_MAX], s_rz0[TILE_CH_MAX], s_rz1[TILE_CH_MAX];
    __shared__ int s_fi[2];

    grid_dep_launch();
    const int4 pw = prog[L];
    const int kw = (blockIdx.y & 1) ? pw.z : pw.x;
    const int it = (blockIdx.y & 1) ? pw.w : pw.y;
    const int kind = kw & 0xff;
    const bool two = (kw & K_DEPTH2) != 0;
    if (kind == K_NONE) return;
    const int cb = shot_base + (blockIdx.y >> 1) * chunk;
    const int n = min(chunk, shot_base + nshot - cb);
    if (n <= 0) return;
    const ShotDesc &A = shots[cb];
    const int Nx = A.Nx, pml = A.pml, G = A.G, Nz = A.Nz;
    const bool fwd = kind == K_FWD0 || kind == K_FWD1;
    const int it2 = kind == K_ADJ ? it - 1 : it + 1;  // the second step
    const int tid = threadIdx.y * TG + threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int X0 = blockIdx.x * TX, G0 = blockIdx.z * TG;
    unsigned char *st_base = smem + Geo::ST_OFF;
    const unsigned sm0 = smem_u32(smem);
    int issued = 0;

    if (warp == NW) {
        if (lane == 0) {
            for (int j = 0; j < NST; ++j) {
                mbar_init(smem_u32(&full[j]), 1);
                mbar_init(smem_u32(&empty[j]), NW);
            }
            mbar_init(smem_u32(&cfbar), 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            int i1, i0, io;
            step_frames(A, kind, it, i1, i0, io);
            s_fi[0] = i1;
            s_fi[1] = i0;
            grid_dep_wait();
            mbar_arrive_expect(smem_u32(&cfbar), Geo::CF_BYTES);
            tma_load3(sm0, &tm_cf, 4 * (G0 - 1), X0 - 3, 0, smem_u32(&cfbar));
            for (; issued < min(n, NST); ++issued) {
                const unsigned b = smem_u32(&full[issued]);
                mbar_arrive_expect(b, Geo::A_BYTES + Geo::B_BYTES);
                unsigned char *stg = st_base + issued * Geo::STAGE;
                tma_load4(smem_u32(stg), &tm_a, 4 * (G0 - 2), X0 - 6, i1, cb + issued - shot_base, b);
                tma_load4(smem_u32(stg + Geo::B_OFF), &tm_b, 4 * (G0 - 1), X0 - 3, i0, cb + issued - shot_base, b);
            }
        }
    } else if (tid < n) {
        const ShotDesc &D = shots[cb + tid];
        s_tr[1][tid] = nullptr;
        for (int s = 0; s < (two ? 2 : 1); ++s) {  // the second step's scalars only where it exists
            const int t = s ? it2 : it;
            int i1, i0, io, iu = -1;
            step_frames(D, kind, t, i1, i0, io);
            if (kind == K_ADJ && t % MST == 0) iu = img_idx(D, t);
            s_out[s][tid] = frame_ptr(D, io);
            s_u[s][tid] = iu >= 0 ? frame_ptr(D, iu) : nullptr;
            // receivers sample the field before the step: u(it) and, with two steps, u(it + 1)
            const int ts = it + s;
            s_tr[s][tid] = (fwd && (s == 0 || two) && ts % D.sr == 0) ? D.traces_t + (long long)(ts / D.sr) * D.ntr
                                                                         : nullptr;
            s_srcd[s][tid] = fwd ? D.srcd[t] : 0.0;
            s_srcf[s][tid] = kind == K_REP ? D.srcf[t] : 0.0f;
        }
        s_isx[tid] = D.isx;
        s_isz[tid] = D.isz;
        s_rz0[tid] = D.rz0;
        s_rz1[tid] = D.rz1;
    }
    __syncthreads();
    grid_dep_wait();

    if (warp == NW) {
        if (lane != 0) return;
        const int i1 = s_fi[0], i0 = s_fi[1];
        for (int j = issued; j < n; ++j) {
            const int st = j % NST;
            if (j >= NST && !mbar_wait(smem_u32(&empty[st]), (j / NST - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            const int sg = cb + j - shot_base;
            const unsigned b = smem_u32(&full[st]);
            mbar_arrive_expect(b, Geo::A_BYTES + Geo::B_BYTES);
            unsigned char *stg = st_base + st * Geo::STAGE;
            tma_load4(smem_u32(stg), &tm_a, 4 * (G0 - 2), X0 - 6, i1, sg, b);
            tma_load4(smem_u32(stg + Geo::B_OFF), &tm_b, 4 * (G0 - 1), X0 - 3, i0, sg, b);
            issued = j + 1;
        }
        mbar_wait(smem_u32(&cfbar), 0);
        for (int j = max(0, issued - NST); j < issued; ++j) mbar_wait(smem_u32(&full[j % NST]), (j / NST) & 1);
        return;
    }

    // ---- consumers
    const int zlo = A.izStart, zhi = Nz - 4;
    const int fs_hi = min(2 * pml, pml + 3);  // last mirrored source row (snapshot steps use the one-step kernel)
    const float invdx = A.invdx, invdz = A.invdz, invdtdt = A.invdtdt;
    const PkConst K = make_pkconst(invdx, invdz, A.invdxdx, A.invdzdz, A.negzero);
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    // shared-memory addresses: coefficient plane f, grown-region column c, group g
    auto cf_at = [&](int f, int c, int g) { return sm0 + (unsigned)(((f * Geo::CX + c) * Geo::CG + g) * 16); };

    // a consumer warp gave up waiting: all of them stop together.  The flag of shot i is read
    // after the barrier of shot i, and written before it; two flags by shot parity, so that a warp
    // already writing shot i + 1's never meets one still reading shot i's
    __shared__ int s_fail[2];
    if (tid < 2) s_fail[tid] = 0;
    consumers_sync(NC);
    {
        const bool ok = mbar_wait(smem_u32(&cfbar), 0);
        if (!__all_sync(0xffffffffu, ok) && lane == 0) {
            atomicExch(err, 1);
            s_fail[0] = 1;  // read by shot 0
        }
    }

    // One group (4 rows of column x, rows z0..z0+3) of step s of shot i: the stencil value v (zero
    // outside the updated range) from its z-window lo/cq/hi, its x-neighbours xn, coefficients and
    // p0, then the epilogue in the reference's order.  inner: the group belongs to the block's
    // tile (global writes, accumulators, receivers); cbuf: shared-memory address of u(t+1) at
    // this group (step 0 only), or 0.
    auto epilogue = [&](int i, int s, int x, int z0, float4 v, const float4 &cq, const float4 &p0, bool inner,
                        unsigned cbuf, unsigned cmir_col) {
        const int t = s ? it2 : it;
        const bool inject = kind == K_ADJ && t >= 1;
        const bool hess = kind == K_FWD1 && A.hessian && (t % MST == 0);
        const bool image = kind == K_ADJ && (t % MST == 0);
        const bool fs_top = A.fs && z0 <= fs_hi;
        const int jpml = (pml >= z0 && pml < z0 + 4) ? pml - z0 : -1;
        const int isx = s_isx[i], isz = s_isz[i];
        const bool src_here = x == isx && isz >= z0 && isz < z0 + 4;
        if (fwd && src_here) setc(v, isz - z0, (float)__dadd_rn((double)comp(v, isz - z0), s_srcd[s][i]));
        float4 mir = zero4;
        if (fs_top) {
            if (jpml >= 0) setc(v, jpml, -0.0f);
            mir = make_float4(-v.x, -v.y, -v.z, -v.w);
        }
        if (kind == K_REP && src_here) setc(v, isz - z0, fa(comp(v, isz - z0), s_srcf[s][i]));
        const long long colx = (long long)x * A.ld, col = colx + z0;
        if (inner && (hess || image) && x >= pml && x < pml + A.nxx && z0 + 3 >= pml && z0 < pml + A.nz) {
            const ShotDesc &D = shots[cb + i];
            const float4 uu = image ? ldg4(s_u[s][i] + col) : zero4;
            double2 *acc = reinterpret_cast<double2 *>((image ? D.Gacc : D.H) + col);
            double2 a0 = acc[0], a1 = acc[1];
            double a[4] = {a0.x, a0.y, a1.x, a1.y};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int z = z0 + j;
                if (z < pml || z >= pml + D.nz) continue;
                float tt = fm(fa(fs_(comp(v, j), fm(2.0f, comp(cq, j))), comp(p0, j)), invdtdt);
                float w = image ? fm(tt, comp(uu, j)) : fm(tt, tt);
                a[j] = __dadd_rn(a[j], (double)w);
            }
            acc[0] = make_double2(a[0], a[1]);
            acc[1] = make_double2(a[2], a[3]);
        }
        if (inject && x >= 0 && x < Nx && z0 + 3 >= s_rz0[i] && z0 <= s_rz1[i]) {
            const ShotDesc &D = shots[cb + i];
            const int e0 = __ldg(D.colptr + x), e1 = __ldg(D.colptr + x + 1);
            const float *arow = D.adj_t + (long long)(t - 1) * D.ntr;
            for (int e = e0; e < e1; ++e) {
                const int2 r = __ldg(D.rec + e);
                if (r.x < z0 || r.x >= z0 + 4) continue;
                const int j = r.x - z0;
                float a = fm(fm(fm(fm(fm(__ldg(arow + r.y), __ldg(D.recK + e)), D.dt), D.dt), invdx), invdz);
                setc(v, j, fs_(comp(v, j), a));
            }
        }
        // the field as stored: into the shared copy (step 0) and, for the tile, into its frame
        const bool partial = fs_top && z0 < pml;
        if (cbuf) {
            if (!partial) sts4(cbuf, v);
            else
                for (int j = 0; j < 4; ++j)
                    if (z0 + j >= pml) sts1(cbuf + 4u * j, comp(v, j));
        }
        if (inner) {
            float *out = s_out[s][i];
            if (!partial) *reinterpret_cast<float4 *>(out + col) = v;
            else
                for (int j = 0; j < 4; ++j)
                    if (z0 + j >= pml) out[col + j] = comp(v, j);
        }
        if (fs_top) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int z = z0 + j;
                if (z > pml && z <= fs_hi) {
                    const int zm = 2 * pml - z;
                    if (inner) s_out[s][i][colx + zm] = comp(mir, j);
                    // the mirrored row inside the grown region's shared copy (cmir_col: the copy's
                    // column base, rows counted from 4 (G0 - 1))
                    const int r = zm - 4 * (G0 - 1);
                    if (cmir_col && r >= 0 && r < 4 * Geo::CG) sts1(cmir_col + 4u * r, comp(mir, j));
                }
            }
        }
        // receivers sample the stored field before the step: u(t) at the first step's p1 (cq), and
        // u(t + 1), the first step's output
        if (inner && z0 + 3 >= s_rz0[i] && z0 <= s_rz1[i]) {
            const ShotDesc &D = shots[cb + i];
            float *tr0 = s_tr[0][i], *tr1 = s_tr[1][i];
            if (s == 0 && (tr0 || tr1)) {
                const int e0 = __ldg(D.colptr + x), e1 = __ldg(D.colptr + x + 1);
                for (int e = e0; e < e1; ++e) {
                    const int2 r = __ldg(D.rec + e);
                    if (r.x < z0 || r.x >= z0 + 4) continue;
                    if (tr0) tr0[r.y] = comp(cq, r.x - z0);
                    if (tr1) tr1[r.y] = comp(v, r.x - z0);
                }
            }
        }
    };

    for (int i = 0; i < n; ++i) {
        const int st = i % NST;
        // the consumer warps give up together (they meet at a barrier below): every warp's wait is
        // bounded, then a shared flag decides for all of them
        const bool ok = mbar_wait(smem_u32(&full[st]), (i / NST) & 1);
        if (!__all_sync(0xffffffffu, ok) && lane == 0) {
            atomicExch(err, 1);
            s_fail[i & 1] = 1;
        }
        consumers_sync(NC);
        if (s_fail[i & 1]) break;
        const unsigned sa = smem_u32(st_base) + (unsigned)(st * Geo::STAGE), sb = sa + Geo::B_OFF;
        const unsigned cb_base = sm0 + Geo::C_OFF + (unsigned)((i & 1) * round128(Geo::C_BYTES));
        // ---- step 1 on the grown region: task q -> column c (0..CX-1), group g (0..CG-1)
        for (int q = tid; q < Geo::TASKS1; q += NC) {
            const int c = q / Geo::CG, g = q - c * Geo::CG;
            const int x = X0 - 3 + c, gg = G0 - 1 + g, z0 = 4 * gg;
            const bool inner = c >= 3 && c < 3 + TX && g >= 1 && g <= TG && x < Nx && gg < G;
            if (!two && !inner) continue;        // one step: the grown region is not needed
            if (A.fs && z0 + 3 < pml) continue;  // above the surface: mirrored rows come from the owners
            const unsigned ca = sa + (unsigned)(((c + 3) * Geo::AG + g + 1) * 16);  // u(t) at this group
            const float4 lo = lds4(ca - 16), cq = lds4(ca), hi = lds4(ca + 16);
            const float4 p0 = lds4(sb + (unsigned)((c * Geo::CG + g) * 16));
            float4 v = zero4;
            const bool xint = x >= 3 && x <= Nx - 4;
            const bool zfd = z0 + 3 >= zlo && z0 <= zhi;
            if (zfd && xint) {
                const unsigned cs = Geo::AG * 16u;
                const float4 xn[6] = {lds4(ca - 3 * cs), lds4(ca - 2 * cs), lds4(ca - cs),
                                      lds4(ca + cs), lds4(ca + 2 * cs), lds4(ca + 3 * cs)};
                const float4 cf[6] = {lds4(cf_at(0, c, g)), lds4(cf_at(1, c, g)), lds4(cf_at(2, c, g)),
                                      lds4(cf_at(3, c, g)), lds4(cf_at(4, c, g)), lds4(cf_at(5, c, g))};
                v = group2<MATH>(lo, cq, hi, xn, cf, p0, K);
                if (z0 < zlo || z0 + 3 > zhi) {
                    if (z0 < zlo || z0 > zhi) v.x = 0.f;
                    if (z0 + 1 < zlo || z0 + 1 > zhi) v.y = 0.f;
                    if (z0 + 2 < zlo || z0 + 2 > zhi) v.z = 0.f;
                    if (z0 + 3 < zlo || z0 + 3 > zhi) v.w = 0.f;
                }
            }
            const unsigned ccol = cb_base + (unsigned)(c * Geo::CG * 16);
            epilogue(i, 0, x, z0, v, cq, p0, inner, two ? ccol + (unsigned)(g * 16) : 0u, two ? ccol : 0u);
        }
        if (two) {
            consumers_sync(NC);  // u(t+1) of the grown region, mirror rows included, is complete
            // ---- step 2 on the tile: column k, group zl
            const int zl = threadIdx.x, k = threadIdx.y;
            const int x = X0 + k, gg = G0 + zl, z0 = 4 * gg;
            if (x < Nx && gg < G && !(A.fs && z0 + 3 < pml)) {
                const int c = k + 3, g = zl + 1;
                const unsigned ca = cb_base + (unsigned)((c * Geo::CG + g) * 16);
                const float4 lo = lds4(ca - 16), cq = lds4(ca), hi = lds4(ca + 16);
                const float4 p0 = lds4(sa + (unsigned)(((k + 6) * Geo::AG + zl + 2) * 16));  // u(t)
                float4 v = zero4;
                const bool xint = x >= 3 && x <= Nx - 4;
                const bool zfd = z0 + 3 >= zlo && z0 <= zhi;
                if (zfd && xint) {
                    const unsigned cs = Geo::CG * 16u;
                    const float4 xn[6] = {lds4(ca - 3 * cs), lds4(ca - 2 * cs), lds4(ca - cs),
                                          lds4(ca + cs), lds4(ca + 2 * cs), lds4(ca + 3 * cs)};
                    const float4 cf[6] = {lds4(cf_at(0, c, g)), lds4(cf_at(1, c, g)), lds4(cf_at(2, c, g)),
                                          lds4(cf_at(3, c, g)), lds4(cf_at(4, c, g)), lds4(cf_at(5, c, g))};
                    v = group2<MATH>(lo, cq, hi, xn, cf, p0, K);
                    if (z0 < zlo || z0 + 3 > zhi) {
                        if (z0 < zlo || z0 > zhi) v.x = 0.f;
                        if (z0 + 1 < zlo || z0 + 1 > zhi) v.y = 0.f;
                        if (z0 + 2 < zlo || z0 + 2 > zhi) v.z = 0.f;
                        if (z0 + 3 < zlo || z0 + 3 > zhi) v.w = 0.f;
                    }
                }
                epilogue(i, 1, x, z0, v, cq, p0, true, 0u, 0u);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&empty[st]));
    }
}

}  // namespace fwi
