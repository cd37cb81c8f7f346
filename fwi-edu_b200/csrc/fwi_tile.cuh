// fwi_tile.cuh -- the TMA-fed time-step kernel.
//
// A block owns one tile of the padded grid (TG = 16 float4 z-groups = 64 rows by TX
// columns, one consumer thread per group and column) and walks a chunk of shots that
// share the model window.  The shots' fields never pass through registers on their way
// in: one extra producer warp issues, per shot, two tensor copies (cp.async.bulk.tensor)
// -- the p1 tile with its halo (one group above and below, three columns left and right)
// and the p0 tile -- into a ring of NST shared-memory stages.  Each stage has a "full"
// mbarrier (the copies landed) and an "empty" one (every consumer warp is done with it);
// consumer warps wait only on the stage they need, so they drift apart by up to NST
// shots instead of meeting at a block-wide barrier per shot.  The six coefficient tiles
// arrive once per block, by one more tensor copy, and stay in registers for all shots
// (k_tile) or are read from shared memory per shot (k_tile3, three blocks per SM).
// Out-of-range parts of a tile (grid edges) are zero-filled by the copy engine.
//
// Arithmetic uses the packed f32x2 add/sub/fma of sm_100 on pairs of neighbouring cells
// (products of two fields as fma(a, b, -0), products by a stencil constant as scalar
// multiplies), with every operation rounded separately in the reference's association order: the
// results are bit-identical to the scalar __fadd_rn/__fmul_rn evaluation of
// acoustic_iso2d_fd_it_6order (propagation.c:13-74) and to the reference's strict IEEE
// build (MATH 0).  MATH 1 contracts multiply-adds into packed FMAs (within the FP32
// tolerance of the seismograms, not bitwise).
//
// The epilogue fuses what the reference does around the stencil: point source (forward:
// double, before the free surface, propagation.c:558; replay: float, after it, :662),
// mirror free surface (:76-101), pseudo-Hessian (:579-594), imaging (:700-714) and the
// adjoint injection (:676-682).  Its branches are uniform over a tile wherever they can
// be: only tiles that reach the free-surface rows, the source or the receiver rows take
// the corresponding code.  Receivers are found through a per-block table of the chunk's
// receivers in the tile (built once per block), both for sampling and for the injection.
//
// Every wait is bounded: a tile copy that has not landed after two seconds sets the
// error word, the block waits (again bounded) for its copies in flight and returns.
#pragma once
#include <cuda.h>  // CUtensorMap, the encoded tensor-copy descriptor type

#include <type_traits>

#include "fwi_step.cuh"

namespace fwi {

typedef unsigned long long u64;

// ------------------------------------------------------------ packed f32x2 arithmetic
__device__ __forceinline__ u64 pk(float a, float b)
{
    u64 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 upk(u64 r)
{
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
    return make_float2(a, b);
}
__device__ __forceinline__ u64 add2(u64 a, u64 b)
{
    u64 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64 sub2(u64 a, u64 b)
{
    u64 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b)
{
    u64 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c)
{
    u64 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// stencil constants (propagation.h)
constexpr float FD_C1 = 0.77793115f, FD_C2 = -0.17388691f, FD_C3 = 0.02338713f;
constexpr float FD_D0 = -2.8215452f, FD_D1 = 1.57663238f, FD_D2 = -0.18347238f, FD_D3 = 0.01761260f;

// the stencil constants and grid spacings as packed pairs (the contracted path uses them all; the
// exact path multiplies by the stencil constants as scalar immediates, which hold no registers), and
// -0 as a pair: NZ, the addend of the exact path's packed products, read at run time (negzero) so
// that the compiler cannot drop it
struct PkConst {
    u64 C1, C2, C3, D0, D1, D2, D3, idx, idz, idxx, idzz, NZ;
};
__device__ __forceinline__ PkConst make_pkconst(float invdx, float invdz, float invdxdx, float invdzdz,
                                                float negzero)
{
    PkConst K;
    K.C1 = pk(FD_C1, FD_C1);
    K.C2 = pk(FD_C2, FD_C2);
    K.C3 = pk(FD_C3, FD_C3);
    K.D0 = pk(FD_D0, FD_D0);
    K.D1 = pk(FD_D1, FD_D1);
    K.D2 = pk(FD_D2, FD_D2);
    K.D3 = pk(FD_D3, FD_D3);
    K.idx = pk(invdx, invdx);
    K.idz = pk(invdz, invdz);
    K.idxx = pk(invdxdx, invdxdx);
    K.idzz = pk(invdzdz, invdzdz);
    K.NZ = pk(negzero, negzero);
    return K;
}

// Two vertically adjacent cells of one column: propagation.c:13-74 with each product and sum
// rounded on its own, in the reference's order.  The exact path (MATH 0) must round every product
// that feeds a sum on its own, and a packed multiply would be fused by the compiler into the packed
// add that follows although both carry .rn.  So a product by a stencil constant is two scalar
// multiplies by an immediate (__fmul_rn is never contracted), and a product of two fields is one
// packed fma(a, b, -0): a*b + (-0) rounds exactly as a*b, signed zeros included, and an fma is not
// fused any further.  The sums stay packed.
template <int MATH>
__device__ __forceinline__ u64 cell2(u64 zm3, u64 zm2, u64 zm1, u64 z0, u64 zp1, u64 zp2, u64 zp3, u64 xm3, u64 xm2,
                                     u64 xm1, u64 xp1, u64 xp2, u64 xp3, u64 c1, u64 c2, u64 ck, u64 irx, u64 irz,
                                     u64 ir, u64 p0, const PkConst &k)
{
    if (MATH == 0) {
        auto mul = [&](u64 a, u64 b) { return fma2(a, b, k.NZ); };
        auto mulk = [&](float c, u64 b) {
            const float2 y = upk(b);
            return pk(__fmul_rn(c, y.x), __fmul_rn(c, y.y));
        };
        // dpdz and dpdx feed multiplies only: a packed multiply there cannot be fused into an add
        const u64 dpdz =
            mul2(add2(add2(mulk(FD_C1, sub2(zp1, zm1)), mulk(FD_C2, sub2(zp2, zm2))), mulk(FD_C3, sub2(zp3, zm3))),
                 k.idz);
        const u64 dpdx =
            mul2(add2(add2(mulk(FD_C1, sub2(xp1, xm1)), mulk(FD_C2, sub2(xp2, xm2))), mulk(FD_C3, sub2(xp3, xm3))),
                 k.idx);
        const u64 d0 = mulk(FD_D0, z0);
        const u64 dzz = mul(k.idzz, add2(add2(add2(d0, mulk(FD_D1, add2(zp1, zm1))), mulk(FD_D2, add2(zp2, zm2))),
                                           mulk(FD_D3, add2(zp3, zm3))));
        const u64 dxx = mul(k.idxx, add2(add2(add2(d0, mulk(FD_D1, add2(xp1, xm1))), mulk(FD_D2, add2(xp2, xm2))),
                                           mulk(FD_D3, add2(xp3, xm3))));
        const u64 lap = add2(add2(mul(irx, dpdx), mul(irz, dpdz)), mul(ir, add2(dxx, dzz)));
        return add2(add2(mul(c1, z0), mul(c2, p0)), mul(ck, lap));
    } else {
        const u64 dpdz = mul2(fma2(k.C3, sub2(zp3, zm3), fma2(k.C2, sub2(zp2, zm2), mul2(k.C1, sub2(zp1, zm1)))), k.idz);
        const u64 dpdx = mul2(fma2(k.C3, sub2(xp3, xm3), fma2(k.C2, sub2(xp2, xm2), mul2(k.C1, sub2(xp1, xm1)))), k.idx);
        const u64 d0 = mul2(k.D0, z0);
        const u64 dzz =
            mul2(fma2(k.D3, add2(zp3, zm3), fma2(k.D2, add2(zp2, zm2), fma2(k.D1, add2(zp1, zm1), d0))), k.idzz);
        const u64 dxx =
            mul2(fma2(k.D3, add2(xp3, xm3), fma2(k.D2, add2(xp2, xm2), fma2(k.D1, add2(xp1, xm1), d0))), k.idxx);
        const u64 lap = fma2(ir, add2(dxx, dzz), fma2(irz, dpdz, mul2(irx, dpdx)));
        return fma2(ck, lap, fma2(c2, p0, mul2(c1, z0)));
    }
}

__device__ __forceinline__ u64 lo2(const float4 &v) { return pk(v.x, v.y); }
__device__ __forceinline__ u64 hi2(const float4 &v) { return pk(v.z, v.w); }

// one float4 group (4 cells) as two packed pairs; lo/cq/hi: groups g-1, g, g+1 of column x;
// xn: column x-3, x-2, x-1, x+1, x+2, x+3 at group g; cf: c1, c2, coef3*K, irx, irz, ir
template <int MATH>
__device__ __forceinline__ float4 group2(const float4 &lo, const float4 &cq, const float4 &hi, const float4 (&xn)[6],
                                         const float4 (&cf)[6], const float4 &p0, const PkConst &k)
{
    const u64 s0 = pk(lo.y, lo.z), s1 = hi2(lo);
    const u64 s2 = pk(lo.w, cq.x), s3 = lo2(cq), s4 = pk(cq.y, cq.z), s5 = hi2(cq), s6 = pk(cq.w, hi.x);
    const u64 s7 = lo2(hi), s8 = pk(hi.y, hi.z);
    const u64 a = cell2<MATH>(s0, s1, s2, s3, s4, s5, s6, lo2(xn[0]), lo2(xn[1]), lo2(xn[2]), lo2(xn[3]), lo2(xn[4]),
                              lo2(xn[5]), lo2(cf[0]), lo2(cf[1]), lo2(cf[2]), lo2(cf[3]), lo2(cf[4]), lo2(cf[5]), lo2(p0),
                              k);
    const u64 b = cell2<MATH>(s2, s3, s4, s5, s6, s7, s8, hi2(xn[0]), hi2(xn[1]), hi2(xn[2]), hi2(xn[3]), hi2(xn[4]),
                              hi2(xn[5]), hi2(cf[0]), hi2(cf[1]), hi2(cf[2]), hi2(cf[3]), hi2(cf[4]), hi2(cf[5]), hi2(p0),
                              k);
    const float2 ra = upk(a), rb = upk(b);
    return make_float4(ra.x, ra.y, rb.x, rb.y);
}

// ------------------------------------------------------------ TMA and mbarrier
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ u64 global_ns()
{
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// arrive (the barrier's one arrival) and announce the bytes its copies will deliver
__device__ __forceinline__ void mbar_arrive_expect(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// announce more bytes without arriving
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// one try (the hardware may suspend the thread briefly while the phase is open)
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0;
}
// waits for the phase of the given parity to complete; false after limit_ns (two seconds unless
// given; the clock is read only when the first try finds the phase still open)
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, u64 limit_ns = 2000000000ull)
{
    if (mbar_try(bar, parity)) return true;
    const u64 t0 = global_ns();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}
// a 16-byte shared-memory load at a 32-bit shared address (volatile: never moved above the
// barrier wait that guards the stage it reads)
__device__ __forceinline__ float4 lds4(unsigned a)
{
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
// programmatic dependent launch: a step may start (launch its blocks, set up barriers and
// per-shot scalars) while the previous step drains; every access to the fields waits for the
// previous step to complete.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// frames read (p1 = t, p0) and written by a step of the given kind
__device__ __forceinline__ void step_frames(const ShotDesc &D, int kind, int it, int &i1, int &i0, int &io)
{
    if (kind == K_FWD0 || kind == K_FWD1) {
        const bool keep = kind == K_FWD1;
        i1 = fwd_idx(D, it, keep); i0 = fwd_idx(D, it - 1, keep); io = fwd_idx(D, it + 1, keep);
    } else if (kind == K_REP) {
        i1 = rep_idx(D, it); i0 = rep_idx(D, it - 1); io = rep_idx(D, it + 1);
    } else {
        i1 = adj_idx(D, it); i0 = adj_idx(D, it + 1); io = adj_idx(D, it - 1);
    }
}

// tile copies global -> this CTA's shared memory, completing on bar (no multicast); the
// tensor maps are __grid_constant__ kernel parameters
__device__ __forceinline__ void tma_load3(unsigned dst, const CUtensorMap *m, int c0, int c1, int c2, unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_load4(unsigned dst, const CUtensorMap *m, int c0, int c1, int c2, int c3,
                                          unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

// ------------------------------------------------------------ tile geometry
constexpr int TILE_CH_MAX = 32;  // most shots one block walks
__host__ __device__ constexpr int round128(int b) { return (b + 127) / 128 * 128; }

template <int TX>
struct TileGeom {
    static constexpr int ZP = 4 * (TG + 2);  // p1 tile rows: groups G0-1 .. G0+TG
    static constexpr int ZC = 4 * TG;        // rows of the computed tile
    static constexpr int XP = TX + 6;        // p1 tile columns: X0-3 .. X0+TX+2
    static constexpr int P1_BYTES = ZP * XP * 4;
    static constexpr int P0_BYTES = ZC * TX * 4;
    static constexpr int CF_BYTES = 6 * ZC * TX * 4;
    static constexpr int P0_OFF = round128(P1_BYTES);
    static constexpr int STAGE = P0_OFF + round128(P0_BYTES);
    static constexpr int ST_OFF = round128(CF_BYTES);
    static constexpr int smem(int nst) { return ST_OFF + nst * STAGE; }
};
// grid: x = column tile (plus one receiver-sampling index), y = 2 * shot chunk + program
// item (passed as `by`), z = tile of TG z-groups.  block = (TG / GPT) x (TX + 32 / (TG / GPT)) threads: rows
// 0..TX-1 are the consumers (GPT consecutive z-groups of one column each), the remaining rows
// form the producer warp.
// Dynamic shared memory: TileGeom<TX>::smem(NST).
// Tensor maps: tm_p1 / tm_p0 describe the group's frame pool {ld, Nx, nfr, nshot} (z
// contiguous; shot s of the group at index s - shot_base) with boxes {ZP, XP, 1, 1} and
// {ZC, TX, 1, 1}; tm_cf the six coefficient planes {ld, Nx, 6} with box {ZC, TX, 6}.
// MINB: blocks per SM the kernel is compiled for.  1 (k_tile, no minimum): with one group per
// thread the six coefficient float4s stay in registers for the chunk; 3 (k_tile3): they are read
// from shared memory per shot instead, which fits three blocks per SM (more warps to hide
// latency, at six more shared loads per group and shot).
// How a step launch waits for the one before it.  flags == null: for the whole previous grid
// (griddepcontrol.wait).  Otherwise for the 3 x 3 neighbouring tiles of the same chunk only: every
// block stores, once its consumers have released all its stages (their stores precede that), the
// program item it completed + 1 into flags[(by * zt + bz) * ntx + bx] (a gpu-scope fence first);
// the producer of a block of item L polls the neighbours' flags for Lprev + 1 (both item halves
// where the launches carry two), then fences (acquire, and the proxy fence for its tensor copies).
// A programmatic dependent launch starts only once every block of the grid before it is resident,
// so a block never waits for a block that cannot run.  The first launch of a pass (Lprev < 0)
// waits for the whole previous grid.  In this mode the grid has no receiver-sampling column: the
// tiles sample their receivers from the stage.
struct TileSync {
    int *flags;
    int Lprev;        // program item of the previous launch of this pass, or -1
    int ntx, zt;      // column and z tiles of the flag layout
    int halves;       // 1 or 2 item halves carried by the launches
};

__device__ __forceinline__ int ld_relaxed(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(int *p, int v)
{
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// the producer's wait for the neighbours' previous item (TileSync); false when it ran out (2 s).
// A set error word ends it at once: after one wait has run out, no launch of the pass waits again.
__device__ __forceinline__ bool wait_neighbours(const TileSync &ts, int by, int bx, int bz, const int *err)
{
    int idx[18], cnt = 0;
    for (int h = 0; h < ts.halves; ++h) {
        const int row = ts.halves == 2 ? ((by & ~1) | h) : by;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dx = -1; dx <= 1; ++dx) {
                const int nz = bz + dz, nx = bx + dx;
                if (nz >= 0 && nz < ts.zt && nx >= 0 && nx < ts.ntx) idx[cnt++] = (row * ts.zt + nz) * ts.ntx + nx;
            }
    }
    const int need = ts.Lprev + 1;
    const u64 t0 = global_ns();
    bool ok = true;
    for (;;) {
        int mn = need;
        for (int q = 0; q < cnt; ++q) mn = min(mn, ld_relaxed(ts.flags + idx[q]));
        if (mn >= need) break;
        if (global_ns() - t0 > 2000000000ull || ld_relaxed(err) != 0) {
            ok = false;
            break;
        }
        __nanosleep(64);
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    asm volatile("fence.proxy.async.global;" ::: "memory");
    return ok;
}

template <int TX, int NST, int MATH, int GPT, int MINB>
__device__ __forceinline__ void tile_body(const CUtensorMap &tm_p1, const CUtensorMap &tm_p0, const CUtensorMap &tm_cf,
                                          const ShotDesc *__restrict__ shots, const int4 *__restrict__ prog, int L,
                                          int shot_base, int nshot, int chunk, int *err, int bx, int by, int bz,
                                          const TileSync &ts)
{
    using Geo = TileGeom<TX>;
    constexpr int NL = TG / GPT;  // consumer lanes per column
    constexpr int NT = NL * TX + 32, NW = NL * TX / 32;
    static_assert(NL * TX >= 32 && 32 % NL == 0, "whole consumer warps, at least one");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long full[NST], empty[NST], cfbar;
    __shared__ float *s_out[TILE_CH_MAX];
    __shared__ const float *s_u[TILE_CH_MAX];
    __shared__ double s_srcd[TILE_CH_MAX];
    __shared__ float s_srcf[TILE_CH_MAX];
    __shared__ int s_isx[TILE_CH_MAX], s_isz[TILE_CH_MAX], s_rz0[TILE_CH_MAX], s_rz1[TILE_CH_MAX];
    __shared__ bool s_spec[TILE_CH_MAX];
    __shared__ int s_fi[2];  // frames of p1 and p0 (the same for every shot of the chunk)
    // TileSync mode: trace row of this step's sample per shot (or null).  The receivers of the
    // chunk's shots in the tile's columns and rows (for that sampling, and for the injection of
    // every adjoint step): (trace << 8) | (row - first row of the tile), -1 none, -2 several
    // (read from the receiver list)
    __shared__ float *s_tr[TILE_CH_MAX];
    __shared__ int s_rcv[TILE_CH_MAX][TX];
    // adjoint steps: each table entry's interpolation weight (recK), and the step's adjoint-source
    // row per shot
    __shared__ float s_rk[TILE_CH_MAX][TX];
    __shared__ const float *s_adj[TILE_CH_MAX];

    grid_dep_launch();  // the next step may begin its set-up once every block of this one runs
    const bool fine = ts.flags != nullptr;
    const int4 pw = prog[L];
    const int kind = (by & 1) ? pw.z : pw.x;
    const int it = (by & 1) ? pw.w : pw.y;
    if (kind == K_NONE) {
        // an idle item half still completes its item in order, for the flags' readers
        if (fine && threadIdx.x == 0 && threadIdx.y == 0) {
            int *own = ts.flags + (by * ts.zt + bz) * ts.ntx + bx;
            const u64 t0 = global_ns();
            while (ts.Lprev >= 0 && ld_relaxed(own) < ts.Lprev + 1 && global_ns() - t0 < 2000000000ull &&
                   ld_relaxed(err) == 0)
                __nanosleep(64);
            asm volatile("fence.acq_rel.gpu;" ::: "memory");
            st_relaxed_gpu(own, L + 1);
        }
        return;
    }
    const int cb = shot_base + (by >> 1) * chunk;
    const int n = min(chunk, shot_base + nshot - cb);
    if (n <= 0) return;
    const ShotDesc &A = shots[cb];  // geometry and coefficients of the chunk
    const int Nx = A.Nx, pml = A.pml, G = A.G, Nz = A.Nz;
    const int ntx = (Nx + TX - 1) / TX;
    const bool fwd = kind == K_FWD0 || kind == K_FWD1;
    const int tid = threadIdx.y * NL + threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    // ---- the receiver-sampling block: p1 is read-only during this launch
    if (bx >= ntx) {
        if (!fwd || it % A.sr != 0 || bx > ntx || bz != 0) return;
        grid_dep_wait();
        for (int s = 0; s < n; ++s) {
            const ShotDesc &D = shots[cb + s];
            const float *p1 = fwd_buf(D, it, kind == K_FWD1);
            float *tr = D.traces_t + (long long)(it / D.sr) * D.ntr;
            for (int r = tid; r < D.ntr; r += NT) tr[r] = p1[D.rec_off[r]];
        }
        return;
    }

    const int X0 = bx * TX, G0 = bz * TG;
    unsigned char *st_base = smem + Geo::ST_OFF;
    const bool producer = warp == NW && lane == 0;
    int issued = 0;  // shots whose copies the producer has issued
    bool spec_here = false;
    if (producer) {
        // ---- barriers, then the coefficient tile and the first NST shots' copies at once: the
        // copies are in flight while the consumers compute the per-shot scalars
        for (int j = 0; j < NST; ++j) {
            mbar_init(smem_u32(&full[j]), 1);
            mbar_init(smem_u32(&empty[j]), NW);
        }
        mbar_init(smem_u32(&cfbar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        int i1, i0, io;
        step_frames(A, kind, it, i1, i0, io);  // the same frames for every shot of the chunk
        s_fi[0] = i1;
        s_fi[1] = i0;
        if (fine && ts.Lprev >= 0) {
            // the coefficients are the pass's own (the pass's first launch read them after waiting
            // for everything before it): their copy overlaps the wait for the neighbours
            mbar_arrive_expect(smem_u32(&cfbar), Geo::CF_BYTES);
            tma_load3(smem_u32(smem), &tm_cf, 4 * G0, X0, 0, smem_u32(&cfbar));
            if (!wait_neighbours(ts, by, bx, bz, err)) atomicExch(err, 1);
        } else {
            grid_dep_wait();
            mbar_arrive_expect(smem_u32(&cfbar), Geo::CF_BYTES);
            tma_load3(smem_u32(smem), &tm_cf, 4 * G0, X0, 0, smem_u32(&cfbar));
        }
        for (; issued < min(n, NST); ++issued) {
            const unsigned b = smem_u32(&full[issued]);
            mbar_arrive_expect(b, Geo::P1_BYTES + Geo::P0_BYTES);
            unsigned char *stg = st_base + issued * Geo::STAGE;
            tma_load4(smem_u32(stg), &tm_p1, 4 * (G0 - 1), X0 - 3, i1, cb + issued - shot_base, b);
            tma_load4(smem_u32(stg + Geo::P0_OFF), &tm_p0, 4 * G0, X0, i0, cb + issued - shot_base, b);
        }
    } else if (tid < n) {
        // ---- per-shot scalars of the chunk (frame indices need divisions: once per block)
        const ShotDesc &D = shots[cb + tid];
        int i1, i0, io, iu = -1;
        step_frames(D, kind, it, i1, i0, io);
        if (kind == K_ADJ && it % MST == 0) iu = img_idx(D, it);
        s_out[tid] = frame_ptr(D, io);
        s_u[tid] = iu >= 0 ? frame_ptr(D, iu) : nullptr;
        s_isx[tid] = D.isx;
        s_isz[tid] = D.isz;
        s_srcd[tid] = fwd ? D.srcd[it] : 0.0;
        s_srcf[tid] = kind == K_REP ? D.srcf[it] : 0.0f;
        s_rz0[tid] = D.rz0;
        s_rz1[tid] = D.rz1;
        // does this tile need the rare parts of the epilogue for this shot (its source, its
        // receiver rows for the adjoint injection)?
        const int X0t = bx * TX, Z0t = 4 * bz * TG;
        const bool src_t = (fwd || kind == K_REP) && D.isx >= X0t && D.isx < X0t + TX && D.isz >= Z0t &&
                           D.isz < Z0t + 4 * TG;
        const bool inj_t = kind == K_ADJ && it >= 1 && Z0t + 4 * TG > D.rz0 && Z0t <= D.rz1;
        // TileSync mode: this tile samples the shot's receivers in its rows
        float *tr = (fine && fwd && it % D.sr == 0) ? D.traces_t + (long long)(it / D.sr) * D.ntr : nullptr;
        const bool smp_t = tr != nullptr && Z0t + 4 * TG > D.rz0 && Z0t <= D.rz1;
        s_tr[tid] = smp_t ? tr : nullptr;
        s_adj[tid] = inj_t ? D.adj_t + (long long)(it - 1) * D.ntr : nullptr;
        s_spec[tid] = src_t || inj_t || smp_t;
        spec_here = s_spec[tid];
    }
    const bool inj_tab = kind == K_ADJ && it >= 1;
    if (((fine && fwd && it % A.sr == 0) || inj_tab) && warp < NW) {
        // the receiver table of the chunk's shots in this tile (one pass of the consumers): for
        // the receiver sampling of a forward step, or the adjoint injection, so that a shot's
        // step finds its receivers without a chain of dependent loads
        const int z_a = 4 * G0, z_b = 4 * G0 + 4 * TG - 1;
        for (int q = tid; q < n * TX; q += NL * TX) {
            const int sq = q / TX, kq = q - sq * TX, xq = X0 + kq;
            const ShotDesc &D = shots[cb + sq];
            int code = -1;
            float rk = 0.0f;
            if (xq < Nx && D.rz1 >= z_a && D.rz0 <= z_b)
                for (int e = D.colptr[xq]; e < D.colptr[xq + 1]; ++e) {
                    const int2 r = D.rec[e];
                    if (r.x < z_a || r.x > z_b) continue;
                    code = code == -1 ? (r.y << 8) | (r.x - z_a) : -2;
                    if (inj_tab) rk = D.recK[e];
                }
            s_rcv[sq][kq] = code;
            if (inj_tab) s_rk[sq][kq] = rk;
        }
    }
    // barriers and the per-shot scalars; no block-wide barrier follows.  any_spec: some shot of
    // the chunk has its source or receiver rows in this tile
    const bool any_spec = __syncthreads_or(spec_here) != 0;
    // fields and accumulators: after the previous step (the producer waited already; with
    // TileSync the consumers touch them only after a stage the producer filled after its wait)
    if (!fine || ts.Lprev < 0) grid_dep_wait();

    if (warp == NW) {
        // ---- producer: shot j into stage j % NST once every consumer warp has released that
        // stage's previous shot
        if (lane != 0) return;
        const int i1 = s_fi[0], i0 = s_fi[1];
        for (int j = issued; j < n; ++j) {
            const int st = j % NST;
            if (j >= NST && !mbar_wait(smem_u32(&empty[st]), (j / NST - 1) & 1)) {
                atomicExch(err, 1);
                break;
            }
            const int sg = cb + j - shot_base;  // shot index in the pool
            const unsigned b = smem_u32(&full[st]);
            mbar_arrive_expect(b, Geo::P1_BYTES + Geo::P0_BYTES);
            unsigned char *stg = st_base + st * Geo::STAGE;
            tma_load4(smem_u32(stg), &tm_p1, 4 * (G0 - 1), X0 - 3, i1, sg, b);
            tma_load4(smem_u32(stg + Geo::P0_OFF), &tm_p0, 4 * G0, X0, i0, sg, b);
            issued = j + 1;
        }
        // keep the block alive until every copy it issued has landed (the consumers wait for
        // them too, unless they gave up)
        mbar_wait(smem_u32(&cfbar), 0);
        for (int j = max(0, issued - NST); j < issued; ++j) mbar_wait(smem_u32(&full[j % NST]), (j / NST) & 1);
        if (fine) {
            // the item is complete once the consumers have released every stage (their stores come
            // before their release): publish it
            for (int j = max(0, n - NST); j < n; ++j) mbar_wait(smem_u32(&empty[j % NST]), (j / NST) & 1);
            asm volatile("fence.acq_rel.gpu;" ::: "memory");
            st_relaxed_gpu(ts.flags + (by * ts.zt + bz) * ts.ntx + bx, L + 1);
        }
        return;
    }

    // ---- consumers: lane zl of column k owns the GPT z-groups G0 + GPT*zl .. G0 + GPT*zl + GPT-1
    const int zl = threadIdx.x, k = threadIdx.y;
    const int x = X0 + k;
    const bool xin = x < Nx, xint = x >= 3 && x <= Nx - 4;
    const int zlo = A.izStart, zhi = Nz - 4;
    // Free surface.  The reference sets row pml to -0 and mirrors rows pml+1..2pml into rows
    // pml-1..0 (propagation.c:76-101).  Only the three mirrored rows next to the surface are ever
    // read again (the stencil updates rows >= pml and reaches three rows up; receivers, imaging
    // and the Hessian lie at rows >= pml), so only rows pml+1..pml+3 are mirrored here: every
    // seismogram and gradient is the reference's, and the rows above pml-3 are never written --
    // except on the steps whose output field is written out as a snapshot (A.snap), which
    // mirror all pml rows so that the snapshot holds what the reference's field holds.
    const int tout = kind == K_ADJ ? it - 1 : it + 1;  // time index of the field this step writes
    const int fs_hi = (A.snap > 0 && tout % A.snap == 0) ? 2 * pml : min(2 * pml, pml + 3);  // last mirrored source row
    const bool inject = kind == K_ADJ && it >= 1;
    const bool hess = kind == K_FWD1 && A.hessian && (it % MST == 0);
    const bool image = kind == K_ADJ && (it % MST == 0);
    const bool xacc = x >= pml && x < pml + A.nxx;
    const bool fs_tile = A.fs && 4 * G0 <= fs_hi;  // tile holds the surface, mirror or rows above
    const bool acc_tile = hess || image;
    const long long colx = (long long)x * A.ld;
    const float invdx = A.invdx, invdz = A.invdz, invdtdt = A.invdtdt;
    const PkConst K = make_pkconst(invdx, invdz, A.invdxdx, A.invdzdz, A.negzero);
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4(*scf)[TX][TG] = reinterpret_cast<const float4(*)[TX][TG]>(smem);
    constexpr bool CF_REG = GPT == 1 && MINB < 3;
    float4 cfh[6];  // CF_REG: the thread's coefficients stay in registers for the chunk

    // group gl of the tile for shot i: stencil from the stage, fused epilogue, store;
    // lo / cq / hi are groups gl-1, gl, gl+1 of column x
    // the updated value of group gl (zero outside the updated rows and columns); p0: the
    // group's previous field, which the general epilogue needs too
    auto group_value = [&](unsigned sb, int gl, const float4 &lo, const float4 &cq, const float4 &hi,
                           float4 &p0) {
        const int z0 = 4 * (G0 + gl);
        const int cx = k + 3, cg = gl + 1;
        const bool zfd = z0 + 3 >= zlo && z0 <= zhi;
        p0 = lds4(sb + Geo::P0_OFF + (unsigned)(k * TG + gl) * 16u);
        float4 v = zero4;
        if (zfd && xint) {
            const unsigned xa = sb + (unsigned)(cx * (TG + 2) + cg) * 16u, cs = (TG + 2) * 16u;
            const float4 xn[6] = {lds4(xa - 3 * cs), lds4(xa - 2 * cs), lds4(xa - cs),
                                  lds4(xa + cs), lds4(xa + 2 * cs), lds4(xa + 3 * cs)};
            if (CF_REG) {
                v = group2<MATH>(lo, cq, hi, xn, cfh, p0, K);
            } else {
                const float4 cf[6] = {scf[0][k][gl], scf[1][k][gl], scf[2][k][gl],
                                      scf[3][k][gl], scf[4][k][gl], scf[5][k][gl]};
                v = group2<MATH>(lo, cq, hi, xn, cf, p0, K);
            }
            if (z0 < zlo || z0 + 3 > zhi) {  // group straddles the edge of the updated rows
                if (z0 < zlo || z0 > zhi) v.x = 0.f;
                if (z0 + 1 < zlo || z0 + 1 > zhi) v.y = 0.f;
                if (z0 + 2 < zlo || z0 + 2 > zhi) v.z = 0.f;
                if (z0 + 3 < zlo || z0 + 3 > zhi) v.w = 0.f;
            }
        }
        return v;
    };

    // group gl of the tile for shot i, in a tile and shot that need none of the rare parts of
    // the epilogue: the value and its store only
    auto consume_group_fast = [&](int i, unsigned sb, int gl, const float4 &lo, const float4 &cq,
                                  const float4 &hi) {
        const int g = G0 + gl;
        if (g >= G || !xin) return;
        float4 p0;
        const float4 v = group_value(sb, gl, lo, cq, hi, p0);
        *reinterpret_cast<float4 *>(s_out[i] + colx + 4 * g) = v;
    };

    // group gl of the tile for shot i with the whole epilogue
    auto consume_group = [&](int i, unsigned sb, int gl, const float4 &lo,
                             const float4 &cq, const float4 &hi) {
        const int g = G0 + gl, z0 = 4 * g;
        if (g >= G || !xin) return;
        if (fine && s_tr[i] != nullptr) {  // receivers sample u(t) before the step
            const int code = s_rcv[i][k];
            if (code >= 0) {
                const int row = 4 * G0 + (code & 255);
                if (row >= z0 && row < z0 + 4) s_tr[i][code >> 8] = comp(cq, row - z0);
            } else if (code == -2) {
                const ShotDesc &D = shots[cb + i];
                for (int e = __ldg(D.colptr + x), e1 = __ldg(D.colptr + x + 1); e < e1; ++e) {
                    const int2 r = __ldg(D.rec + e);
                    if (r.x >= z0 && r.x < z0 + 4) s_tr[i][r.y] = comp(cq, r.x - z0);
                }
            }
        }
        // above the free surface (rows < pml): never updated, stored or accumulated; the
        // mirrored rows pml-3..pml-1 are written by the groups that hold pml+1..pml+3
        if (A.fs && z0 + 3 < pml) return;
        // adjoint injection of a tile column with one receiver: its sample is loaded first, so
        // that the load overlaps the stencil
        const int code_inj = inject ? s_rcv[i][k] : -1;
        int inj_j = -1;
        float adjv = 0.0f;
        if (code_inj >= 0) {
            const int row = 4 * G0 + (code_inj & 255);
            if (row >= z0 && row < z0 + 4) {
                inj_j = row - z0;
                adjv = __ldg(s_adj[i] + (code_inj >> 8));
            }
        }
        float4 p0;
        float4 v = group_value(sb, gl, lo, cq, hi, p0);
        const long long col = colx + z0;
        const bool fs_top = A.fs && z0 <= fs_hi;  // the surface row, the mirror source rows, or above
        const int jpml = (pml >= z0 && pml < z0 + 4) ? pml - z0 : -1;
        const int isx = s_isx[i], isz = s_isz[i];
        const bool src_here = x == isx && isz >= z0 && isz < z0 + 4;
        // forward: the source enters before the free surface, in double (propagation.c:558-564)
        if (fwd && src_here) setc(v, isz - z0, (float)__dadd_rn((double)comp(v, isz - z0), s_srcd[i]));
        float4 mir = zero4;
        if (fs_top) {
            if (jpml >= 0) setc(v, jpml, -0.0f);
            mir = make_float4(-v.x, -v.y, -v.z, -v.w);
        }
        // replay: free surface first, then the float source (propagation.c:656-662)
        if (kind == K_REP && src_here) setc(v, isz - z0, fa(comp(v, isz - z0), s_srcf[i]));
        if (acc_tile && xacc && z0 + 3 >= pml && z0 < pml + A.nz) {
            const ShotDesc &D = shots[cb + i];
            const float4 uu = image ? ldg4(s_u[i] + col) : zero4;
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
        if (inject && z0 + 3 >= s_rz0[i] && z0 <= s_rz1[i] && code_inj >= 0) {
            // the tile column's one receiver (the table): its sample was loaded before the stencil
            if (inj_j >= 0) {
                const float a = fm(fm(fm(fm(fm(adjv, s_rk[i][k]), A.dt), A.dt), invdx), invdz);
                setc(v, inj_j, fs_(comp(v, inj_j), a));
            }
        } else if (inject && z0 + 3 >= s_rz0[i] && z0 <= s_rz1[i] && code_inj == -2) {
            // several receivers in the tile column: the column's list, in its order
            const ShotDesc &D = shots[cb + i];
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
        float *out = s_out[i];
        if (!fs_top || z0 >= pml) {
            *reinterpret_cast<float4 *>(out + col) = v;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (z0 + j >= pml) out[col + j] = comp(v, j);
        }
        if (fs_top) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int z = z0 + j;
                if (z > pml && z <= fs_hi) out[colx + 2 * pml - z] = comp(mir, j);
            }
        }
    };

    // one shot of the chunk from ring stage st: the lane's GPT groups, sharing their z-window;
    // FAST: the store-only epilogue
    auto consume_shot = [&](int i, int st, auto fast) {
        // stage st as a 32-bit shared address: p1 tile [XP][TG + 2] float4, then p0 [TX][TG]
        const unsigned sb = smem_u32(st_base) + (unsigned)(st * Geo::STAGE);
        const int gl0 = GPT * zl;
        float4 w[GPT + 2];  // groups gl0-1 .. gl0+GPT of column x (stage rows gl0 .. gl0+GPT+1)
        const unsigned wa = sb + (unsigned)((k + 3) * (TG + 2) + gl0) * 16u;
#pragma unroll
        for (int q = 0; q < GPT + 2; ++q) w[q] = lds4(wa + 16u * q);
#pragma unroll
        for (int j = 0; j < GPT; ++j) {
            if (decltype(fast)::value) consume_group_fast(i, sb, gl0 + j, w[j], w[j + 1], w[j + 2]);
            else consume_group(i, sb, gl0 + j, w[j], w[j + 1], w[j + 2]);
        }
    };

    const bool rare_tile = fs_tile || acc_tile;
    {  // coefficient tiles, once for all shots
        bool ok = mbar_wait(smem_u32(&cfbar), 0);
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) atomicExch(err, 1);
            return;
        }
        if (CF_REG) {
#pragma unroll
            for (int f = 0; f < 6; ++f) cfh[f] = scf[f][k][zl];
        }
    }
    // the shots of the chunk in order; PLAIN: no shot needs the rare parts of the epilogue in
    // this tile (surface, accumulators, source, injection), so the loop holds the store-only
    // consumer alone and stays lean
    auto walk = [&](auto plain) {
        for (int i = 0; i < n; ++i) {
            const int st = i % NST;
            bool ok = mbar_wait(smem_u32(&full[st]), (i / NST) & 1);
            if (!__all_sync(0xffffffffu, ok)) {  // the warp gives up as one
                if (lane == 0) atomicExch(err, 1);
                break;
            }
            if (decltype(plain)::value || (!rare_tile && !s_spec[i])) consume_shot(i, st, std::true_type());
            else consume_shot(i, st, std::false_type());
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&empty[st]));
        }
    };
    if (!rare_tile && !any_spec) walk(std::true_type());
    else walk(std::false_type());
}

// the step kernel; the tensor maps are kernel parameters in constant space (the body takes
// their addresses)
// halves: 2 -- grid row y is 2 * chunk + item half; 1 -- the items' second halves are empty and
// row y is the chunk (its first half)
template <int TX, int NST, int MATH, int GPT>
__global__ void __launch_bounds__(TG / GPT * TX + 32)
    k_tile(const __grid_constant__ CUtensorMap tm_p1, const __grid_constant__ CUtensorMap tm_p0,
           const __grid_constant__ CUtensorMap tm_cf, const ShotDesc *__restrict__ shots, const int4 *__restrict__ prog,
           int L, int shot_base, int nshot, int chunk, int halves, int *err, const TileSync ts)
{
    tile_body<TX, NST, MATH, GPT, 1>(tm_p1, tm_p0, tm_cf, shots, prog, L, shot_base, nshot, chunk, err, blockIdx.x,
                                     halves == 2 ? blockIdx.y : 2 * blockIdx.y, blockIdx.z, ts);
}

// the same step compiled for three blocks per SM, one group per thread, coefficients read from
// shared memory per shot
template <int TX, int NST, int MATH>
__global__ void __launch_bounds__(TG * TX + 32, 3)
    k_tile3(const __grid_constant__ CUtensorMap tm_p1, const __grid_constant__ CUtensorMap tm_p0,
            const __grid_constant__ CUtensorMap tm_cf, const ShotDesc *__restrict__ shots, const int4 *__restrict__ prog,
            int L, int shot_base, int nshot, int chunk, int halves, int *err, const TileSync ts)
{
    tile_body<TX, NST, MATH, 1, 3>(tm_p1, tm_p0, tm_cf, shots, prog, L, shot_base, nshot, chunk, err, blockIdx.x,
                                   halves == 2 ? blockIdx.y : 2 * blockIdx.y, blockIdx.z, ts);
}

// ------------------------------------------------------------ several groups in one launch
// One shot group of a launch that advances several independent runs at once (the continuous
// batching of the request loop): its own tensor maps (in global memory), shots, program and the
// launch index at which its program started.  The launch is a flat list of blocks: group g owns
// blocks b0 .. b0 + nblk - 1, one per (column tile or receiver column, z tile, row), so no block
// of the launch is idle by construction; a block finds its group by its index.
struct __align__(128) TileGroup {
    CUtensorMap p1, p0, cf;       // as the single-group kernel's parameters
    const ShotDesc *shots;        // descriptors of the run's shots (shot_base .. shot_base + nshot - 1)
    const int4 *prog;             // the group's current program
    long long L0;                 // launch index of the program's item 0
    int nprog;                    // items of the program
    int shot_base, nshot, chunk;  // as the single-group kernel's parameters
    int b0, nblk;                 // first block and blocks of the group
    int ntx, zt;                  // column tiles (ntx: the receiver-sampling column) and z tiles
    int halves;                   // 1: the program uses item halves .x only (forward); 2: both
    int *flags;                   // non-null: neighbour waits (TileSync) over the group's own flags,
                                  // no sampling column; null: whole-grid waits
};

// the group's block l as (column tile, row, z tile) in the single-group grid's order (column tile
// fastest, then the chunk and item half, then the z tile), and its TileSync
__device__ __forceinline__ void group_block(const TileGroup &T, long long Lg, int l, int &bx, int &by, int &bz,
                                            TileSync &ts)
{
    const int cols = T.flags ? T.ntx : T.ntx + 1;
    const int rows = T.nblk / (cols * T.zt);
    bx = l % cols;
    const int rest = l / cols;
    const int row = rest % rows;
    bz = rest / rows;
    by = T.halves == 2 ? row : 2 * row;
    ts = TileSync{T.flags, Lg > 0 ? (int)Lg - 1 : -1, T.ntx, T.zt, T.halves};
}

template <int TX, int NST, int MATH>
__global__ void __launch_bounds__(TG * TX + 32, 3)
    k_tile_groups(const TileGroup *__restrict__ groups, int ngroups, long long L, int *err)
{
    // the block's group: the last one whose first block is at or before this one (b0 rises with
    // the group index).  Each warp counts them 32 at a time with one load per lane and a ballot,
    // instead of one dependent load per group.
    int g = -1;
    {
        const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
        for (int base = 0; base < ngroups; base += 32) {
            const int i = base + lane;
            const bool le = i < ngroups && __ldg(&groups[i].b0) <= (int)blockIdx.x;
            g += __popc(__ballot_sync(0xffffffffu, le));
        }
        g = max(g, 0);
    }
    const TileGroup &T = groups[g];
    const long long Lg = L - T.L0;
    if (Lg < 0 || Lg >= T.nprog) return;
    const int l = (int)blockIdx.x - T.b0;
    // blocks in the single-group kernel's order (the surface tiles, whose epilogue is longest,
    // start first)
    int bx, by, bz;
    TileSync ts;
    group_block(T, Lg, l, bx, by, bz, ts);
    // the maps live in global memory, written before the launch: the producer warp (the only
    // one that issues tensor copies) makes them visible to its tensor-map proxy and brings them
    // into the descriptor cache before its copies use them
    if (threadIdx.y * TG + threadIdx.x >= TG * TX) {
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&T.p1) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&T.p0) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&T.cf) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&T.p1) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&T.p0) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&T.cf) : "memory");
    }
    tile_body<TX, NST, MATH, 1, 3>(T.p1, T.p0, T.cf, T.shots, T.prog, (int)Lg, T.shot_base, T.nshot, T.chunk, err,
                                   bx, by, bz, ts);
}

// The same launch with the group table as a kernel parameter (constant space, up to
// GROUPS_PARAM groups: 24 KB of the 32 KB a launch may pass).  The tensor maps are then
// parameters like those of the single-group kernels: no fences, no descriptor fetches from global
// memory.
constexpr int GROUPS_PARAM = 48;
struct __align__(128) GroupTable {
    TileGroup g[GROUPS_PARAM];
};

template <int TX, int NST, int MATH>
__global__ void __launch_bounds__(TG * TX + 32, 3)
    k_tile_groups_p(const __grid_constant__ GroupTable tab, int ngroups, long long L, int *err)
{
    int g = -1;
    {
        const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
        for (int base = 0; base < ngroups; base += 32) {
            const int i = base + lane;
            const bool le = i < ngroups && tab.g[i].b0 <= (int)blockIdx.x;
            g += __popc(__ballot_sync(0xffffffffu, le));
        }
        g = max(g, 0);
    }
    const TileGroup &T = tab.g[g];
    const long long Lg = L - T.L0;
    if (Lg < 0 || Lg >= T.nprog) return;
    const int l = (int)blockIdx.x - T.b0;
    // blocks in the single-group kernel's order (the surface tiles, whose epilogue is longest,
    // start first)
    int bx, by, bz;
    TileSync ts;
    group_block(T, Lg, l, bx, by, bz, ts);
    tile_body<TX, NST, MATH, 1, 3>(T.p1, T.p0, T.cf, T.shots, T.prog, (int)Lg, T.shot_base, T.nshot, T.chunk, err,
                                   bx, by, bz, ts);
}

}  // namespace fwi
