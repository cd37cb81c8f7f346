// fwi_wave.cuh -- the forward pass as one persistent launch (a wavefront over tiles and steps).
//
// The step kernel of fwi_tile.cuh is launched once per time step.  Every launch pays a fixed
// price on top of its work: the tail of its last wave of blocks (the next step cannot begin
// until the slowest block of this one has finished), the drain and refill of the copy pipeline
// at that boundary, and each block's prologue (barriers, the coefficient tile, the first ring
// copies).  Measured on the 221 x 601 survey that is ~5.7 us per launch against a marginal
// 0.65 us per shot and step.
//
// Here one launch runs a whole forward program.  Every block owns one tile (16 columns x 64
// rows) and one range of the group's shots for all steps, so the coefficient tile is copied
// once per launch and the block's ring of shared-memory stages streams (step, shot) items
// without a break.  The blocks are all resident (cooperative launch) and synchronise with
// their eight neighbouring tiles only: item (L, s) may read the fields once the 3 x 3 tiles
// around it have finished item (L-1, s) of the same shot range.  Each block publishes, in a
// counter in global memory, how many of its items are complete; its producer warp publishes
// items once the consumer warps have released their stages (their stores precede that release),
// in batches, with a gpu-scope fence before the counter store, and acquires the neighbours'
// counters, followed by a proxy fence, before its tensor copies read what they wrote.  Every
// dependency points at an earlier step, and publishing never waits for copies to be issued, so
// the launch cannot deadlock while all blocks are resident.  The wavefront condition covers
// the frame reuse too: a step writes u(t+1) over the frame of u(t-3), whose last readers (the
// neighbours at step t-3 and this tile at step t-2) precede it through the chain of
// dependencies.
//
// Receivers are sampled inside the tile, from u(t) in the stage (the launch path has a separate
// column of sampling blocks for that).  The stencil, the forward source, the free surface and
// the pseudo-Hessian are those of the step kernel (the same arithmetic, bit for bit).
//
// Every wait is bounded: a counter or a copy that does not arrive within two seconds sets the
// error word and the abort word; the other blocks see the abort word in their own waits, and
// every block waits (bounded) for its copies in flight before it exits.
//
// Measured on B200 (60 shots, 221 x 601, 1001 steps): 57.8 us per step against 43.6 us for the
// step launches, so the engine uses it only on request (FWI_PERSIST=1).  The fixed cost it removes
// is real, but a block's tile is fixed for the whole pass: the tiles with the free surface and the
// sources take the longer epilogue every step and pace every other tile through the dependency
// chain (53.0 us with the receiver sampling removed, 48.0 us with every tile on the store-only
// epilogue, both timing-only builds), while the step launches let the hardware balance uneven
// blocks across the SMs.
#pragma once
#include "fwi_tile.cuh"

namespace fwi {

constexpr int WAVE_TX = 16;      // tile columns
constexpr int WAVE_CH_MAX = 32;  // most shots one block owns
constexpr int WAVE_NB = 4;       // per-step scalar buffers: the consumers trail the producer by at
                                 // most ceil(NST / n) <= 2 steps (n >= 2 shots per block)

struct WaveStep {  // one step of the block's shots
    int kind, it;
    int i1, i0;    // frames read (the same for every shot of a group)
    int hess;      // the step accumulates the pseudo-Hessian
    int sample;    // the step samples the receivers
};
struct WaveShot {  // one step of one shot
    float *out;    // frame written
    float *tr;     // trace row of this step's sample, or null
    double srcd;   // forward source term (propagation.c:558)
};

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(int *p, int v)
{
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0;
}

// grid: ntx * zt * nranges blocks (block b: tile b / nranges, shot range b % nranges), all
// resident; block = (TG, WAVE_TX + 32 / TG) threads, the last row the producer warp.
// Shot range r holds shots shot_base + r*n .. + n - 1 (the last one fewer).  The program's
// items L0 .. L1-1 are forward steps (item L advances every shot from u(L) to u(L+1)).
// flags[0]: abort word; flags[1 + b]: items block b has completed in this launch (item
// (L, s) of a block is its (L - L0) * n_r + s-th); zero before the launch.
// Tensor maps and dynamic shared memory as k_tile3's (TileGeom<16>::smem(NST)).
template <int NST, int MATH>
__global__ void __launch_bounds__(TG * WAVE_TX + 32, 3)
    k_wave(const __grid_constant__ CUtensorMap tm_p1, const __grid_constant__ CUtensorMap tm_p0,
           const __grid_constant__ CUtensorMap tm_cf, const ShotDesc *__restrict__ shots, const int4 *__restrict__ prog,
           int L0, int L1, int shot_base, int nshot, int n, int ntx, int zt, int nranges, int *flags, int *err)
{
    constexpr int TX = WAVE_TX;
    using Geo = TileGeom<TX>;
    constexpr int NC = TG * TX, NW = NC / 32;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long full[NST], empty[NST], cfbar;
    __shared__ WaveStep s_step[WAVE_NB];
    __shared__ WaveShot s_shot[WAVE_NB][WAVE_CH_MAX];
    __shared__ int s_isx[WAVE_CH_MAX], s_isz[WAVE_CH_MAX], s_rz0[WAVE_CH_MAX], s_rz1[WAVE_CH_MAX];
    __shared__ double *s_H[WAVE_CH_MAX];
    // receivers of the block's shots in its columns and rows: (trace << 8) | (row - first row of
    // the tile) for the one receiver of a column; -1 none; -2 several (rare: read from the list)
    __shared__ int s_rcv[WAVE_CH_MAX][WAVE_TX];

    const int b = blockIdx.x;
    const int tile = b / nranges, range = b - tile * nranges;
    const int bx = tile % ntx, bz = tile / ntx;
    const int cb = shot_base + range * n;
    const int nr = min(n, shot_base + nshot - cb);  // shots of this block
    const ShotDesc &A = shots[cb];
    const int Nx = A.Nx, pml = A.pml, G = A.G, Nz = A.Nz;
    const int X0 = bx * TX, G0 = bz * TG;
    const int tid = threadIdx.y * TG + threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    int *abort_w = flags;
    int *mine = flags + 1 + b;
    unsigned char *st_base = smem + Geo::ST_OFF;
    const int total = (L1 - L0) * nr;

    if (tid == NC) {
        for (int j = 0; j < NST; ++j) {
            mbar_init(smem_u32(&full[j]), 1);
            mbar_init(smem_u32(&empty[j]), NW);
        }
        mbar_init(smem_u32(&cfbar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    } else if (tid < nr) {
        const ShotDesc &D = shots[cb + tid];
        s_isx[tid] = D.isx;
        s_isz[tid] = D.isz;
        s_rz0[tid] = D.rz0;
        s_rz1[tid] = D.rz1;
        s_H[tid] = D.H;
    }
    if (tid < NC) {
        const int z_a = 4 * G0, z_b = 4 * G0 + 4 * TG - 1;
        for (int q = tid; q < nr * TX; q += NC) {
            const int sq = q / TX, kq = q - sq * TX, xq = X0 + kq;
            int code = -1;
            if (xq < Nx) {
                const ShotDesc &D = shots[cb + sq];
                for (int e = D.colptr[xq]; e < D.colptr[xq + 1]; ++e) {
                    const int2 r = D.rec[e];
                    if (r.x < z_a || r.x > z_b) continue;
                    code = code == -1 ? (r.y << 8) | (r.x - z_a) : -2;
                }
            }
            s_rcv[sq][kq] = code;
        }
    }
    __syncthreads();

    if (warp == NW) {
        // ------------------------------------------------------------ producer warp
        // lanes 0..8 watch the counters of the 3 x 3 tiles around this one (same shot range)
        const int *nb = nullptr;
        if (lane < 9) {
            const int nx = bx + lane % 3 - 1, nz = bz + lane / 3 - 1;
            if (nx >= 0 && nx < ntx && nz >= 0 && nz < zt) nb = flags + 1 + (nz * ntx + nx) * nranges + range;
        }
        int seen = 0;        // the last value read from nb
        int done_l = 0;      // items whose stages the consumers have released (in order)
        int pub = 0;         // items published in the counter (lane 0)
        bool failed = false;
        const u64 limit = 2000000000ull;
        // warp-uniform: the wait begun at t0 has run out, or another block gave up (the abort word
        // is read only once a wait has lasted 20 us: a normal wait is far shorter)
        auto expired = [&](u64 t0) {
            const u64 w = global_ns() - t0;
            return __any_sync(0xffffffffu, w > limit || (w > 20000 && *(volatile int *)abort_w != 0));
        };
        // Count the items whose stages the consumers have released, and publish them: in batches
        // of PUB_BATCH (each publication costs a gpu-scope fence, and the neighbours need an
        // item only a step of the block's shots later), and all of them whenever the producer is
        // about to wait for a neighbour or is done, so that no block ever waits on an item that
        // its owner has finished but holds back.
        constexpr int PUB_BATCH = 8;
        auto publish = [&](int issued, bool force) {
            if (lane == 0) {
                while (done_l < issued && mbar_test(smem_u32(&empty[done_l % NST]), (done_l / NST) & 1)) ++done_l;
                if (done_l != pub && (force || done_l - pub >= PUB_BATCH)) {
                    asm volatile("fence.acq_rel.gpu;" ::: "memory");
                    st_relaxed(mine, done_l);
                    pub = done_l;
                }
            }
            done_l = __shfl_sync(0xffffffffu, done_l, 0);
        };
        if (lane == 0) {
            mbar_arrive_expect(smem_u32(&cfbar), Geo::CF_BYTES);
            tma_load3(smem_u32(smem), &tm_cf, 4 * G0, X0, 0, smem_u32(&cfbar));
        }
        int j = 0;
        for (; j < total; ++j) {
            const int Lr = j / nr, s = j - Lr * nr, L = L0 + Lr;
            if (s == 0) {
                // this step's scalars (buffer L % 4 is free: the consumers are within two steps)
                const int4 pw = prog[L];
                const int kind = pw.x, it = pw.y;
                for (int q = lane; q < nr; q += 32) {
                    const ShotDesc &D = shots[cb + q];
                    int i1, i0, io;
                    step_frames(D, kind, it, i1, i0, io);
                    WaveShot w;
                    w.out = frame_ptr(D, io);
                    w.tr = it % D.sr == 0 ? D.traces_t + (long long)(it / D.sr) * D.ntr : nullptr;
                    w.srcd = D.srcd[it];
                    s_shot[L & (WAVE_NB - 1)][q] = w;
                }
                if (lane == 0) {
                    WaveStep w;
                    int io;
                    step_frames(A, kind, it, w.i1, w.i0, io);
                    w.kind = kind;
                    w.it = it;
                    w.hess = kind == K_FWD1 && A.hessian && it % MST == 0;
                    w.sample = it % A.sr == 0;
                    s_step[L & (WAVE_NB - 1)] = w;
                }
                __syncwarp();  // lane 0's arrive below releases the whole warp's writes
            }
            const int st = j % NST;
            // the stage's previous item must be consumed (and is then published)
            if (j >= NST) {
                // suspend on the stage's barrier (the hardware wakes the thread when it completes)
                if (lane == 0 && done_l <= j - NST) mbar_try(smem_u32(&empty[st]), ((j - NST) / NST) & 1);
                const u64 t0 = global_ns();
                for (;;) {
                    publish(j, false);
                    if (done_l > j - NST) break;
                    if (expired(t0)) {
                        failed = true;
                        break;
                    }
                }
                if (failed) break;
            }
            // the neighbours' item (L-1, s); the counters seen last often cover it already
            bool fresh = false;
            if (Lr > 0) {
                const int need = (Lr - 1) * nr + s + 1;
                const u64 t0 = global_ns();
                for (;;) {
                    bool ok = nb == nullptr || seen >= need;
                    if (!ok) {
                        seen = ld_acquire(nb);
                        ok = seen >= need;
                        fresh = true;
                    }
                    if (__all_sync(0xffffffffu, ok)) break;
                    publish(j, true);
                    if (expired(t0)) {
                        failed = true;
                        break;
                    }
                }
                if (failed) break;
                fresh = __any_sync(0xffffffffu, fresh);
            }
            __syncwarp();  // the lanes' acquires precede lane 0's copies
            if (lane == 0) {
                // the copies read what the neighbours stored: after a new acquire, order them
                // behind it (copies after an earlier acquire are ordered by that one's fence)
                if (fresh) asm volatile("fence.proxy.async.global;" ::: "memory");
                const WaveStep &S = s_step[L & (WAVE_NB - 1)];
                const unsigned bar = smem_u32(&full[st]);
                mbar_arrive_expect(bar, Geo::P1_BYTES + Geo::P0_BYTES);
                unsigned char *stg = st_base + st * Geo::STAGE;
                tma_load4(smem_u32(stg), &tm_p1, 4 * (G0 - 1), X0 - 3, S.i1, cb + s - shot_base, bar);
                tma_load4(smem_u32(stg + Geo::P0_OFF), &tm_p0, 4 * G0, X0, S.i0, cb + s - shot_base, bar);
            }
            __syncwarp();
        }
        // publish the rest as the consumers finish, then let the copies in flight land
        if (!failed) {
            const u64 t0 = global_ns();
            for (;;) {
                publish(j, true);
                if (done_l >= j) break;
                if (expired(t0)) {
                    failed = true;
                    break;
                }
            }
        }
        if (failed && lane == 0) {
            atomicExch(err, 1);
            atomicExch(abort_w, 1);
        }
        if (lane == 0) {
            mbar_wait(smem_u32(&cfbar), 0);
            for (int q = max(0, j - NST); q < j; ++q) mbar_wait(smem_u32(&full[q % NST]), (q / NST) & 1);
        }
        return;
    }

    // ---------------------------------------------------------------- consumer warps
    const int zl = threadIdx.x, k = threadIdx.y;
    const int x = X0 + k;
    const bool xin = x < Nx, xint = x >= 3 && x <= Nx - 4;
    const int zlo = A.izStart, zhi = Nz - 4;
    const int fs_hi = min(2 * pml, pml + 3);  // last mirrored source row (no snapshots on this path)
    const bool xacc = x >= pml && x < pml + A.nxx;
    const bool fs_tile = A.fs && 4 * G0 <= fs_hi;
    const long long colx = (long long)x * A.ld;
    const float invdtdt = A.invdtdt;
    const PkConst K = make_pkconst(A.invdx, A.invdz, A.invdxdx, A.invdzdz, A.negzero);
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4(*scf)[TX][TG] = reinterpret_cast<const float4(*)[TX][TG]>(smem);
    const int gl = zl, g = G0 + gl, z0 = 4 * g;
    const bool zfd = z0 + 3 >= zlo && z0 <= zhi;
    const bool straddle = z0 < zlo || z0 + 3 > zhi;
    const bool live = g < G && xin;
    {
        const bool ok = mbar_wait(smem_u32(&cfbar), 0);
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) atomicExch(err, 1);
            return;
        }
    }
    const int z_t0 = 4 * G0, z_t1 = 4 * G0 + 4 * TG - 1;  // rows of this tile

    // the updated value of the lane's group for the item in stage sb; p0 its previous field
    auto value = [&](unsigned sb, const float4 &lo, const float4 &cq, const float4 &hi, float4 &p0) {
        p0 = lds4(sb + Geo::P0_OFF + (unsigned)(k * TG + gl) * 16u);
        float4 v = zero4;
        if (zfd && xint) {
            const unsigned xa = sb + (unsigned)((k + 3) * (TG + 2) + gl + 1) * 16u, cs = (TG + 2) * 16u;
            const float4 xn[6] = {lds4(xa - 3 * cs), lds4(xa - 2 * cs), lds4(xa - cs),
                                  lds4(xa + cs), lds4(xa + 2 * cs), lds4(xa + 3 * cs)};
            const float4 cf[6] = {scf[0][k][gl], scf[1][k][gl], scf[2][k][gl],
                                  scf[3][k][gl], scf[4][k][gl], scf[5][k][gl]};
            v = group2<MATH>(lo, cq, hi, xn, cf, p0, K);
            if (straddle) {
                if (z0 < zlo || z0 > zhi) v.x = 0.f;
                if (z0 + 1 < zlo || z0 + 1 > zhi) v.y = 0.f;
                if (z0 + 2 < zlo || z0 + 2 > zhi) v.z = 0.f;
                if (z0 + 3 < zlo || z0 + 3 > zhi) v.w = 0.f;
            }
        }
        return v;
    };

    for (int j = 0; j < total; ++j) {
        const int Lr = j / nr, s = j - Lr * nr, L = L0 + Lr;
        const int st = j % NST;
        const bool ok = mbar_wait(smem_u32(&full[st]), (j / NST) & 1);
        if (!__all_sync(0xffffffffu, ok)) {  // the warp gives up as one
            if (lane == 0) {
                atomicExch(err, 1);
                atomicExch(abort_w, 1);
            }
            break;
        }
        const WaveStep &S = s_step[L & (WAVE_NB - 1)];
        const WaveShot &W = s_shot[L & (WAVE_NB - 1)][s];
        const unsigned sb = smem_u32(st_base) + (unsigned)(st * Geo::STAGE);
        const unsigned wa = sb + (unsigned)((k + 3) * (TG + 2) + gl) * 16u;
        const float4 lo = lds4(wa), cq = lds4(wa + 16u), hi = lds4(wa + 32u);
        const int isx = s_isx[s], isz = s_isz[s];
        const bool src_t = isx >= X0 && isx < X0 + TX && isz >= z_t0 && isz <= z_t1;
        // receivers sample u(t) before the step
        if (S.sample && W.tr != nullptr && live) {
            const int code = s_rcv[s][k];
            if (code >= 0) {
                const int row = z_t0 + (code & 255);
                if (row >= z0 && row < z0 + 4) W.tr[code >> 8] = comp(cq, row - z0);
            } else if (code == -2) {
                const ShotDesc &D = shots[cb + s];
                for (int e = __ldg(D.colptr + x), e1 = __ldg(D.colptr + x + 1); e < e1; ++e) {
                    const int2 r = __ldg(D.rec + e);
                    if (r.x >= z0 && r.x < z0 + 4) W.tr[r.y] = comp(cq, r.x - z0);
                }
            }
        }
        if (!(fs_tile || S.hess || src_t)) {
            // ---- store-only epilogue
            if (live) {
                float4 p0;
                const float4 v = value(sb, lo, cq, hi, p0);
                *reinterpret_cast<float4 *>(W.out + colx + z0) = v;
            }
        } else if (live) {
            // above the free surface (rows < pml): never updated, stored or accumulated
            if (!(A.fs && z0 + 3 < pml)) {
                float4 p0;
                float4 v = value(sb, lo, cq, hi, p0);
                const long long col = colx + z0;
                const bool fs_top = A.fs && z0 <= fs_hi;
                const int jpml = (pml >= z0 && pml < z0 + 4) ? pml - z0 : -1;
                // the forward source enters before the free surface, in double
                if (x == isx && isz >= z0 && isz < z0 + 4)
                    setc(v, isz - z0, (float)__dadd_rn((double)comp(v, isz - z0), W.srcd));
                float4 mir = zero4;
                if (fs_top) {
                    if (jpml >= 0) setc(v, jpml, -0.0f);
                    mir = make_float4(-v.x, -v.y, -v.z, -v.w);
                }
                if (S.hess && xacc && z0 + 3 >= pml && z0 < pml + A.nz) {
                    double2 *acc = reinterpret_cast<double2 *>(s_H[s] + col);
                    double2 a0 = acc[0], a1 = acc[1];
                    double a[4] = {a0.x, a0.y, a1.x, a1.y};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int z = z0 + q;
                        if (z < pml || z >= pml + A.nz) continue;
                        const float t = fm(fa(fs_(comp(v, q), fm(2.0f, comp(cq, q))), comp(p0, q)), invdtdt);
                        a[q] = __dadd_rn(a[q], (double)fm(t, t));
                    }
                    acc[0] = make_double2(a[0], a[1]);
                    acc[1] = make_double2(a[2], a[3]);
                }
                float *out = W.out;
                if (!fs_top || z0 >= pml) {
                    *reinterpret_cast<float4 *>(out + col) = v;
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (z0 + q >= pml) out[col + q] = comp(v, q);
                }
                if (fs_top) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int z = z0 + q;
                        if (z > pml && z <= fs_hi) out[colx + 2 * pml - z] = comp(mir, q);
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&empty[st]));
    }
}

}  // namespace fwi
