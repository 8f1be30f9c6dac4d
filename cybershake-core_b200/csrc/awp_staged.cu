/*
 * awp_staged.cu -- the two-sweep stepper with TMA-staged xy tiles (2.5D blocking).
 *
 * A thread block owns a 32 x 8 column tile of one component and marches up a
 * chunk of z levels.  A producer warp issues, for every level, TMA tile loads
 * (cp.async.bulk.tensor over 3D tensor maps of the padded volume) into a ring
 * of shared-memory slots ahead of the level being computed: stencil tiles
 * with a 4-column and 2-row halo, media tiles with the row below, and the
 * point-wise state as 32 x 8 tiles.  A "full" mbarrier per slot counts the
 * bytes in; the eight consumer warps release a slot through its "empty"
 * mbarrier.  Values needed only along the cell's own column (z neighbours)
 * travel in per-thread register queues, loaded one level ahead.  Results are
 * written with coalesced stores.  The bytes in flight per SM are set by the
 * ring depth, not by registers or resident warps.
 *
 * Work items (x tile, y tile, z chunk, component) are spread over a
 * persistent grid, one component after the other or the components of a
 * tile side by side (split_item).
 *
 * The per-cell arithmetic is the shared code of awp_stencil.cuh, evaluated in
 * the same order as the other steppers (bit-identical results).  FP32 media
 * only; memory variables FP32 or bf16.
 *
 * Every wait on an mbarrier is bounded (2 s of %globaltimer); on expiry the
 * block records AWP_KERR_TMA_WAIT in the error word and its warps leave; the
 * producer first waits (bounded again) for its own copies in flight.
 */
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/awp_sgt.h"
#include "awp_internal.h"
#include "awp_kernels.h"
#include "awp_stencil.cuh"

#define ST_X 32                      /* tile width: one warp along x            */
#define ST_Y 8                       /* tile rows                               */
#define ST_W 40                      /* staged row: 4 halo + 32 + 4 halo        */
#define ST_HR (ST_Y + 4)             /* stencil tile rows: 2 below, 2 above     */
#define ST_MR (ST_Y + 1)             /* media tile rows: 1 below                */
#define ST_VT (ST_W * ST_HR)         /* floats of a stencil tile (1920 B)       */
#define ST_MT (ST_W * ST_MR)         /* floats a media tile receives (1440 B)   */
#define ST_MP 384                    /* floats reserved per media tile (1536 B) */
#define ST_PT (ST_X * ST_Y)          /* floats of a point tile (no halo)        */

/* bound of every barrier wait (the solver's setting, 2 s by default) and the
 * test-only injection of AwpStepArgs::withhold */
struct AwpWait {
    unsigned long long ns;
    int withhold;
};
#define ST_VEL_D 3                   /* levels in flight, velocity sweep        */

struct AwpStagedVelMaps {
    CUtensorMap st[AWP_MAX_COMP][5]; /* xx yy xy xz yz, box 40 x 12           */
    CUtensorMap d1;                  /* box 40 x 9                             */
    CUtensorMap p[AWP_MAX_COMP][3];  /* u v w, box 32 x 8                      */
};
struct AwpStagedStrMaps {
    CUtensorMap v[AWP_MAX_COMP][3];  /* u v w, box 40 x 12                     */
    CUtensorMap med[4];              /* lam mu qp qs, box 40 x 9               */
    CUtensorMap s[AWP_MAX_COMP][6];  /* xx yy zz xy xz yz, box 32 x 8          */
    CUtensorMap r[AWP_MAX_COMP][6];  /* r1..r6 (FP32, bf16 or int16), box 32 x 8 */
    CUtensorMap rx[AWP_MAX_COMP];    /* exponent words of block floating point r */
};
struct AwpStaged {
    AwpStagedVelMaps vm;
    AwpStagedStrMaps sm;
};

/* The kernels live in an anonymous namespace: this file is compiled twice,
 * without (the bit-exact stepper) and with multiply-add contraction
 * (AWP_STAGED_FMA: AWP_KERNEL_STAGED_FMA), and the two sets must not merge. */
namespace {

/* ------------------------------------------------------------------ */
/* mbarrier / TMA primitives (PTX ISA: mbarrier, cp.async.bulk.tensor) */
/* ------------------------------------------------------------------ */

__device__ __forceinline__ uint32_t s_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mb_init(uint64_t *b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_addr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mb_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mb_expect(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_addr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mb_try(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(s_addr(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* true once the phase of the given parity has completed; false after the bound */
__device__ __forceinline__ bool mb_wait(uint64_t *b, uint32_t parity, uint64_t limit_ns)
{
    if (mb_try(b, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t n = 0; n < (1u << 26); ++n) {
        if (mb_try(b, parity)) return true;
        if ((n & 63) == 63 && global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

/* generic-proxy accesses to a slot are ordered before the async-proxy refill */
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tma_3d(void *dst, const CUtensorMap *map, uint64_t *b, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(s_addr(dst)),
                 "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(s_addr(b))
                 : "memory");
}

/* memory coordinates of a tile: column of cell i0 - 4 (a multiple of 4, so
 * the copy starts on a 16-byte boundary), row of cell j0 - 2 (stencil) or
 * j0 - 1 (media), level k */
__device__ __forceinline__ int tile_x(int i0) { return i0 + AWP_XO - 1 - 4; }

/* component q and tile item t of work item `item`: the components of one
 * tile side by side (qslow = 0; their common media tiles come from L2) or one
 * component over all tiles at a time (qslow = 1; fewer arrays streamed at once) */
__device__ __forceinline__ void split_item(int item, int ncomp, int ntile, int qslow, int &q, int &t)
{
    if (qslow) {
        q = item / ntile;
        t = item - q * ntile;
    } else {
        q = item % ncomp;
        t = item / ncomp;
    }
}

__device__ __forceinline__ float *pick(const AwpCompSet<AWP_MAX_COMP> &cs, int q, int f)
{
    return q == 0 ? cs.c[0].f[f] : (q == 1 ? cs.c[1].f[f] : cs.c[2].f[f]);
}

/* ------------------------------------------------------------------ */
/* warp roles and the ring                                             */
/* ------------------------------------------------------------------ */

/* Eight consumer warps (one tile row each) and one producer warp whose lane
 * 0 issues the copies.  Ring slot s has a "full" barrier (the producer's
 * expect_tx arrival plus the bytes) and an "empty" barrier (one arrival per
 * consumer warp once it is done with the slot's level); the producer refills
 * a slot only after its empty phase completes, so no block-wide barrier
 * stands in the level loop and warps drift within the ring depth. */
#define ST_CW 8
#define ST_THREADS (32 * (ST_CW + 1))

__device__ __forceinline__ void mb_arrive(uint64_t *b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s_addr(b)) : "memory");
}

/* bounded wait that also gives up once another thread has flagged an abort */
__device__ __forceinline__ bool mb_wait_or_abort(uint64_t *b, uint32_t parity, const volatile int *abort,
                                                 uint64_t limit_ns)
{
    if (mb_try(b, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t n = 0; n < (1u << 26); ++n) {
        if (mb_try(b, parity)) return true;
        if ((n & 63) == 63 && (*abort || global_ns() - t0 > limit_ns)) return false;
    }
    return false;
}

/* the ring starts at the first 128-byte boundary of the dynamic shared
 * memory; the pad is added to the shared pointer itself (no round trip
 * through an integer), so the compiler keeps knowing the ring is shared
 * memory and reads its tiles with shared-memory loads, not generic ones */
__device__ __forceinline__ float *ring_base(unsigned char *raw)
{
    const unsigned pad = (unsigned)(-(uintptr_t)raw) & 127u;
    return (float *)(raw + pad);
}

/* GL: the same address through an integer, so that the compiler reads the
 * ring with generic loads.  On the 1400 x 1000 x 400 workload (78 GB of
 * state, one component per work item) the sweeps ran faster that way:
 * 28.7 against 24.4 Gcell-updates/s on one box, velocity sweep 12.3 against
 * 14.3 ms and stress sweep 26.1 against 31.6 ms per launch, while on the 6.4
 * and 14.7 GB workloads shared-memory loads are 5-8 % faster.  The cause is
 * not known; the solver picks GL above 32 GiB of state (AWP_TUNE_GENERIC). */
template <bool GL>
__device__ __forceinline__ float *ring_base_t(unsigned char *raw)
{
    if (GL) return (float *)(((uintptr_t)raw + 127) & ~(uintptr_t)127);
    return ring_base(raw);
}

template <int S>
__device__ __forceinline__ void ring_init(uint64_t *full, uint64_t *empty, volatile int *abort, int consumers = ST_CW)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < S; ++s) {
            mb_init(&full[s], 1);
            mb_init(&empty[s], consumers);
        }
        mb_fence_init();
        *abort = 0;
    }
    __syncthreads();
}

/* the producer's last act: the most recent use of every slot has landed, so
 * no copy into this block's shared memory is still in flight when it exits
 * (`skip`: a use it issued nothing for) */
template <int S>
__device__ __forceinline__ void ring_drain(uint64_t *full, uint32_t uses, uint64_t limit_ns, uint32_t skip = 0xffffffffu)
{
    for (uint32_t u = uses > (uint32_t)S ? uses - S : 0; u < uses; ++u)
        if (u != skip && !mb_wait(&full[u % S], (u / S) & 1, limit_ns)) return;
}

/* the ring use block 0's producer withholds under the test injection */
__device__ __forceinline__ uint32_t withheld_use(const AwpWait &wt)
{
    return blockIdx.x == 0 && wt.withhold >= 0 ? (uint32_t)wt.withhold : 0xffffffffu;
}

/* producer: wait until use `use` of its slot may be refilled */
template <int S>
__device__ __forceinline__ bool ring_acquire(uint64_t *empty, uint32_t use, const volatile int *abort,
                                             uint64_t limit_ns)
{
    return use < (uint32_t)S || mb_wait_or_abort(&empty[use % S], ((use / S) - 1) & 1, abort, limit_ns);
}

/* ------------------------------------------------------------------ */
/* velocity sweep                                                      */
/* ------------------------------------------------------------------ */

/* slot layout: xx yy xy xz yz stencil tiles, the d1 media tile, then the
 * u v w point tiles */
#define VEL_PT (5 * ST_VT + ST_MP)
#define VEL_SLOT (VEL_PT + 3 * ST_PT)
#define VEL_TXB ((5 * ST_VT + ST_MT + 3 * ST_PT) * 4)

/* stresses of plane k from the slot (in-plane) and from the register queue (z) */
struct TStr {
    const float *t; /* slot + cell offset */
    float xz_m2, xz_m1, xz_p1, yz_m2, yz_m1, yz_p1, zz_m1, zz_0, zz_p1, zz_p2;
    __device__ __forceinline__ float s(int a, int dx, int dy, int dz) const
    {
        if (a == S_ZZ) return dz == -1 ? zz_m1 : (dz == 0 ? zz_0 : (dz == 1 ? zz_p1 : zz_p2));
        if (dz == 0) {
            const int n = a == S_XX ? 0 : (a == S_YY ? 1 : (a == S_XY ? 2 : (a == S_XZ ? 3 : 4)));
            return t[n * ST_VT + dy * ST_W + dx];
        }
        if (a == S_XZ) return dz == -2 ? xz_m2 : (dz == -1 ? xz_m1 : xz_p1);
        return dz == -2 ? yz_m2 : (dz == -1 ? yz_m1 : yz_p1);
    }
};

template <int S>
__device__ __forceinline__ void vel_issue(const CUtensorMap *ms, const CUtensorMap *md1, const CUtensorMap *mp,
                                          float *ring, uint64_t *full, uint32_t use, int i0, int j0, int k)
{
    float *sl = ring + (use % S) * VEL_SLOT;
    uint64_t *b = &full[use % S];
    fence_async_smem();
    mb_expect(b, VEL_TXB);
    const int x = tile_x(i0);
#pragma unroll
    for (int a = 0; a < 5; ++a) tma_3d(sl + a * ST_VT, ms + a, b, x, j0 - 1, k + 1);
    tma_3d(sl + 5 * ST_VT, md1, b, x, j0, k + 1);
#pragma unroll
    for (int a = 0; a < 3; ++a) tma_3d(sl + VEL_PT + a * ST_PT, mp + a, b, i0 + AWP_XO - 1, j0 + 1, k + 1);
}

/* work items: (x tile, y tile, z chunk, component); see split_item for the order */
template <int D, int UNR, int RPT, bool GL = false>
__global__ void __launch_bounds__(32 * (ST_Y / RPT + 1), 3)
k_vel_tma(const __grid_constant__ AwpStagedVelMaps maps, AwpGeom g, AwpCompSet<AWP_MAX_COMP> cs, int ncomp, int qslow,
          const float *__restrict__ d1, const float *__restrict__ cx, const float *__restrict__ cy,
          const float *__restrict__ cz, float dth, AwpWork w, int *err, AwpWait wt)
{
    constexpr int S = 1 + D;          /* level k in use, D in flight */
    constexpr int CW = ST_Y / RPT;    /* consumer warps */
    extern __shared__ unsigned char st_smem[];
    float *ring = ring_base_t<GL>(st_smem);
    uint64_t *full = (uint64_t *)(ring + S * VEL_SLOT), *empty = full + S;
    __shared__ volatile int abort_s;
    ring_init<S>(full, empty, &abort_s, CW);
    const int tx = threadIdx.x, ty = threadIdx.y;

    if (ty == CW) {                   /* producer warp */
        if (tx != 0) return;
        uint32_t use = 0;
        bool ok = true;
        for (int item = blockIdx.x; ok && item < w.nitems; item += gridDim.x) {
            int q, t;
            split_item(item, ncomp, w.nitems / ncomp, qslow, q, t);
            int bx, by, k0, k1;
            work_item(g, w, t, bx, by, k0, k1);
            for (int k = k0; k <= k1; ++k, ++use) {
                ok = ring_acquire<S>(empty, use, &abort_s, wt.ns);
                if (!ok) break;
                vel_issue<S>(maps.st[q], &maps.d1, maps.p[q], ring, full, use, bx * ST_X + 1, by * ST_Y + 1, k);
            }
        }
        if (!ok) {
            abort_s = 1;
            atomicOr(err, AWP_KERR_TMA_WAIT);
        }
        ring_drain<S>(full, use, wt.ns);
        return;
    }

    const int sy = g.px, sz = g.plane;
    uint32_t use = 0;
    for (int item = blockIdx.x; item < w.nitems; item += gridDim.x) {
        int q, t;
        split_item(item, ncomp, w.nitems / ncomp, qslow, q, t);
        int bx, by, k0, k1;
        work_item(g, w, t, bx, by, k0, k1);
        const int i = bx * ST_X + 1 + tx;
        float *U = pick(cs, q, AF_U), *V = pick(cs, q, AF_V), *W = pick(cs, q, AF_W);
        const float *XZ = pick(cs, q, AF_XZ), *YZ = pick(cs, q, AF_YZ), *ZZ = pick(cs, q, AF_ZZ);
        /* per row: column queues, each loaded one level before it is needed */
        float xz_m2[RPT], xz_m1[RPT], xz_p1[RPT], yz_m2[RPT], yz_m1[RPT], yz_p1[RPT];
        float zz_m1[RPT], zz_0[RPT], zz_p1[RPT], zz_p2[RPT], dA[RPT], dB[RPT], dE[RPT], cxy[RPT];
        bool live[RPT];
        const int c0 = g.idx(i, by * ST_Y + 1 + ty, k0);
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int j = by * ST_Y + 1 + ty + r * CW, c = c0 + r * CW * sy;
            live[r] = i <= g.nx && j <= g.ny;
            xz_m2[r] = xz_m1[r] = xz_p1[r] = yz_m2[r] = yz_m1[r] = yz_p1[r] = 0.f;
            zz_m1[r] = zz_0[r] = zz_p1[r] = zz_p2[r] = dA[r] = dB[r] = dE[r] = cxy[r] = 0.f;
            if (live[r]) {
                xz_m2[r] = XZ[c - 2 * sz]; xz_m1[r] = XZ[c - sz]; xz_p1[r] = XZ[c + sz];
                yz_m2[r] = YZ[c - 2 * sz]; yz_m1[r] = YZ[c - sz]; yz_p1[r] = YZ[c + sz];
                zz_m1[r] = ZZ[c - sz]; zz_0[r] = ZZ[c]; zz_p1[r] = ZZ[c + sz]; zz_p2[r] = ZZ[c + 2 * sz];
                dA[r] = d1[c - sz]; dB[r] = d1[c - sy - sz]; dE[r] = d1[c + 1 - sz];
                cxy[r] = cx[i] * cy[j];
            }
        }
        int cc = c0;
#pragma unroll (UNR)
        for (int k = k0; k <= k1; ++k, cc += sz, ++use) {
            float xz_n[RPT], yz_n[RPT], zz_n[RPT];
            const float czk = cz[k];
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int c = cc + r * CW * sy;
                xz_n[r] = yz_n[r] = zz_n[r] = 0.f;
                if (live[r] && k < k1) { xz_n[r] = XZ[c + 2 * sz]; yz_n[r] = YZ[c + 2 * sz]; zz_n[r] = ZZ[c + 3 * sz]; }
            }
            /* warp-uniform outcome, so a warp leaves together or not at all */
            if (!__all_sync(0xffffffffu, mb_wait_or_abort(&full[use % S], (use / S) & 1, &abort_s, wt.ns))) {
                abort_s = 1;
                atomicOr(err, AWP_KERR_TMA_WAIT);
                return;
            }
            const float *sl = ring + (use % S) * VEL_SLOT;
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int row = ty + r * CW, c = cc + r * CW * sy;
                const int cv = (row + 2) * ST_W + tx + 4, cm = (row + 1) * ST_W + tx + 4, cp = row * ST_X + tx;
                if (live[r]) {
                    const float u0 = sl[VEL_PT + cp], v0 = sl[VEL_PT + ST_PT + cp], w0 = sl[VEL_PT + 2 * ST_PT + cp];
                    const float *t1 = sl + 5 * ST_VT + cm;
                    const float da = t1[0], db = t1[-ST_W], de = t1[1], dg = t1[1 - ST_W];
                    float fu, fv, fw;
                    vel_factors7(da, db, dA[r], dB[r], de, dE[r], dg, dth, fu, fv, fw);
                    const TStr A{sl + cv, xz_m2[r], xz_m1[r], xz_p1[r], yz_m2[r], yz_m1[r], yz_p1[r],
                                 zz_m1[r], zz_0[r], zz_p1[r], zz_p2[r]};
                    float u, v, w_;
                    vel_one_t(A, u0, v0, w0, fu, fv, fw, u, v, w_);
                    const float crj = cxy[r] * czk;
                    U[c] = u * crj;
                    V[c] = v * crj;
                    W[c] = w_ * crj;
                    xz_m2[r] = xz_m1[r]; xz_m1[r] = sl[3 * ST_VT + cv];
                    yz_m2[r] = yz_m1[r]; yz_m1[r] = sl[4 * ST_VT + cv];
                    zz_m1[r] = zz_0[r]; zz_0[r] = zz_p1[r]; zz_p1[r] = zz_p2[r]; zz_p2[r] = zz_n[r];
                    xz_p1[r] = xz_n[r]; yz_p1[r] = yz_n[r];
                    dA[r] = da; dB[r] = db; dE[r] = de;
                }
            }
            __syncwarp();
            if (tx == 0) mb_arrive(&empty[use % S]);
        }
    }
}

/* ---- velocity sweep, components side by side ---------------------------- */

/* One work item per (x tile, y tile, z chunk) for every component.  The d1
 * tile of a level comes once into a small ring of its own and the three
 * density factors of the cell are computed once for all components (plane
 * k-1 of d1 travels in registers); each component's stress stencil tiles and
 * u v w point tiles follow in a ring of sub-slots, one per (level,
 * component).  Column loads of the stresses are issued a full level before
 * they rotate in. */
#define VB_MS 3                                   /* d1 slots                */
#define VB_CPT (5 * ST_VT)                        /* first point tile        */
#define VB_CSLOT (VB_CPT + 3 * ST_PT)

template <int NCB, int CS>
__global__ void __launch_bounds__(ST_THREADS, 2)
k_vel_tmab(const __grid_constant__ AwpStagedVelMaps maps, AwpGeom g, AwpCompSet<AWP_MAX_COMP> cs,
           const float *__restrict__ d1, const float *__restrict__ cx, const float *__restrict__ cy,
           const float *__restrict__ cz, float dth, AwpWork w, int *err, AwpWait wt)
{
    extern __shared__ unsigned char st_smem[];
    float *mring = ring_base(st_smem);
    float *cring = mring + VB_MS * ST_MP;
    uint64_t *mfull = (uint64_t *)(cring + CS * VB_CSLOT), *mempty = mfull + VB_MS;
    uint64_t *cfull = mempty + VB_MS, *cempty = cfull + CS;
    __shared__ volatile int abort_s;
    __shared__ AwpComp tab[AWP_MAX_COMP];
    if (threadIdx.y == 0 && threadIdx.x < AWP_MAX_COMP) {
#pragma unroll
        for (int f = 0; f < AWP_NF_ARRAYS; ++f) tab[threadIdx.x].f[f] = pick(cs, threadIdx.x, f);
    }
    ring_init<VB_MS>(mfull, mempty, &abort_s, ST_CW);
    ring_init<CS>(cfull, cempty, &abort_s, ST_CW);
    const int tx = threadIdx.x, ty = threadIdx.y;

    if (ty == ST_CW) {                /* producer warp */
        if (tx != 0) return;
        uint32_t um = 0, uc = 0;
        bool ok = true;
        for (int item = blockIdx.x; ok && item < w.nitems; item += gridDim.x) {
            int bx, by, k0, k1;
            work_item(g, w, item, bx, by, k0, k1);
            const int i0 = bx * ST_X + 1, j0 = by * ST_Y + 1;
            const int x = tile_x(i0), xp = i0 + AWP_XO - 1;
            for (int k = k0; ok && k <= k1; ++k) {
                ok = ring_acquire<VB_MS>(mempty, um, &abort_s, wt.ns);
                if (!ok) break;
                {
                    float *sl = mring + (um % VB_MS) * ST_MP;
                    uint64_t *b = &mfull[um % VB_MS];
                    fence_async_smem();
                    mb_expect(b, ST_MT * 4);
                    tma_3d(sl, &maps.d1, b, x, j0, k + 1);
                }
                ++um;
#pragma unroll
                for (int q = 0; q < NCB; ++q) {
                    ok = ring_acquire<CS>(cempty, uc, &abort_s, wt.ns);
                    if (!ok) break;
                    float *sl = cring + (uc % CS) * VB_CSLOT;
                    uint64_t *b = &cfull[uc % CS];
                    fence_async_smem();
                    mb_expect(b, (5 * ST_VT + 3 * ST_PT) * 4);
#pragma unroll
                    for (int a = 0; a < 5; ++a) tma_3d(sl + a * ST_VT, &maps.st[q][a], b, x, j0 - 1, k + 1);
#pragma unroll
                    for (int a = 0; a < 3; ++a) tma_3d(sl + VB_CPT + a * ST_PT, &maps.p[q][a], b, xp, j0 + 1, k + 1);
                    ++uc;
                }
            }
        }
        if (!ok) {
            abort_s = 1;
            atomicOr(err, AWP_KERR_TMA_WAIT);
        }
        ring_drain<VB_MS>(mfull, um, wt.ns);
        ring_drain<CS>(cfull, uc, wt.ns);
        return;
    }

    const int sy = g.px, sz = g.plane;
    const int cv = (ty + 2) * ST_W + tx + 4, cm = (ty + 1) * ST_W + tx + 4, cp = ty * ST_X + tx;
    uint32_t um = 0, uc = 0;
    for (int item = blockIdx.x; item < w.nitems; item += gridDim.x) {
        int bx, by, k0, k1;
        work_item(g, w, item, bx, by, k0, k1);
        const int i = bx * ST_X + 1 + tx, j = by * ST_Y + 1 + ty;
        const bool live = i <= g.nx && j <= g.ny;
        const int c0 = g.idx(i, j, k0);
        /* per component: stresses along the column (xz, yz at k-2, k-1 from
         * earlier tiles, k+1 from the pending load; zz at k-1 .. k+2), the
         * pending loads one level ahead (pxz, pyz, pzz) */
        float xz_m2[NCB], xz_m1[NCB], xz_p1[NCB], yz_m2[NCB], yz_m1[NCB], yz_p1[NCB];
        float zz_m1[NCB], zz_0[NCB], zz_p1[NCB], zz_p2[NCB], pxz[NCB], pyz[NCB], pzz[NCB];
        float dA = 0.f, dB = 0.f, dE = 0.f;
#pragma unroll
        for (int q = 0; q < NCB; ++q) {
            xz_m2[q] = xz_m1[q] = xz_p1[q] = yz_m2[q] = yz_m1[q] = yz_p1[q] = 0.f;
            zz_m1[q] = zz_0[q] = zz_p1[q] = zz_p2[q] = pxz[q] = pyz[q] = pzz[q] = 0.f;
            if (live) {
                const float *XZ = tab[q].f[AF_XZ], *YZ = tab[q].f[AF_YZ], *ZZ = tab[q].f[AF_ZZ];
                xz_m2[q] = XZ[c0 - 2 * sz]; xz_m1[q] = XZ[c0 - sz]; pxz[q] = XZ[c0 + sz];
                yz_m2[q] = YZ[c0 - 2 * sz]; yz_m1[q] = YZ[c0 - sz]; pyz[q] = YZ[c0 + sz];
                zz_0[q] = ZZ[c0 - sz]; zz_p1[q] = ZZ[c0]; zz_p2[q] = ZZ[c0 + sz]; pzz[q] = ZZ[c0 + 2 * sz];
            }
        }
        if (live) {
            dA = d1[c0 - sz];
            dB = d1[c0 - sy - sz];
            dE = d1[c0 + 1 - sz];
        }
        const float cxy = live ? cx[i] * cy[j] : 0.f;
        int cc = c0;
#pragma unroll 1
        for (int k = k0; k <= k1; ++k, cc += sz, ++um) {
            const float czk = cz[k];
            if (!__all_sync(0xffffffffu, mb_wait_or_abort(&mfull[um % VB_MS], (um / VB_MS) & 1, &abort_s, wt.ns))) {
                abort_s = 1;
                atomicOr(err, AWP_KERR_TMA_WAIT);
                return;
            }
            float fu, fv, fw;
            {
                const float *t1 = mring + (um % VB_MS) * ST_MP + cm;
                const float da = t1[0], db = t1[-ST_W], de = t1[1], dg = t1[1 - ST_W];
                vel_factors7(da, db, dA, dB, de, dE, dg, dth, fu, fv, fw);
                dA = da; dB = db; dE = de;
            }
            __syncwarp();
            if (tx == 0) mb_arrive(&mempty[um % VB_MS]);
#pragma unroll
            for (int q = 0; q < NCB; ++q, ++uc) {
                zz_m1[q] = zz_0[q]; zz_0[q] = zz_p1[q]; zz_p1[q] = zz_p2[q]; zz_p2[q] = pzz[q];
                xz_p1[q] = pxz[q]; yz_p1[q] = pyz[q];
                pxz[q] = pyz[q] = pzz[q] = 0.f;
                if (live && k < k1) {
                    pxz[q] = tab[q].f[AF_XZ][cc + 2 * sz];
                    pyz[q] = tab[q].f[AF_YZ][cc + 2 * sz];
                    pzz[q] = tab[q].f[AF_ZZ][cc + 3 * sz];
                }
                if (!__all_sync(0xffffffffu, mb_wait_or_abort(&cfull[uc % CS], (uc / CS) & 1, &abort_s, wt.ns))) {
                    abort_s = 1;
                    atomicOr(err, AWP_KERR_TMA_WAIT);
                    return;
                }
                const float *sl = cring + (uc % CS) * VB_CSLOT;
                const float nxz = sl[3 * ST_VT + cv], nyz = sl[4 * ST_VT + cv];
                if (live) {
                    const float u0 = sl[VB_CPT + cp], v0 = sl[VB_CPT + ST_PT + cp], w0 = sl[VB_CPT + 2 * ST_PT + cp];
                    const TStr A{sl + cv, xz_m2[q], xz_m1[q], xz_p1[q], yz_m2[q], yz_m1[q], yz_p1[q],
                                 zz_m1[q], zz_0[q], zz_p1[q], zz_p2[q]};
                    float u, v, w_;
                    vel_one_t(A, u0, v0, w0, fu, fv, fw, u, v, w_);
                    const float crj = cxy * czk;
                    tab[q].f[AF_U][cc] = u * crj;
                    tab[q].f[AF_V][cc] = v * crj;
                    tab[q].f[AF_W][cc] = w_ * crj;
                }
                __syncwarp();
                if (tx == 0) mb_arrive(&cempty[uc % CS]);
                xz_m2[q] = xz_m1[q]; xz_m1[q] = nxz;
                yz_m2[q] = yz_m1[q]; yz_m1[q] = nyz;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* stress sweep                                                        */
/* ------------------------------------------------------------------ */

/* Slot layout (floats): u v w stencil tiles, lam mu qp qs media tiles, the
 * six stresses and the six memory variables of the tile (32 x 8 each; the
 * memory variables in their storage type).  Levels k-1 and k are in use
 * while level k+1 is in flight. */
#define STR_D 1
#define STR_ST (3 * ST_VT + 4 * ST_MP)           /* first stress tile        */
#define STR_SLOT (STR_ST + 12 * ST_PT)           /* r tiles fit in 6 x 256   */

/* media of planes k and k-1 at the cell */
/* the six stresses of a cell, times the sponge factor, to global memory
 * (the array pointers come from a shared-memory table) */
__device__ __forceinline__ void gst6(const AwpComp &o, int c, const Stress6 &s, float crj)
{
    __stwb(o.f[AF_XX] + c, s.xx * crj); __stwb(o.f[AF_YY] + c, s.yy * crj); __stwb(o.f[AF_ZZ] + c, s.zz * crj);
    __stwb(o.f[AF_XY] + c, s.xy * crj); __stwb(o.f[AF_XZ] + c, s.xz * crj); __stwb(o.f[AF_YZ] + c, s.yz * crj);
}

struct TMed {
    const float *p0, *pm; /* media tiles (lam first) of planes k and k-1, at the cell */
    __device__ __forceinline__ float m(int a, int dx, int dy, int dz) const
    {
        const int n = a == AM_LAM ? 0 : (a == AM_MU ? 1 : (a == AM_QP ? 2 : 3));
        return (dz == 0 ? p0 : pm)[n * ST_MP + dy * ST_W + dx];
    }
};

/* velocities: plane k from the slot, the column from registers */
struct TVel {
    const float *t;   /* u tile of plane k at the cell; v and w tiles follow */
    float um1, vm1, wm1, up1, up2, vp1, vp2, wm2, wp1;
    __device__ __forceinline__ float u(int dx, int dy, int dz) const
    {
        return dz == 0 ? t[dy * ST_W + dx] : (dz == -1 ? um1 : (dz == 1 ? up1 : up2));
    }
    __device__ __forceinline__ float v(int dx, int dy, int dz) const
    {
        return dz == 0 ? t[ST_VT + dy * ST_W + dx] : (dz == -1 ? vm1 : (dz == 1 ? vp1 : vp2));
    }
    __device__ __forceinline__ float w(int dx, int dy, int dz) const
    {
        return dz == 0 ? t[2 * ST_VT + dy * ST_W + dx] : (dz == -1 ? wm1 : (dz == -2 ? wm2 : wp1));
    }
};

/* the memory-variable tiles of a slot by storage type: element size, tile
 * count (block floating point adds the tile of exponent words) and the six
 * values of the cell at point-tile offset cp */
template <class TR>
struct RTile {
    static constexpr int size = (int)sizeof(TR), ntiles = 6;
    static __device__ __forceinline__ void ld(const unsigned char *base, int cp, float r[6])
    {
#pragma unroll
        for (int a = 0; a < 6; ++a) r[a] = Store<TR>::ld((const TR *)base + cp, a * ST_PT, 1.0f);
    }
};
template <>
struct RTile<RBfp> {
    static constexpr int size = 2, ntiles = 7;
    static __device__ __forceinline__ void ld(const unsigned char *base, int cp, float r[6])
    {
        bfp_load6((const short *)base + cp, ST_PT, ((const unsigned short *)base)[6 * ST_PT + cp], r);
    }
};

/* bytes one level brings in (rbytes: the r tiles of one cell row set) */
__host__ __device__ __forceinline__ uint32_t str_txb(int nve, int rtile_bytes)
{
    return (uint32_t)((3 * ST_VT + (nve == 1 ? 4 : 2) * ST_MT + 6 * ST_PT) * 4 + (nve == 1 ? rtile_bytes : 0));
}

/* issues the r tiles of component q at a point-tile position */
template <class TR>
__device__ __forceinline__ void r_issue(const AwpStagedStrMaps &maps, int q, unsigned char *rb, uint64_t *b, int xp,
                                        int y, int z)
{
#pragma unroll
    for (int a = 0; a < 6; ++a) tma_3d(rb + a * ST_PT * RTile<TR>::size, &maps.r[q][a], b, xp, y, z);
    if (RTile<TR>::ntiles == 7) tma_3d(rb + 6 * ST_PT * RTile<TR>::size, &maps.rx[q], b, xp, y, z);
}

template <int S, class TR>
__device__ __forceinline__ void str_issue(const AwpStagedStrMaps &maps, int q, int nve, float *ring, uint64_t *full,
                                          uint32_t use, int i0, int j0, int k)
{
    float *sl = ring + (use % S) * STR_SLOT;
    uint64_t *b = &full[use % S];
    fence_async_smem();
    mb_expect(b, str_txb(nve, RTile<TR>::ntiles * ST_PT * RTile<TR>::size));
    const int x = tile_x(i0);
#pragma unroll
    for (int a = 0; a < 3; ++a) tma_3d(sl + a * ST_VT, &maps.v[q][a], b, x, j0 - 1, k + 1);
    const int nmed = nve == 1 ? 4 : 2;
    for (int a = 0; a < nmed; ++a) tma_3d(sl + 3 * ST_VT + a * ST_MP, &maps.med[a], b, x, j0, k + 1);
    /* point tiles start at cell (i0, j0): memory column i0 + 7 (a multiple of 8) */
    const int xp = i0 + AWP_XO - 1;
#pragma unroll
    for (int a = 0; a < 6; ++a) tma_3d(sl + STR_ST + a * ST_PT, &maps.s[q][a], b, xp, j0 + 1, k + 1);
    if (nve == 1) r_issue<TR>(maps, q, (unsigned char *)(sl + STR_ST + 6 * ST_PT), b, xp, j0 + 1, k + 1);
}

/* work items: (x tile, y tile, z chunk, component); see split_item for the order.
 * RPT rows of the tile per consumer thread (ST_Y / RPT consumer warps): with
 * RPT = 2 a thread carries two independent cells per level. */
template <class TR, int UNR, int RPT, bool GL = false>
__global__ void __launch_bounds__(32 * (ST_Y / RPT + 1), 3)
k_str_tma(const __grid_constant__ AwpStagedStrMaps maps, AwpGeom g, AwpCompSet<AWP_MAX_COMP> cs, int ncomp, int qslow,
          const float *__restrict__ cx, const float *__restrict__ cy, const float *__restrict__ cz,
          const float *__restrict__ tau, float dth, float dt, float dh1, AwpWork w, int nve, int *err, AwpWait wt)
{
    constexpr int S = 2 + STR_D;      /* levels k-1 and k in use, STR_D in flight */
    constexpr int CW = ST_Y / RPT;    /* consumer warps */
    extern __shared__ unsigned char st_smem[];
    float *ring = ring_base_t<GL>(st_smem);
    uint64_t *full = (uint64_t *)(ring + S * STR_SLOT), *empty = full + S;
    __shared__ volatile int abort_s;
    __shared__ AwpComp tab[AWP_MAX_COMP];
    if (threadIdx.y == 0 && threadIdx.x < AWP_MAX_COMP) {
#pragma unroll
        for (int f = 0; f < AWP_NF_ARRAYS; ++f) tab[threadIdx.x].f[f] = pick(cs, threadIdx.x, f);
    }
    ring_init<S>(full, empty, &abort_s, CW);
    const int tx = threadIdx.x, ty = threadIdx.y;

    if (ty == CW) {                   /* producer warp */
        if (tx != 0) return;
        uint32_t use = 0;
        bool ok = true;
        for (int item = blockIdx.x; ok && item < w.nitems; item += gridDim.x) {
            int q, t;
            split_item(item, ncomp, w.nitems / ncomp, qslow, q, t);
            int bx, by, k0, k1;
            work_item(g, w, t, bx, by, k0, k1);
            for (int k = k0 - 1; k <= k1; ++k, ++use) {
                ok = ring_acquire<S>(empty, use, &abort_s, wt.ns);
                if (!ok) break;
                if (use == withheld_use(wt)) continue;   /* test injection: nothing issued, no arrival */
                str_issue<S, TR>(maps, q, nve, ring, full, use, bx * ST_X + 1, by * ST_Y + 1, k);
            }
        }
        if (!ok) {
            abort_s = 1;
            atomicOr(err, AWP_KERR_TMA_WAIT);
        }
        ring_drain<S>(full, use, wt.ns, withheld_use(wt));
        return;
    }

    const int sz = g.plane, sy = g.px;
    uint32_t use0 = 0;                /* ring use of the item's first level */
    for (int item = blockIdx.x; item < w.nitems; item += gridDim.x) {
        int q, t;
        split_item(item, ncomp, w.nitems / ncomp, qslow, q, t);
        int bx, by, k0, k1;
        work_item(g, w, t, bx, by, k0, k1);
        const int i = bx * ST_X + 1 + tx;
        const int np = k1 - k0 + 2;   /* levels k0-1 .. k1 */
        const float *U = tab[q].f[AF_U], *V = tab[q].f[AF_V], *W = tab[q].f[AF_W];
        /* per row: column queues u, v at k+1, k+2 (k+3 loaded one level ahead), w at k-2, k+1 (k+2 ahead) */
        float up1[RPT], up2[RPT], vp1[RPT], vp2[RPT], wm2[RPT], wp1[RPT], cxy[RPT];
        bool live[RPT];
        int itxy[RPT];
        const int c0 = g.idx(i, by * ST_Y + 1 + ty, k0);
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int j = by * ST_Y + 1 + ty + r * CW, c = c0 + r * CW * sy;
            live[r] = i <= g.nx && j <= g.ny;
            itxy[r] = ((j & 1) << 1) | (i & 1);
            up1[r] = up2[r] = vp1[r] = vp2[r] = wm2[r] = wp1[r] = cxy[r] = 0.f;
            if (live[r]) {
                up1[r] = __ldg(&U[c + sz]); up2[r] = __ldg(&U[c + 2 * sz]);
                vp1[r] = __ldg(&V[c + sz]); vp2[r] = __ldg(&V[c + 2 * sz]);
                wm2[r] = __ldg(&W[c - 2 * sz]); wp1[r] = __ldg(&W[c + sz]);
                cxy[r] = cx[i] * cy[j];
            }
        }
        int cc = c0;
#pragma unroll (UNR)
        for (int k = k0; k <= k1; ++k, cc += sz) {
            const uint32_t use = use0 + (uint32_t)(k - k0 + 1), usem = use - 1;
            float up3[RPT], vp3[RPT], wp2[RPT];
            const float czk = cz[k];
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int c = cc + r * CW * sy;
                up3[r] = vp3[r] = wp2[r] = 0.f;
                if (live[r] && k < k1) {
                    if (GL) { up3[r] = U[c + 3 * sz]; vp3[r] = V[c + 3 * sz]; wp2[r] = W[c + 2 * sz]; }
                    else { up3[r] = __ldg(&U[c + 3 * sz]); vp3[r] = __ldg(&V[c + 3 * sz]); wp2[r] = __ldg(&W[c + 2 * sz]); }
                }
            }
            bool ok = true;
            if (k == k0) ok = mb_wait_or_abort(&full[usem % S], (usem / S) & 1, &abort_s, wt.ns);
            if (ok) ok = mb_wait_or_abort(&full[use % S], (use / S) & 1, &abort_s, wt.ns);
            if (!__all_sync(0xffffffffu, ok)) {   /* warp-uniform outcome */
                abort_s = 1;
                atomicOr(err, AWP_KERR_TMA_WAIT);
                return;
            }
            const float *sk = ring + (use % S) * STR_SLOT, *sm = ring + (usem % S) * STR_SLOT;
            const int ipar = ((g.nz + 1 - k) & 1) << 2;                    /* viscoop.f:93-101 */
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int row = ty + r * CW, c = cc + r * CW * sy;
                const int cv = (row + 2) * ST_W + tx + 4, cm = (row + 1) * ST_W + tx + 4, cp = row * ST_X + tx;
                const float wm1 = sm[2 * ST_VT + cv];
                if (live[r]) {
                    const int it = ipar | itxy[r];
                    const TMed M{sk + 3 * ST_VT + cm, sm + 3 * ST_VT + cm};
                    const StrCoef kc = str_coef_t(M, nve, tau[it], tau[8 + it]);
                    const float *ps = sk + STR_ST + cp;
                    const Stress6 s0{ps[0], ps[ST_PT], ps[2 * ST_PT], ps[3 * ST_PT], ps[4 * ST_PT], ps[5 * ST_PT]};
                    const TVel Vq{sk + cv, sm[cv], sm[ST_VT + cv], wm1, up1[r], up2[r], vp1[r], vp2[r], wm2[r], wp1[r]};
                    Stress6 o;
                    if (nve == 1) {
                        float rr[6];
                        RTile<TR>::ld((const unsigned char *)(sk + STR_ST + 6 * ST_PT), cp, rr);
                        const VelDiff dd = vel_diff(Vq);
                        o = str_visco(kc, dd, s0, rr, dth, dt, dh1);
                        RVars<TR>::st(tab[q], c, rr);
                    } else {
                        o = str_elastic(kc, Vq, s0, dth);
                    }
                    const float crj = cxy[r] * czk;
                    if (GL) {
                        tab[q].f[AF_XX][c] = o.xx * crj; tab[q].f[AF_YY][c] = o.yy * crj; tab[q].f[AF_ZZ][c] = o.zz * crj;
                        tab[q].f[AF_XY][c] = o.xy * crj; tab[q].f[AF_XZ][c] = o.xz * crj; tab[q].f[AF_YZ][c] = o.yz * crj;
                    } else {
                        gst6(tab[q], c, o, crj);
                    }
                }
                up1[r] = up2[r]; up2[r] = up3[r];
                vp1[r] = vp2[r]; vp2[r] = vp3[r];
                wm2[r] = wm1; wp1[r] = wp2[r];
            }
            __syncwarp();
            if (tx == 0) mb_arrive(&empty[usem % S]);
        }
        __syncwarp();
        if (tx == 0) mb_arrive(&empty[(use0 + np - 1) % S]);
        use0 += np;
        if (k1 == g.nz) {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                if (!live[r]) continue;
                /* fstr (operator.f:594-606) on this thread's own column; the top
                 * chunk holds at least levels nz-2..nz, all written by this thread */
                const int ct = g.idx(i, by * ST_Y + 1 + ty + r * CW, g.nz);
                float *ZZ = tab[q].f[AF_ZZ], *XZ = tab[q].f[AF_XZ], *YZ = tab[q].f[AF_YZ];
                ZZ[ct + sz] = -__ldcg(&ZZ[ct]);
                ZZ[ct + 2 * sz] = -__ldcg(&ZZ[ct - sz]);
                XZ[ct + sz] = -__ldcg(&XZ[ct - sz]);
                XZ[ct + 2 * sz] = -__ldcg(&XZ[ct - 2 * sz]);
                YZ[ct + sz] = -__ldcg(&YZ[ct - sz]);
                YZ[ct + 2 * sz] = -__ldcg(&YZ[ct - 2 * sz]);
                XZ[ct] = 0.0f;
                YZ[ct] = 0.0f;
            }
        }
    }
}

/* ---- components side by side in one work item -------------------------- */

/* A work item is (x tile, y tile, z chunk) with every component.  The media
 * tiles of a level, and the cell coefficients computed from them (the 8-cell
 * sums and the five divisions), serve all components: the media ring (levels
 * k-1 and k in use, k+1 in flight) is filled once per level.  The components'
 * tiles follow in a ring of their own, one sub-slot per (level, component);
 * a component's plane k-1 values at the cell (u, v, w) travel in registers,
 * so a sub-slot is released as soon as its level is done. */
#define STB_MS 3                                  /* media slots              */
#define STB_MSLOT (4 * ST_MP)
#define STB_CST (3 * ST_VT)                       /* first stress tile        */
#define STB_CSLOT (STB_CST + 12 * ST_PT)          /* r tiles fit in 6 x 256   */

__host__ __device__ __forceinline__ uint32_t strb_med_txb(int nve) { return (uint32_t)((nve == 1 ? 4 : 2) * ST_MT * 4); }
__host__ __device__ __forceinline__ uint32_t strb_comp_txb(int nve, int rtile_bytes)
{
    return (uint32_t)((3 * ST_VT + 6 * ST_PT) * 4 + (nve == 1 ? rtile_bytes : 0));
}

/* RPT tile rows per consumer thread (ST_Y / RPT consumer warps) */
template <class TR, int NCB, int STB_CS, int RPT>
__global__ void __launch_bounds__(32 * (ST_Y / RPT + 1), 2)
k_str_tmab(const __grid_constant__ AwpStagedStrMaps maps, AwpGeom g, AwpCompSet<AWP_MAX_COMP> cs,
           const float *__restrict__ cx, const float *__restrict__ cy, const float *__restrict__ cz,
           const float *__restrict__ tau, float dth, float dt, float dh1, AwpWork w, int nve, int *err, AwpWait wt)
{
    constexpr int CW = ST_Y / RPT;    /* consumer warps */
    extern __shared__ unsigned char st_smem[];
    float *mring = ring_base(st_smem);
    float *cring = mring + STB_MS * STB_MSLOT;
    uint64_t *mfull = (uint64_t *)(cring + STB_CS * STB_CSLOT), *mempty = mfull + STB_MS;
    uint64_t *cfull = mempty + STB_MS, *cempty = cfull + STB_CS;
    __shared__ volatile int abort_s;
    __shared__ AwpComp tab[AWP_MAX_COMP];
    if (threadIdx.y == 0 && threadIdx.x < AWP_MAX_COMP) {
#pragma unroll
        for (int f = 0; f < AWP_NF_ARRAYS; ++f) tab[threadIdx.x].f[f] = pick(cs, threadIdx.x, f);
    }
    ring_init<STB_MS>(mfull, mempty, &abort_s, CW);
    ring_init<STB_CS>(cfull, cempty, &abort_s, CW);
    const int tx = threadIdx.x, ty = threadIdx.y;

    if (ty == CW) {                   /* producer warp */
        if (tx != 0) return;
        uint32_t um = 0, uc = 0;
        bool ok = true;
        const int nmed = nve == 1 ? 4 : 2;
        for (int item = blockIdx.x; ok && item < w.nitems; item += gridDim.x) {
            int bx, by, k0, k1;
            work_item(g, w, item, bx, by, k0, k1);
            const int i0 = bx * ST_X + 1, j0 = by * ST_Y + 1;
            const int x = tile_x(i0), xp = i0 + AWP_XO - 1;
            for (int k = k0 - 1; ok && k <= k1; ++k) {
                ok = ring_acquire<STB_MS>(mempty, um, &abort_s, wt.ns);
                if (!ok) break;
                if (um != withheld_use(wt)) {                 /* test injection: nothing issued, no arrival */
                    float *sl = mring + (um % STB_MS) * STB_MSLOT;
                    uint64_t *b = &mfull[um % STB_MS];
                    fence_async_smem();
                    mb_expect(b, strb_med_txb(nve));
                    for (int a = 0; a < nmed; ++a) tma_3d(sl + a * ST_MP, &maps.med[a], b, x, j0, k + 1);
                }
                ++um;
                if (k < k0) continue;
#pragma unroll
                for (int q = 0; q < NCB; ++q) {
                    ok = ring_acquire<STB_CS>(cempty, uc, &abort_s, wt.ns);
                    if (!ok) break;
                    float *sl = cring + (uc % STB_CS) * STB_CSLOT;
                    uint64_t *b = &cfull[uc % STB_CS];
                    fence_async_smem();
                    mb_expect(b, strb_comp_txb(nve, RTile<TR>::ntiles * ST_PT * RTile<TR>::size));
#pragma unroll
                    for (int a = 0; a < 3; ++a) tma_3d(sl + a * ST_VT, &maps.v[q][a], b, x, j0 - 1, k + 1);
#pragma unroll
                    for (int a = 0; a < 6; ++a) tma_3d(sl + STB_CST + a * ST_PT, &maps.s[q][a], b, xp, j0 + 1, k + 1);
                    if (nve == 1) r_issue<TR>(maps, q, (unsigned char *)(sl + STB_CST + 6 * ST_PT), b, xp, j0 + 1, k + 1);
                    ++uc;
                }
            }
        }
        if (!ok) {
            abort_s = 1;
            atomicOr(err, AWP_KERR_TMA_WAIT);
        }
        ring_drain<STB_MS>(mfull, um, wt.ns, withheld_use(wt));
        ring_drain<STB_CS>(cfull, uc, wt.ns);
        return;
    }

    const int sz = g.plane, sy = g.px;
    uint32_t um0 = 0, uc = 0;         /* media use of the item's level k0 - 1; next component use */
    for (int item = blockIdx.x; item < w.nitems; item += gridDim.x) {
        int bx, by, k0, k1;
        work_item(g, w, item, bx, by, k0, k1);
        const int i = bx * ST_X + 1 + tx;
        const int c0 = g.idx(i, by * ST_Y + 1 + ty, k0);
        /* per row and component: column queues u, v at k+1, k+2 and w at k+1,
         * fed by loads one level ahead (pu, pv, pw) that rotate in when the
         * component comes up at the next level, a full level after their
         * issue; w at k-2, k-1 and u, v at k-1 come from earlier tiles */
        float up1[RPT][NCB], up2[RPT][NCB], pu[RPT][NCB], vp1[RPT][NCB], vp2[RPT][NCB], pv[RPT][NCB];
        float wp1[RPT][NCB], pw[RPT][NCB], wm2[RPT][NCB], wm1[RPT][NCB], um1[RPT][NCB], vm1[RPT][NCB];
        bool live[RPT];
        int itxy[RPT];
        float cxy[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int j = by * ST_Y + 1 + ty + r * CW, c = c0 + r * CW * sy;
            live[r] = i <= g.nx && j <= g.ny;
            itxy[r] = ((j & 1) << 1) | (i & 1);
            cxy[r] = live[r] ? cx[i] * cy[j] : 0.f;
#pragma unroll
            for (int q = 0; q < NCB; ++q) {
                up1[r][q] = up2[r][q] = pu[r][q] = vp1[r][q] = vp2[r][q] = pv[r][q] = wp1[r][q] = pw[r][q] = 0.f;
                wm2[r][q] = wm1[r][q] = um1[r][q] = vm1[r][q] = 0.f;
                if (live[r]) {
                    const float *U = tab[q].f[AF_U], *V = tab[q].f[AF_V], *W = tab[q].f[AF_W];
                    up2[r][q] = __ldg(&U[c + sz]); pu[r][q] = __ldg(&U[c + 2 * sz]);
                    vp2[r][q] = __ldg(&V[c + sz]); pv[r][q] = __ldg(&V[c + 2 * sz]);
                    pw[r][q] = __ldg(&W[c + sz]);
                    wm2[r][q] = __ldg(&W[c - 2 * sz]); wm1[r][q] = __ldg(&W[c - sz]);
                    um1[r][q] = __ldg(&U[c - sz]); vm1[r][q] = __ldg(&V[c - sz]);
                }
            }
        }
        int cc = c0;
#pragma unroll 1
        for (int k = k0; k <= k1; ++k, cc += sz) {
            const uint32_t mk = um0 + (uint32_t)(k - k0 + 1), mm = mk - 1;
            const float czk = cz[k];
            bool ok = true;
            if (k == k0) ok = mb_wait_or_abort(&mfull[mm % STB_MS], (mm / STB_MS) & 1, &abort_s, wt.ns);
            if (ok) ok = mb_wait_or_abort(&mfull[mk % STB_MS], (mk / STB_MS) & 1, &abort_s, wt.ns);
            if (!__all_sync(0xffffffffu, ok)) {   /* warp-uniform outcome */
                abort_s = 1;
                atomicOr(err, AWP_KERR_TMA_WAIT);
                return;
            }
            const int ipar = ((g.nz + 1 - k) & 1) << 2;                        /* viscoop.f:93-101 */
            StrCoef kc[RPT];
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int cm = (ty + r * CW + 1) * ST_W + tx + 4;
                const int it = ipar | itxy[r];
                const TMed M{mring + (mk % STB_MS) * STB_MSLOT + cm, mring + (mm % STB_MS) * STB_MSLOT + cm};
                kc[r] = str_coef_t(M, nve, tau[it], tau[8 + it]);
            }
            __syncwarp();
            if (tx == 0) mb_arrive(&mempty[mm % STB_MS]);
#pragma unroll
            for (int q = 0; q < NCB; ++q, ++uc) {
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    /* rotate this component's queues, then load one level ahead */
                    const int c = cc + r * CW * sy;
                    up1[r][q] = up2[r][q]; up2[r][q] = pu[r][q];
                    vp1[r][q] = vp2[r][q]; vp2[r][q] = pv[r][q];
                    wp1[r][q] = pw[r][q];
                    pu[r][q] = pv[r][q] = pw[r][q] = 0.f;
                    if (live[r] && k < k1) {
                        pu[r][q] = __ldg(&tab[q].f[AF_U][c + 3 * sz]);
                        pv[r][q] = __ldg(&tab[q].f[AF_V][c + 3 * sz]);
                        pw[r][q] = __ldg(&tab[q].f[AF_W][c + 2 * sz]);
                    }
                }
                ok = mb_wait_or_abort(&cfull[uc % STB_CS], (uc / STB_CS) & 1, &abort_s, wt.ns);
                if (!__all_sync(0xffffffffu, ok)) {
                    abort_s = 1;
                    atomicOr(err, AWP_KERR_TMA_WAIT);
                    return;
                }
                const float *sk = cring + (uc % STB_CS) * STB_CSLOT;
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    const int row = ty + r * CW, c = cc + r * CW * sy;
                    const int cv = (row + 2) * ST_W + tx + 4, cp = row * ST_X + tx;
                    const float nu = sk[cv], nv = sk[ST_VT + cv], nw = sk[2 * ST_VT + cv];
                    if (live[r]) {
                        const float *ps = sk + STB_CST + cp;
                        const Stress6 s0{ps[0], ps[ST_PT], ps[2 * ST_PT], ps[3 * ST_PT], ps[4 * ST_PT], ps[5 * ST_PT]};
                        const TVel Vq{sk + cv, um1[r][q], vm1[r][q], wm1[r][q], up1[r][q], up2[r][q], vp1[r][q],
                                      vp2[r][q], wm2[r][q], wp1[r][q]};
                        Stress6 o;
                        if (nve == 1) {
                            float rr[6];
                            RTile<TR>::ld((const unsigned char *)(sk + STB_CST + 6 * ST_PT), cp, rr);
                            const VelDiff dd = vel_diff(Vq);
                            o = str_visco(kc[r], dd, s0, rr, dth, dt, dh1);
                            RVars<TR>::st(tab[q], c, rr);
                        } else {
                            o = str_elastic(kc[r], Vq, s0, dth);
                        }
                        const float crj = cxy[r] * czk;
                        gst6(tab[q], c, o, crj);
                    }
                    wm2[r][q] = wm1[r][q];
                    um1[r][q] = nu; vm1[r][q] = nv; wm1[r][q] = nw;
                }
                __syncwarp();
                if (tx == 0) mb_arrive(&cempty[uc % STB_CS]);
            }
        }
        __syncwarp();
        if (tx == 0) mb_arrive(&mempty[(um0 + (uint32_t)(k1 - k0 + 1)) % STB_MS]);
        um0 += (uint32_t)(k1 - k0 + 2);
        if (k1 == g.nz) {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                if (!live[r]) continue;
#pragma unroll
                for (int q = 0; q < NCB; ++q) {
                    /* fstr (operator.f:594-606) on this thread's own column */
                    const int ct = g.idx(i, by * ST_Y + 1 + ty + r * CW, g.nz);
                    float *ZZ = tab[q].f[AF_ZZ], *XZ = tab[q].f[AF_XZ], *YZ = tab[q].f[AF_YZ];
                    ZZ[ct + sz] = -__ldcg(&ZZ[ct]);
                    ZZ[ct + 2 * sz] = -__ldcg(&ZZ[ct - sz]);
                    XZ[ct + sz] = -__ldcg(&XZ[ct - sz]);
                    XZ[ct + 2 * sz] = -__ldcg(&XZ[ct - 2 * sz]);
                    YZ[ct + sz] = -__ldcg(&YZ[ct - sz]);
                    YZ[ct + 2 * sz] = -__ldcg(&YZ[ct - 2 * sz]);
                    XZ[ct] = 0.0f;
                    YZ[ct] = 0.0f;
                }
            }
        }
    }
}

}  // namespace

/* ------------------------------------------------------------------ */
/* host side                                                           */
/* ------------------------------------------------------------------ */

#ifdef AWP_STAGED_FMA
#define AWP_STAGED_ENTRY(name) name##_fma
#else
#define AWP_STAGED_ENTRY(name) name
#endif

#ifndef AWP_STAGED_FMA
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = NULL;
    if (!fn) {
        void *p = NULL;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) == cudaSuccess &&
            qr == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

/* tensor map of one padded volume (pitch, ny + 4, nz + 4) of 4- or 2-byte
 * elements, box w x rows x 1 */
static bool make_map(CUtensorMap *m, const AwpGeom &g, const void *base, int w, int rows, int esize = 4)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn || !base || ((uintptr_t)base & 15) || (g.px * esize) % 16 || (w * esize) % 16) return false;
    const cuuint64_t dim[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.nz + 4};
    const cuuint64_t stride[2] = {(cuuint64_t)g.px * esize, (cuuint64_t)g.plane * esize};
    const cuuint32_t box[3] = {(cuuint32_t)w, (cuuint32_t)rows, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUtensorMapDataType t = esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    return fn(m, t, 3, (void *)base, dim, stride, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t awp_staged_create(AwpStaged **out, const AwpGeom &g, int ncomp, const AwpComp *comp, const AwpMediaT &md,
                              int rtype)
{
    *out = NULL;
    if (md.type != AWP_STORE_F32 || ncomp < 1 || ncomp > AWP_MAX_COMP) return cudaErrorInvalidValue;
    if (g.px % 8 != 0) return cudaErrorInvalidValue;
    AwpStaged *s = (AwpStaged *)aligned_alloc(64, sizeof(AwpStaged));
    if (!s) return cudaErrorMemoryAllocation;
    memset(s, 0, sizeof *s);
    static const int vel_f[5] = {AF_XX, AF_YY, AF_XY, AF_XZ, AF_YZ};
    static const int med_f[4] = {AM_LAM, AM_MU, AM_QP, AM_QS};
    const int rsize = rtype == AWP_STORE_F32 ? 4 : 2;
    bool ok = make_map(&s->vm.d1, g, md.m[AM_D1], ST_W, ST_MR);
    for (int q = 0; q < ncomp; ++q) {
        for (int a = 0; a < 5; ++a) ok = ok && make_map(&s->vm.st[q][a], g, comp[q].f[vel_f[a]], ST_W, ST_HR);
        for (int a = 0; a < 3; ++a) ok = ok && make_map(&s->vm.p[q][a], g, comp[q].f[AF_U + a], ST_X, ST_Y);
        for (int a = 0; a < 3; ++a) ok = ok && make_map(&s->sm.v[q][a], g, comp[q].f[AF_U + a], ST_W, ST_HR);
        for (int a = 0; a < 6; ++a) ok = ok && make_map(&s->sm.s[q][a], g, comp[q].f[AF_XX + a], ST_X, ST_Y);
        for (int a = 0; a < 6; ++a)     /* absent in the elastic scheme, which never loads them */
            if (comp[q].f[AF_R1 + a]) ok = ok && make_map(&s->sm.r[q][a], g, comp[q].f[AF_R1 + a], ST_X, ST_Y, rsize);
        if (rtype == AWP_STORE_BFP && comp[q].f[AF_R1])
            ok = ok && comp[q].f[AF_RX] && make_map(&s->sm.rx[q], g, comp[q].f[AF_RX], ST_X, ST_Y, 2);
    }
    for (int a = 0; a < 4; ++a) ok = ok && make_map(&s->sm.med[a], g, md.m[med_f[a]], ST_W, ST_MR);
    if (!ok) {
        free(s);
        return cudaErrorInvalidValue;
    }
    *out = s;
    return cudaSuccess;
}

void awp_staged_destroy(AwpStaged *s) { free(s); }
#endif

static AwpWait awp_wait_of(const AwpStepArgs &s)
{
    AwpWait w;
    w.ns = s.wait_ns ? s.wait_ns : 2000000000ull;
    w.withhold = s.withhold;
    return w;
}

static AwpWork staged_work(const AwpGeom &g, int kchunk, int ncomp)
{
    AwpWork w;
    w.ntx = (g.nx + ST_X - 1) / ST_X;
    w.nty = (g.ny + ST_Y - 1) / ST_Y;
    w.kchunk = kchunk;
    w.nzc = (g.nz + kchunk - 1) / kchunk;
    w.nitems = w.ntx * w.nty * w.nzc * ncomp;
    return w;
}

template <class K>
static cudaError_t staged_grid(K kernel, size_t smem, int nitems, int *grid, int sm_limit, int threads = ST_THREADS)
{
    int dev = 0, nsm = 148, per = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (sm_limit > 0 && sm_limit < nsm) nsm = sm_limit;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    if (per < 1) return cudaErrorInvalidConfiguration;
    *grid = nsm * per < nitems ? nsm * per : nitems;
    return cudaSuccess;
}

static AwpCompSet<AWP_MAX_COMP> comp_set3(const AwpStepArgs &s)
{
    AwpCompSet<AWP_MAX_COMP> cs;
    memset(&cs, 0, sizeof cs);
    for (int q = 0; q < s.ncomp; ++q) cs.c[q] = s.comp[q];
    return cs;
}

/* dynamic shared memory of a ring: alignment slack, slots, full + empty barriers */
static size_t ring_bytes(int slots, int slot_floats) { return 128 + (size_t)slots * slot_floats * 4 + 2 * 8 * slots; }

template <int UNR>
static cudaError_t launch_vel_u(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    constexpr int RPT = UNR < 0 ? 2 : 1;            /* UNR -1: two rows per thread, level loop rolled */
    constexpr int U = UNR < 0 ? 1 : UNR;
    constexpr int CW = ST_Y / RPT;
    const size_t smem = ring_bytes(1 + ST_VEL_D, VEL_SLOT);
    const AwpWork w = staged_work(s.g, s.kchunk_staged, s.ncomp);
    int grid = 0;
    if (s.staged_generic && UNR == 2) {                 /* generic ring loads (ring_base_t) */
        cudaError_t e = staged_grid(k_vel_tma<ST_VEL_D, 2, 1, true>, smem, w.nitems, &grid, s.sm_limit, 32 * (ST_Y + 1));
        if (e != cudaSuccess) return e;
        k_vel_tma<ST_VEL_D, 2, 1, true><<<grid, dim3(32, ST_Y + 1), smem, stream>>>(
            st->vm, s.g, comp_set3(s), s.ncomp, s.staged_qslow, (const float *)s.md.m[AM_D1], s.cx, s.cy, s.cz, s.dth,
            w, s.kerr, awp_wait_of(s));
        return cudaGetLastError();
    }
    cudaError_t e = staged_grid(k_vel_tma<ST_VEL_D, U, RPT>, smem, w.nitems, &grid, s.sm_limit, 32 * (CW + 1));
    if (e != cudaSuccess) return e;
    k_vel_tma<ST_VEL_D, U, RPT><<<grid, dim3(32, CW + 1), smem, stream>>>(
        st->vm, s.g, comp_set3(s), s.ncomp, s.staged_qslow, (const float *)s.md.m[AM_D1], s.cx, s.cy, s.cz, s.dth, w,
        s.kerr, awp_wait_of(s));
    return cudaGetLastError();
}

template <class TR, int UNR, int RPT>
static cudaError_t launch_str_rpt(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    constexpr int CW = ST_Y / RPT;
    const size_t smem = ring_bytes(2 + STR_D, STR_SLOT);
    const AwpWork w = staged_work(s.g, s.kchunk_staged, s.ncomp);
    int grid = 0;
    if (s.staged_generic && UNR == 2 && RPT == 1) {     /* generic ring loads (ring_base_t) */
        cudaError_t e = staged_grid(k_str_tma<TR, 2, 1, true>, smem, w.nitems, &grid, s.sm_limit, 32 * (ST_Y + 1));
        if (e != cudaSuccess) return e;
        k_str_tma<TR, 2, 1, true><<<grid, dim3(32, ST_Y + 1), smem, stream>>>(st->sm, s.g, comp_set3(s), s.ncomp,
                                                                            s.staged_qslow, s.cx, s.cy, s.cz, s.tau,
                                                                            s.dth, s.dt, s.dh1, w, s.nve, s.kerr,
                                                                            awp_wait_of(s));
        return cudaGetLastError();
    }
    cudaError_t e = staged_grid(k_str_tma<TR, UNR, RPT>, smem, w.nitems, &grid, s.sm_limit, 32 * (CW + 1));
    if (e != cudaSuccess) return e;
    k_str_tma<TR, UNR, RPT><<<grid, dim3(32, CW + 1), smem, stream>>>(st->sm, s.g, comp_set3(s), s.ncomp,
                                                                       s.staged_qslow, s.cx, s.cy, s.cz, s.tau,
                                                                       s.dth, s.dt, s.dh1, w, s.nve, s.kerr, awp_wait_of(s));
    return cudaGetLastError();
}

/* CS component sub-slots: CS - 1 (level, component) tiles in flight */
template <class TR, int NCB, int CS, int RPT>
static cudaError_t launch_str_bc(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    constexpr int CW = ST_Y / RPT;
    const size_t smem = 128 + (size_t)(STB_MS * STB_MSLOT + CS * STB_CSLOT) * 4 + 2 * 8 * (STB_MS + CS);
    const AwpWork w = staged_work(s.g, s.kchunk_staged, 1);
    int grid = 0;
    cudaError_t e = staged_grid(k_str_tmab<TR, NCB, CS, RPT>, smem, w.nitems, &grid, s.sm_limit, 32 * (CW + 1));
    if (e != cudaSuccess) return e;
    k_str_tmab<TR, NCB, CS, RPT><<<grid, dim3(32, CW + 1), smem, stream>>>(
        st->sm, s.g, comp_set3(s), s.cx, s.cy, s.cz, s.tau, s.dth, s.dt, s.dh1, w, s.nve, s.kerr, awp_wait_of(s));
    return cudaGetLastError();
}

/* five sub-slots (109 KB with the media ring, two blocks per SM) measured
 * slightly ahead of four on the 400 x 400 x 200 three-component grid; one
 * row per thread: with two (161 registers) a launch took 3.00 ms against
 * 2.39 ms there, so staged_rpt applies to the one-component-per-item form only */
template <class TR, int NCB>
static cudaError_t launch_str_b(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    return launch_str_bc<TR, NCB, 5, 1>(st, s, stream);
}

/* two rows per thread carry twice the live state already: that variant keeps
 * its level loop rolled (unrolled twice it needs 128 registers and runs slower) */
template <class TR>
static cudaError_t launch_str_tr(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    if ((s.staged_batch & 1) && s.ncomp == 3) return launch_str_b<TR, 3>(st, s, stream);
    if ((s.staged_batch & 1) && s.ncomp == 2) return launch_str_b<TR, 2>(st, s, stream);
    if (s.staged_rpt == 2) return launch_str_rpt<TR, 1, 2>(st, s, stream);
    return s.unroll == 1 ? launch_str_rpt<TR, 1, 1>(st, s, stream) : launch_str_rpt<TR, 2, 1>(st, s, stream);
}

template <int NCB, int CS>
static cudaError_t launch_vel_b(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    const size_t smem = 128 + (size_t)(VB_MS * ST_MP + CS * VB_CSLOT) * 4 + 2 * 8 * (VB_MS + CS);
    const AwpWork w = staged_work(s.g, s.kchunk_staged, 1);
    int grid = 0;
    cudaError_t e = staged_grid(k_vel_tmab<NCB, CS>, smem, w.nitems, &grid, s.sm_limit);
    if (e != cudaSuccess) return e;
    k_vel_tmab<NCB, CS><<<grid, dim3(32, ST_CW + 1), smem, stream>>>(
        st->vm, s.g, comp_set3(s), (const float *)s.md.m[AM_D1], s.cx, s.cy, s.cz, s.dth, w, s.kerr, awp_wait_of(s));
    return cudaGetLastError();
}

/* eight sub-slots (two blocks per SM): 1.20 ms per launch on the 400 x 400 x
 * 200 three-component grid against 1.28 with six, and 1.05 for one component
 * per item, which stays the default */
template <int NCB>
static cudaError_t launch_vel_bn(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    return launch_vel_b<NCB, 8>(st, s, stream);
}

/* level loops unrolled twice unless asked otherwise: the column queues then
 * rotate by register renaming instead of moves that wait for loads in flight */
cudaError_t AWP_STAGED_ENTRY(awp_launch_vel_staged)(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    if (!st || s.md.type != AWP_STORE_F32) return cudaErrorInvalidValue;
    if ((s.staged_batch & 2) && s.ncomp == 3) return launch_vel_bn<3>(st, s, stream);
    if ((s.staged_batch & 2) && s.ncomp == 2) return launch_vel_bn<2>(st, s, stream);
    if (s.staged_rpt_vel == 2) return launch_vel_u<-1>(st, s, stream);
    return s.unroll == 1 ? launch_vel_u<1>(st, s, stream) : launch_vel_u<2>(st, s, stream);
}

cudaError_t AWP_STAGED_ENTRY(awp_launch_str_staged)(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream)
{
    if (!st || s.md.type != AWP_STORE_F32) return cudaErrorInvalidValue;
    if (s.rtype == AWP_STORE_BF16) return launch_str_tr<__nv_bfloat16>(st, s, stream);
    if (s.rtype == AWP_STORE_BFP) return launch_str_tr<RBfp>(st, s, stream);
    return launch_str_tr<float>(st, s, stream);
}
