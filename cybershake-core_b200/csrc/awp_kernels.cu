/*
 * awp_kernels.cu -- sm_100a kernels of the AWP-ODC-SGT stepper.
 *
 * Arithmetic follows the Fortran statement by statement with the same
 * evaluation order (awp_stencil.cuh); this translation unit is compiled with
 * --fmad=false so every product and sum is rounded once, as in the FP32 CPU
 * reference, and the FP32 steppers reproduce it bit for bit.
 *
 * Kernels:
 *   k_media_interior  structure.f:449-533   media -> compliances + Q transform
 *   k_media_ghosts    structure.f:563-707   padmedia / afsmedia
 *   k_media_homo      structure.f:709-765   inihomo
 *   k_media_convert   FP32 media -> bf16 / scaled binary16 storage
 *   k_sg_coeffs       pmcl3d.f:1158-1171    sg1 sg2 sg3 at the SGT points
 *   two-sweep stepper:
 *     k_vel           operator.f:92-244 + cerjan.f:292-330   velocity sweep
 *     k_fsvel         operator.f:246-306    free-surface velocity images
 *     k_str           viscoop.f:49-191 + cerjan.f:249-290 + operator.f:575-612
 *   fused stepper:
 *     k_fused         one z-march per xy tile: new velocities on the tile plus
 *                     a 2-cell halo into a 6-level shared-memory ring, then the
 *                     stress/memory-variable update of the tile two levels
 *                     below; free surface and fstr folded in; reads the old
 *                     wavefield buffer and writes the other one (ping-pong)
 *   k_post            source.f:812-913, pmcl3d.f:1379-1385, 1478-1479
 *   k_sgt             pmcl3d.f:1537-1557    SGT gather into the file image
 * NC = number of unit-force components stepped together (they share media).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "awp_internal.h"
#include "awp_kernels.h"
#include "awp_stencil.cuh"

/* ------------------------------------------------------------------ */
/* media                                                               */
/* ------------------------------------------------------------------ */

__device__ __forceinline__ void block_minmax6(float v[6], int *ext)
{
    /* v[0..2] are minima candidates (vp, vs, rho), v[3..5] maxima.  All
     * values are positive, so their IEEE bit patterns order like ints. */
    __shared__ int sh[6][32];
    const int lane = threadIdx.x & 31, warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    const int nwarp = (blockDim.x * blockDim.y + 31) >> 5;
    int b[6];
#pragma unroll
    for (int q = 0; q < 6; q++) b[q] = __float_as_int(v[q]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int q = 0; q < 3; q++) b[q] = min(b[q], __shfl_xor_sync(0xffffffffu, b[q], off));
#pragma unroll
        for (int q = 3; q < 6; q++) b[q] = max(b[q], __shfl_xor_sync(0xffffffffu, b[q], off));
    }
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 6; q++) sh[q][warp] = b[q];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < 6; q++) b[q] = (lane < nwarp) ? sh[q][lane] : sh[q][0];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
            for (int q = 0; q < 3; q++) b[q] = min(b[q], __shfl_xor_sync(0xffffffffu, b[q], off));
#pragma unroll
            for (int q = 3; q < 6; q++) b[q] = max(b[q], __shfl_xor_sync(0xffffffffu, b[q], off));
        }
        if (lane == 0) {
            for (int q = 0; q < 3; q++) atomicMin(&ext[q], b[q]);
            for (int q = 3; q < 6; q++) atomicMax(&ext[q], b[q]);
        }
    }
}

/* One z-slab of the media file (file z = zf0 .. zf0+nzs-1) -> interior cells.
 * Order of operations as structure.f:452-524. */
__global__ void k_media_interior(AwpGeom g, AwpMedia md, const float *__restrict__ raw, int zf0, int nzs,
                                 int nvar, int var_offset, int socalq, int nve,
                                 float pi, float lw, float tmp1, float tmp2, int *ext)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int zs = blockIdx.z;
    float v[6] = {99999.f, 99999.f, 99999.f, 0.f, 0.f, 0.f};
    if (i <= g.nx && j <= g.ny && zs < nzs) {
        const float *rec = raw + (((int64_t)zs * g.ny + (j - 1)) * g.nx + (i - 1)) * nvar + var_offset;
        float vp = rec[0], vs = rec[1], dd = rec[2];
        float pq = 0.f, sq = 0.f;
        if (nvar > 3) { pq = rec[3]; sq = rec[4]; }
        if (nvar == 3) { sq = 0.05f * vs; pq = 2.0f * sq; }
        if (socalq == 1) {
            vs = vs * (1.0f + (lw) / (pi * sq));
            vp = vp * (1.0f + (lw) / (pi * pq));
            float vpvs = vp / vs;
            if (vpvs < 1.45f) vs = vp / 1.45f;
        }
        const int k = g.nz - (zf0 + zs);
        const int c = g.idx(i, j, k);
        md.m[AM_MU][c] = 1.0f / (dd * vs * vs);
        md.m[AM_LAM][c] = 1.0f / (dd * (vp * vp - 2.0f * vs * vs));
        md.m[AM_D1][c] = dd;
        if (nve == 1) {
            float qpinv, qsinv;
            if (pq <= 0.0f) { qpinv = 0.f; qsinv = 0.f; }
            else { qpinv = 1.0f / pq; qsinv = 1.0f / sq; }
            md.m[AM_QP][c] = tmp1 * qpinv / (1.0f - tmp2 * qpinv);
            md.m[AM_QS][c] = tmp1 * qsinv / (1.0f - tmp2 * qsinv);
        }
        v[0] = vp; v[1] = vs; v[2] = dd; v[3] = vp; v[4] = vs; v[5] = dd;
    }
    block_minmax6(v, ext);
}

/* Ghost cells 0 and n+1 of lam/mu/d1 take the value of the nearest interior
 * cell (padmedia's planes, lines and corners and afsmedia's top plane all
 * reduce to this clamp), except the two assignments of structure.f:654-655
 * that copy lam(nxt,1,1) into mu and d1 at (nxt+1,0,0).  qp/qs get only the
 * afsmedia plane above the surface; their other ghosts stay zero. */
__global__ void k_media_ghosts(AwpGeom g, AwpMedia md, int nve)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;        /* 0..nx+1 */
    const int j = blockIdx.y * blockDim.y + threadIdx.y;        /* 0..ny+1 */
    const int k = blockIdx.z;                                   /* 0..nz+1 */
    if (i > g.nx + 1 || j > g.ny + 1 || k > g.nz + 1) return;
    const bool ghost = (i == 0 || i == g.nx + 1 || j == 0 || j == g.ny + 1 || k == 0 || k == g.nz + 1);
    if (!ghost) return;
    const int ic = min(max(i, 1), g.nx), jc = min(max(j, 1), g.ny), kc = min(max(k, 1), g.nz);
    const int c = g.idx(i, j, k), s = g.idx(ic, jc, kc);
    const bool quirk = (i == g.nx + 1 && j == 0 && k == 0);
    md.m[AM_LAM][c] = md.m[AM_LAM][s];
    md.m[AM_MU][c] = quirk ? md.m[AM_LAM][s] : md.m[AM_MU][s];
    md.m[AM_D1][c] = quirk ? md.m[AM_LAM][s] : md.m[AM_D1][s];
    if (nve == 1 && k == g.nz + 1 && i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) {
        md.m[AM_QP][c] = md.m[AM_QP][s];
        md.m[AM_QS][c] = md.m[AM_QS][s];
    }
}

/* inihomo: lam, mu, d1 constant over 0..n+1 in every direction; qp = qs = 0. */
__global__ void k_media_homo(AwpGeom g, AwpMedia md, float lam, float mu, float d1)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i > g.nx + 1 || j > g.ny + 1 || k > g.nz + 1) return;
    const int c = g.idx(i, j, k);
    md.m[AM_LAM][c] = lam;
    md.m[AM_MU][c] = mu;
    md.m[AM_D1][c] = d1;
}

/* |value| maxima and minima of the nonzero interior entries of each media
 * array (for the binary16 scale and range check).  Ghost cells hold copies
 * of interior values, except the padmedia corner (nx+1,0,0) whose d1 takes a
 * compliance; no stencil reads that d1, so it is left out of the range. */
__global__ void k_media_range(AwpGeom g, AwpMedia md, unsigned *mx, unsigned *mn)
{
    unsigned lmx[AM_N], lmn[AM_N];
    for (int a = 0; a < AM_N; a++) { lmx[a] = 0u; lmn[a] = 0x7f800000u; }
    const int64_t n = (int64_t)g.nx * g.ny * g.nz;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.nx) + 1;
        const int j = (int)((t / g.nx) % g.ny) + 1;
        const int k = (int)(t / ((int64_t)g.nx * g.ny)) + 1;
        const int c = g.idx(i, j, k);
        for (int a = 0; a < AM_N; a++) {
            unsigned b = __float_as_uint(fabsf(md.m[a][c]));
            if (b) { lmx[a] = max(lmx[a], b); lmn[a] = min(lmn[a], b); }
        }
    }
    for (int a = 0; a < AM_N; a++) {
        for (int off = 16; off > 0; off >>= 1) {
            lmx[a] = max(lmx[a], __shfl_xor_sync(0xffffffffu, lmx[a], off));
            lmn[a] = min(lmn[a], __shfl_xor_sync(0xffffffffu, lmn[a], off));
        }
        if ((threadIdx.x & 31) == 0) { atomicMax(&mx[a], lmx[a]); atomicMin(&mn[a], lmn[a]); }
    }
}

template <class TM>
__global__ void k_media_convert(AwpMedia src, void *d0, void *d1, void *d2, void *d3, void *d4, AwpMediaScale sc,
                                int64_t n)
{
    TM *dst[AM_N] = {(TM *)d0, (TM *)d1, (TM *)d2, (TM *)d3, (TM *)d4};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < AM_N; a++)
            if (dst[a]) Store<TM>::st(dst[a], (int)t, src.m[a][t], sc.scale[a]);
}

/* pmcl3d.f:1166-1168, evaluated at the SGT points only. */
template <class TM>
__global__ void k_sg_coeffs(MediaT<TM> md, int npts, const int *__restrict__ pt_idx, float *sg)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= npts) return;
    const int c = pt_idx[n];
    const float lam = md(AM_LAM, c), mu = md(AM_MU, c);
    sg[3 * n] = (1.0f / lam + 1.0f / mu) / (1.0f / mu * (3.0f / lam + 2.0f / mu));
    sg[3 * n + 1] = -(1.0f / lam / (2.0f / mu * (3.0f / lam + 2.0f / mu)));
    sg[3 * n + 2] = mu;
}

/* ------------------------------------------------------------------ */
/* two-sweep stepper                                                   */
/* ------------------------------------------------------------------ */

/* register budgets: 256-thread blocks, more blocks per SM for one component */
#define VEL_MINB(NC, UNR) ((UNR) == 1 ? ((NC) == 1 ? 6 : 4) : ((NC) == 1 ? 3 : 2))
#define STR_MINB(NC, UNR) ((NC) == 1 ? 4 : ((NC) == 2 ? 3 : 2))

template <int NC, class TM, int UNR>
__global__ void __launch_bounds__(256, VEL_MINB(NC, UNR))
k_vel(AwpGeom g, MediaT<TM> md, AwpCompSet<NC> cs, const float *__restrict__ cx, const float *__restrict__ cy,
      const float *__restrict__ cz, float dth, AwpWork w)
{
    const int sy = g.px, sz = g.plane;
    for (int item = blockIdx.x; item < w.nitems; item += gridDim.x) {
        int bx, by, k0, k1;
        work_item(g, w, item, bx, by, k0, k1);
        const int i = bx * blockDim.x + threadIdx.x + 1;
        const int j = by * blockDim.y + threadIdx.y + 1;
        if (i > g.nx || j > g.ny) continue;
        const float cxy = cx[i] * cy[j];
#pragma unroll (UNR)
        for (int k = k0; k <= k1; ++k) {
            const int c = g.idx(i, j, k);
            float fu, fv, fw;
            vel_factors(md, c, sy, sz, dth, fu, fv, fw);
            const float crj = cxy * cz[k];
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                float u, v, w_;
                vel_one(cs.c[q], c, sy, sz, fu, fv, fw, u, v, w_);
                /* Cerjan: the factor is exactly 1 outside the sponge zones */
                cs.c[q].f[AF_U][c] = u * crj;
                cs.c[q].f[AF_V][c] = v * crj;
                cs.c[q].f[AF_W][c] = w_ * crj;
            }
        }
    }
}

/* fvelxy then fvelz.  Each thread recomputes the two neighbouring fvelxy
 * values fvelz needs, so one launch covers both routines. */
template <int NC, class TM>
__global__ void k_fsvel(AwpGeom g, MediaT<TM> md, AwpCompSet<NC> cs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.nx || j > g.ny) return;
    const int nz = g.nz;
    const int c = g.idx(i, j, nz), sy = g.px, sz = g.plane;
    const float xl = 1.0f / md(AM_LAM, c);
    const float xl2m = 2.0f / md(AM_MU, c) + xl;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        float *u1 = cs.c[q].f[AF_U], *v1 = cs.c[q].f[AF_V], *w1 = cs.c[q].f[AF_W];
        const float u_fs = u1[c] - (w1[c] - w1[c - 1]);
        const float v_fs = v1[c] - (w1[c + sy] - w1[c]);
        const float u_fs_e = (i + 1 <= g.nx) ? (u1[c + 1] - (w1[c + 1] - w1[c])) : 0.0f;
        const float v_fs_s = (j - 1 >= 1) ? (v1[c - sy] - (w1[c] - w1[c - sy])) : 0.0f;
        const float w_fs = w1[c - sz] - (xl / xl2m) * (
            (u_fs_e - u_fs) +
            (u1[c + 1] - u1[c]) +
            (v_fs - v_fs_s) +
            (v1[c] - v1[c - sy]));
        u1[c + sz] = u_fs;
        v1[c + sz] = v_fs;
        w1[c + sz] = w_fs;
    }
}

template <int NC, class TM, class TR, int UNR>
__global__ void __launch_bounds__(256, STR_MINB(NC, UNR))
k_str(AwpGeom g, MediaT<TM> md, AwpCompSet<NC> cs, const float *__restrict__ cx, const float *__restrict__ cy,
      const float *__restrict__ cz, const float *__restrict__ tau, float dth, float dt, float dh1, AwpWork w,
      int nve)
{
    const int sy = g.px, sz = g.plane;
    for (int item = blockIdx.x; item < w.nitems; item += gridDim.x) {
        int bx, by, k0, k1;
        work_item(g, w, item, bx, by, k0, k1);
        const int i = bx * blockDim.x + threadIdx.x + 1;
        const int j = by * blockDim.y + threadIdx.y + 1;
        if (i > g.nx || j > g.ny) continue;
        const float cxy = cx[i] * cy[j];
        const int itxy = ((j & 1) << 1) | (i & 1);
#pragma unroll (UNR)
        for (int k = k0; k <= k1; ++k) {
            const int c = g.idx(i, j, k);
            const int it = (((g.nz + 1 - k) & 1) << 2) | itxy;   /* viscoop.f:93-101 */
            const StrCoef kc = str_coef(md, c, sy, sz, nve, tau[it], tau[8 + it]);
            const float crj = cxy * cz[k];
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                AwpComp &cp = cs.c[q];
                const GVel V{cp.f[AF_U], cp.f[AF_V], cp.f[AF_W], c, sy, sz};
                const Stress6 s{cp.f[AF_XX][c], cp.f[AF_YY][c], cp.f[AF_ZZ][c], cp.f[AF_XY][c], cp.f[AF_XZ][c], cp.f[AF_YZ][c]};
                Stress6 o;
                if (nve == 1) {
                    float r[6];
                    RVars<TR>::ld(cp, c, r);
                    const VelDiff d = vel_diff(V);
                    o = str_visco(kc, d, s, r, dth, dt, dh1);
                    RVars<TR>::st(cp, c, r);
                } else {
                    o = str_elastic(kc, V, s, dth);
                }
                cp.f[AF_XX][c] = o.xx * crj; cp.f[AF_YY][c] = o.yy * crj; cp.f[AF_ZZ][c] = o.zz * crj;
                cp.f[AF_XY][c] = o.xy * crj; cp.f[AF_XZ][c] = o.xz * crj; cp.f[AF_YZ][c] = o.yz * crj;
            }
        }
        if (k1 == g.nz) {
            /* fstr (operator.f:594-606) on this thread's own column */
            const int c = g.idx(i, j, g.nz);
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                float *zz = cs.c[q].f[AF_ZZ], *xz = cs.c[q].f[AF_XZ], *yz = cs.c[q].f[AF_YZ];
                zz[c + sz] = -__ldcg(&zz[c]);
                zz[c + 2 * sz] = -__ldcg(&zz[c - sz]);
                xz[c + sz] = -__ldcg(&xz[c - sz]);
                xz[c + 2 * sz] = -__ldcg(&xz[c - 2 * sz]);
                yz[c + sz] = -__ldcg(&yz[c - sz]);
                yz[c + 2 * sz] = -__ldcg(&yz[c - 2 * sz]);
                xz[c] = 0.0f;
                yz[c] = 0.0f;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* fused stepper                                                       */
/* ------------------------------------------------------------------ */

#define FX 32                      /* tile width (one warp along x)      */
#define FSLOT 6                    /* velocity levels kept in the ring   */

/* velocity accessor over the shared-memory ring (fused stress phase) */
template <int RX>
struct SVel {
    const float *lat_u, *lat_v, *lat_w;   /* level k planes, at the cell    */
    const float *zu[5], *zv[5], *zw[5];   /* levels k-2..k+2, at the cell   */
    __device__ __forceinline__ float u(int dx, int dy, int dz) const { return dz ? zu[dz + 2][0] : lat_u[dy * RX + dx]; }
    __device__ __forceinline__ float v(int dx, int dy, int dz) const { return dz ? zv[dz + 2][0] : lat_v[dy * RX + dx]; }
    __device__ __forceinline__ float w(int dx, int dy, int dz) const { return dz ? zw[dz + 2][0] : lat_w[dy * RX + dx]; }
};

template <int NC, class TM, class TR, int TY>
__global__ void __launch_bounds__(FX * TY)
k_fused(AwpGeom g, MediaT<TM> md, AwpCompSet<NC> old, AwpCompSet<NC> nw, const float *__restrict__ cx,
        const float *__restrict__ cy, const float *__restrict__ cz, const float *__restrict__ tau, float dth,
        float dt, float dh1, AwpWork wk, int nve)
{
    constexpr int RX = FX + 4, RY = TY + 4, NV = RX * RY, NT = FX * TY;
    constexpr int PLANE = 3 * NC * NV;                 /* one ring slot      */
    extern __shared__ float ring[];                    /* [FSLOT][NC][3][NV] */
    const int tx = threadIdx.x, ty = threadIdx.y, t = ty * FX + tx;
    const int sy = g.px, sz = g.plane, nz = g.nz;
    (void)RY;
    for (int item = blockIdx.x; item < wk.nitems; item += gridDim.x) {
    int bx, by, k0, k1;
    work_item(g, wk, item, bx, by, k0, k1);
    const int x0 = bx * FX + 1, y0 = by * TY + 1;

    /* this thread's cell in the stress phase */
    const int is = x0 + tx, js = y0 + ty;
    const bool sact = is <= g.nx && js <= g.ny;
    const int lps = (ty + 2) * RX + (tx + 2);
    const float cxy_s = sact ? cx[is] * cy[js] : 0.f;
    const int itxy = ((js & 1) << 1) | (is & 1);
    float hzz[NC], hxz[NC][2], hyz[NC][2];             /* new values below k  */
#pragma unroll
    for (int q = 0; q < NC; ++q) { hzz[q] = 0.f; hxz[q][0] = hxz[q][1] = hyz[q][0] = hyz[q][1] = 0.f; }

    for (int m = k0 - 2; m <= k1 + 2; ++m) {
        /* ---- velocity at level m on the tile plus a 2-cell halo ---- */
        float *sl = ring + ((m + 2 * FSLOT) % FSLOT) * PLANE;
        for (int vcell = t; vcell < NV; vcell += NT) {
            const int lx = vcell % RX, ly = vcell / RX;
            const int i = x0 - 2 + lx, j = y0 - 2 + ly;
            const bool inside = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
            const bool inter = lx >= 2 && lx < FX + 2 && ly >= 2 && ly < TY + 2;
            float val[NC][3];
#pragma unroll
            for (int q = 0; q < NC; ++q) val[q][0] = val[q][1] = val[q][2] = 0.f;
            if (inside && m >= 1 && m <= nz) {
                const int c = g.idx(i, j, m);
                float fu, fv, fw;
                vel_factors(md, c, sy, sz, dth, fu, fv, fw);
                const float crj = (cx[i] * cy[j]) * cz[m];
                const bool own = inter && m >= k0 && m <= k1;
#pragma unroll
                for (int q = 0; q < NC; ++q) {
                    float u, v, w;
                    vel_one(old.c[q], c, sy, sz, fu, fv, fw, u, v, w);
                    val[q][0] = u * crj; val[q][1] = v * crj; val[q][2] = w * crj;
                    if (own) {
                        nw.c[q].f[AF_U][c] = val[q][0];
                        nw.c[q].f[AF_V][c] = val[q][1];
                        nw.c[q].f[AF_W][c] = val[q][2];
                    }
                }
            } else if (inside && inter && m == nz + 1) {
                /* fvelxy + fvelz from level nz (and w at nz-1) of the ring */
                const float *p0 = ring + ((nz + 2 * FSLOT) % FSLOT) * PLANE;
                const float *p1 = ring + ((nz - 1 + 2 * FSLOT) % FSLOT) * PLANE;
                const int ct = g.idx(i, j, nz);
                const float xl = 1.0f / md(AM_LAM, ct);
                const float xl2m = 2.0f / md(AM_MU, ct) + xl;
#pragma unroll
                for (int q = 0; q < NC; ++q) {
                    const float *U = p0 + (q * 3 + 0) * NV + vcell;
                    const float *V = p0 + (q * 3 + 1) * NV + vcell;
                    const float *W = p0 + (q * 3 + 2) * NV + vcell;
                    const float u_fs = U[0] - (W[0] - W[-1]);
                    const float v_fs = V[0] - (W[RX] - W[0]);
                    const float u_fs_e = (i + 1 <= g.nx) ? (U[1] - (W[1] - W[0])) : 0.0f;
                    const float v_fs_s = (j - 1 >= 1) ? (V[-RX] - (W[0] - W[-RX])) : 0.0f;
                    const float w_fs = p1[(q * 3 + 2) * NV + vcell] - (xl / xl2m) * (
                        (u_fs_e - u_fs) + (U[1] - U[0]) + (v_fs - v_fs_s) + (V[0] - V[-RX]));
                    val[q][0] = u_fs; val[q][1] = v_fs; val[q][2] = w_fs;
                    if (k1 == nz) {
                        nw.c[q].f[AF_U][ct + sz] = u_fs;
                        nw.c[q].f[AF_V][ct + sz] = v_fs;
                        nw.c[q].f[AF_W][ct + sz] = w_fs;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                sl[(q * 3 + 0) * NV + vcell] = val[q][0];
                sl[(q * 3 + 1) * NV + vcell] = val[q][1];
                sl[(q * 3 + 2) * NV + vcell] = val[q][2];
            }
        }
        __syncthreads();

        /* ---- stress + memory variables at level k = m - 2 on the tile ---- */
        const int k = m - 2;
        if (k >= k0 && k <= k1 && sact) {
            const int c = g.idx(is, js, k);
            const int it = (((nz + 1 - k) & 1) << 2) | itxy;
            const StrCoef kc = str_coef(md, c, sy, sz, nve, tau[it], tau[8 + it]);
            const float crj = cxy_s * cz[k];
            const float *lv = ring + ((k + 2 * FSLOT) % FSLOT) * PLANE + lps;
            const float *zl[5];
#pragma unroll
            for (int d = 0; d < 5; ++d) zl[d] = ring + ((k - 2 + d + 2 * FSLOT) % FSLOT) * PLANE + lps;
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                SVel<RX> V;
                V.lat_u = lv + (q * 3 + 0) * NV;
                V.lat_v = lv + (q * 3 + 1) * NV;
                V.lat_w = lv + (q * 3 + 2) * NV;
#pragma unroll
                for (int d = 0; d < 5; ++d) {
                    V.zu[d] = zl[d] + (q * 3 + 0) * NV;
                    V.zv[d] = zl[d] + (q * 3 + 1) * NV;
                    V.zw[d] = zl[d] + (q * 3 + 2) * NV;
                }
                const AwpComp &o = old.c[q];
                const Stress6 s{o.f[AF_XX][c], o.f[AF_YY][c], o.f[AF_ZZ][c], o.f[AF_XY][c], o.f[AF_XZ][c], o.f[AF_YZ][c]};
                Stress6 ns;
                if (nve == 1) {
                    float r[6];
                    RVars<TR>::ld(o, c, r);
                    const VelDiff d = vel_diff(V);
                    ns = str_visco(kc, d, s, r, dth, dt, dh1);
                    RVars<TR>::st(o, c, r);
                } else {
                    ns = str_elastic(kc, V, s, dth);
                }
                ns.xx = ns.xx * crj; ns.yy = ns.yy * crj; ns.zz = ns.zz * crj;
                ns.xy = ns.xy * crj; ns.xz = ns.xz * crj; ns.yz = ns.yz * crj;
                AwpComp &n = nw.c[q];
                n.f[AF_XX][c] = ns.xx; n.f[AF_YY][c] = ns.yy; n.f[AF_ZZ][c] = ns.zz; n.f[AF_XY][c] = ns.xy;
                if (k == nz) {
                    /* fstr (operator.f:594-606) from this thread's own column */
                    n.f[AF_ZZ][c + sz] = -ns.zz;
                    n.f[AF_ZZ][c + 2 * sz] = -hzz[q];
                    n.f[AF_XZ][c + sz] = -hxz[q][0];
                    n.f[AF_XZ][c + 2 * sz] = -hxz[q][1];
                    n.f[AF_YZ][c + sz] = -hyz[q][0];
                    n.f[AF_YZ][c + 2 * sz] = -hyz[q][1];
                    n.f[AF_XZ][c] = 0.0f;
                    n.f[AF_YZ][c] = 0.0f;
                } else {
                    n.f[AF_XZ][c] = ns.xz;
                    n.f[AF_YZ][c] = ns.yz;
                }
                hzz[q] = ns.zz;
                hxz[q][1] = hxz[q][0]; hxz[q][0] = ns.xz;
                hyz[q][1] = hyz[q][0]; hyz[q][0] = ns.yz;
            }
        }
    }
    __syncthreads();   /* the next item's first velocity levels reuse the ring */
    }
}

/* ------------------------------------------------------------------ */
/* per-step serial work: source insertion, fstr redo, CHKJ probe       */
/* ------------------------------------------------------------------ */

__device__ void fstr_column(const AwpGeom &g, AwpComp &cp, int i, int j)
{
    const int nz = g.nz, sz = g.plane;
    const int c = g.idx(i, j, nz);
    float *zz = cp.f[AF_ZZ], *xz = cp.f[AF_XZ], *yz = cp.f[AF_YZ];
    zz[c + sz] = -zz[c];
    zz[c + 2 * sz] = -zz[c - sz];
    xz[c + sz] = -xz[c - sz];
    xz[c + 2 * sz] = -xz[c - 2 * sz];
    yz[c + sz] = -yz[c - sz];
    yz[c + 2 * sz] = -yz[c - 2 * sz];
    xz[c] = 0.0f;
    yz[c] = 0.0f;
}

__device__ __forceinline__ float d1_at(const AwpPostArgs &a, int c)
{
    switch (a.media_type) {
    case 1: return __bfloat162float(((const __nv_bfloat16 *)a.d1)[c]);
    case 2: return __half2float(((const __half *)a.d1)[c]) * a.d1_inv;
    default: return ((const float *)a.d1)[c];
    }
}

/* One block; thread q handles component q and walks its sources in order,
 * as the Fortran loop over j=1,npsrc does.
 * initial != 0: addsrc(1) before the time loop (pmcl3d.f:966-988).
 * otherwise: step n = *step + 1 just finished its stress update:
 *   addsrc(n+1) [and fstr again where a moment source sits in the top three
 *   layers, since pmcl3d.f:1383-1384 inserts before fstr], CHKJ sample,
 *   then *step = n. */
__global__ void k_post(AwpPostArgs a, int initial)
{
    const int q = threadIdx.x;
    const int n = initial ? 0 : (*a.step + 1);
    const int sample = initial ? 1 : n + 1;
    if (q < a.ncomp && sample <= a.nst && !a.kinematic) {
        const AwpSrcDev &s = a.src[q];
        AwpComp &cp = a.comp[q];
        const AwpGeom &g = a.g;
        const int nz = g.nz, sz = g.plane;
        for (int m = 0; m < s.nsrc; ++m) {
            const int i = s.ijk[3 * m], j = s.ijk[3 * m + 1], k = s.ijk[3 * m + 2];
            const float *t = s.stf + ((int64_t)m * a.nst + (sample - 1)) * 6;
            const float axx = t[0], ayy = t[1], azz = t[2], axz = t[3], ayz = t[4], axy = t[5];
            const int c = g.idx(i, j, k);
            const int ct = g.idx(i, j, nz);
            switch (s.igreen) {
            case -1:
                cp.f[AF_XX][c] = cp.f[AF_XX][c] - a.vtst * axx;
                cp.f[AF_YY][c] = cp.f[AF_YY][c] - a.vtst * ayy;
                cp.f[AF_ZZ][c] = cp.f[AF_ZZ][c] - a.vtst * azz;
                cp.f[AF_XZ][c] = cp.f[AF_XZ][c] - a.vtst * axz;
                cp.f[AF_YZ][c] = cp.f[AF_YZ][c] - a.vtst * ayz;
                cp.f[AF_XY][c] = cp.f[AF_XY][c] - a.vtst * axy;
                break;
            case 1:
                cp.f[AF_U][c] = cp.f[AF_U][c] + axx * a.vtst / d1_at(a, c);
                break;
            case 2:
                cp.f[AF_V][c] = cp.f[AF_V][c] + ayy * a.vtst / d1_at(a, c);
                break;
            case 3:
                cp.f[AF_W][c] = cp.f[AF_W][c] + azz * a.vtst / d1_at(a, c);
                break;
            case -2:
                cp.f[AF_U][c] = cp.f[AF_U][c] + axx * a.vtst / d1_at(a, c);
                cp.f[AF_V][c] = cp.f[AF_V][c] + ayy * a.vtst / d1_at(a, c);
                cp.f[AF_W][c] = cp.f[AF_W][c] + azz * a.vtst / d1_at(a, c);
                break;
            case 4: {
                float *F = cp.f[AF_XZ];
                F[ct] = axx * a.vtst1;
                F[ct + sz] = 2.0f * axx * a.vtst1 - F[ct - sz];
                F[ct + 2 * sz] = 2.0f * axx * a.vtst1 - F[ct - 2 * sz];
            } break;
            case 5: {
                float *F = cp.f[AF_YZ];
                F[ct] = ayy * a.vtst1;
                F[ct + sz] = 2.0f * ayy * a.vtst1 - F[ct - sz];
                F[ct + 2 * sz] = 2.0f * ayy * a.vtst1 - F[ct - 2 * sz];
            } break;
            case 6: {
                float *F = cp.f[AF_ZZ];
                F[ct + sz] = 2.0f * azz * a.vtst1 - F[ct];
                F[ct + 2 * sz] = 2.0f * azz * a.vtst1 - F[ct - sz];
            } break;
            default:
                break;
            }
        }
        if (!initial && s.igreen == -1) {
            for (int m = 0; m < s.nsrc; ++m)
                if (s.ijk[3 * m + 2] >= nz - 2) fstr_column(g, cp, s.ijk[3 * m], s.ijk[3 * m + 1]);
        }
    }
    if (initial) return;
    __syncthreads();
    if (q < a.ncomp && a.probe > 0 && n >= 1 && n <= a.nt) {
        const int c = a.g.idx(a.probe, a.probe, a.probe);
        a.chkj[q][3 * (n - 1)] = a.comp[q].f[AF_U][c];
        a.chkj[q][3 * (n - 1) + 1] = a.comp[q].f[AF_V][c];
        a.chkj[q][3 * (n - 1) + 2] = a.comp[q].f[AF_W][c];
    }
    __syncthreads();
    if (q == 0) *a.step = n;
}

/* SGT gather, pmcl3d.f:1537-1557.  Sample s (0-based) of every point goes
 * straight to its place in the raw file image, [pt][6][nt_file]. */
__global__ void k_sgt(AwpSgtArgs a)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.npts * a.ncomp) return;
    const int n = *a.step;
    if (n < a.ntiskp || n % a.ntiskp) return;
    const int s = n / a.ntiskp - 1;
    if (s >= a.nsamp_written) return;
    const int p = t % a.npts, q = t / a.npts;
    if (!a.active[q]) return;   /* no SGT output for moment sources (pmcl3d.f:1536) */
    const int c = a.pt_idx[p];
    const float sg1 = a.sg[3 * p], sg2 = a.sg[3 * p + 1], sg3 = a.sg[3 * p + 2];
    const AwpComp &cp = a.comp[q];
    const float xx = cp.f[AF_XX][c], yy = cp.f[AF_YY][c], zz = cp.f[AF_ZZ][c];
    const float xy = cp.f[AF_XY][c], xz = cp.f[AF_XZ][c], yz = cp.f[AF_YZ][c];
    float *o = a.file[q] + (int64_t)p * 6 * a.nt_file + s;
    o[0] = sg1 * xx + sg2 * yy + sg2 * zz;
    o[a.nt_file] = sg2 * xx + sg1 * yy + sg2 * zz;
    o[2 * a.nt_file] = sg2 * xx + sg2 * yy + sg1 * zz;
    o[3 * a.nt_file] = sg3 * xy;
    o[4 * a.nt_file] = sg3 * xz;
    o[5 * a.nt_file] = sg3 * yz;
}

/* ------------------------------------------------------------------ */
/* FP64 energy (stability monitor): two deterministic passes           */
/* ------------------------------------------------------------------ */

/* pass 1: block b sums u^2+v^2+w^2 over the rows r = b, b+G, ... of the
 * interior (a row is one (j,k) line of nx cells), in a fixed order, and
 * writes partial[b*ncomp + q] */
__global__ void __launch_bounds__(AWP_EN_BLOCK) k_energy_partial(AwpEnergyArgs a, double *partial)
{
    __shared__ double sh[3][AWP_EN_BLOCK];
    double acc[3] = {0.0, 0.0, 0.0};
    const int nrow = a.g.ny * a.g.nz;
    for (int r = blockIdx.x; r < nrow; r += gridDim.x) {
        const int j = r % a.g.ny + 1, k = r / a.g.ny + 1;
        const int c0 = a.g.idx(1, j, k);
        for (int i = threadIdx.x; i < a.g.nx; i += blockDim.x) {
            for (int q = 0; q < a.ncomp; ++q) {
                const double u = a.f[3 * q][c0 + i], v = a.f[3 * q + 1][c0 + i], w = a.f[3 * q + 2][c0 + i];
                acc[q] += u * u + v * v + w * w;
            }
        }
    }
    for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s = AWP_EN_BLOCK / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < (unsigned)a.ncomp) partial[blockIdx.x * a.ncomp + threadIdx.x] = sh[threadIdx.x][0];
}

/* pass 2: out[q] = sum of the block partials in block order; a non-finite
 * energy raises the instability flag */
__global__ void k_energy_final(const double *partial, int nblocks, int ncomp, double *out, int *flag)
{
    const int q = threadIdx.x;
    if (q >= ncomp) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[b * ncomp + q];
    out[q] = s;
    if (flag && !isfinite(s)) atomicExch(flag, 1);
}

cudaError_t awp_launch_energy(const AwpEnergyArgs &a, double *partial, int nblocks, double *out, int *flag,
                              cudaStream_t st)
{
    k_energy_partial<<<nblocks, AWP_EN_BLOCK, 0, st>>>(a, partial);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_energy_final<<<1, 32, 0, st>>>(partial, nblocks, a.ncomp, out, flag);
    return cudaGetLastError();
}

/* ------------------------------------------------------------------ */
/* launchers                                                           */
/* ------------------------------------------------------------------ */

static dim3 plane_grid(const AwpGeom &g, dim3 b, int nzb)
{
    return dim3((g.nx + b.x - 1) / b.x, (g.ny + b.y - 1) / b.y, nzb);
}

cudaError_t awp_launch_media_interior(const AwpGeom &g, const AwpMedia &md, const float *raw, int zf0, int nzs,
                                      int nvar, int var_offset, int socalq, int nve, float pi, float lw,
                                      float tmp1, float tmp2, int *ext, cudaStream_t st)
{
    dim3 b(32, 8);
    k_media_interior<<<plane_grid(g, b, nzs), b, 0, st>>>(g, md, raw, zf0, nzs, nvar, var_offset, socalq, nve,
                                                          pi, lw, tmp1, tmp2, ext);
    return cudaGetLastError();
}

cudaError_t awp_launch_media_ghosts(const AwpGeom &g, const AwpMedia &md, int nve, cudaStream_t st)
{
    dim3 b(32, 8);
    dim3 gr((g.nx + 2 + b.x - 1) / b.x, (g.ny + 2 + b.y - 1) / b.y, g.nz + 2);
    k_media_ghosts<<<gr, b, 0, st>>>(g, md, nve);
    return cudaGetLastError();
}

/* integer hash of the index (murmur3 finaliser), top 24 bits to [-amp, amp) */
__global__ void k_fill_noise(float *p, int64_t n, unsigned seed, float amp)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned h = (unsigned)i * 0x9E3779B1u ^ (unsigned)(i >> 32) ^ seed;
        h ^= h >> 16;
        h *= 0x85EBCA6Bu;
        h ^= h >> 13;
        h *= 0xC2B2AE35u;
        h ^= h >> 16;
        p[i] = amp * ((float)(h >> 8) * (1.0f / 8388608.0f) - 1.0f);
    }
}

cudaError_t awp_launch_fill_noise(float *p, int64_t n, unsigned seed, float amp, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_fill_noise<<<(int)blocks, 256, 0, st>>>(p, n, seed, amp);
    return cudaGetLastError();
}

cudaError_t awp_launch_media_homo(const AwpGeom &g, const AwpMedia &md, float lam, float mu, float d1, cudaStream_t st)
{
    dim3 b(32, 8);
    dim3 gr((g.nx + 2 + b.x - 1) / b.x, (g.ny + 2 + b.y - 1) / b.y, g.nz + 2);
    k_media_homo<<<gr, b, 0, st>>>(g, md, lam, mu, d1);
    return cudaGetLastError();
}

cudaError_t awp_launch_media_range(const AwpGeom &g, const AwpMedia &md, unsigned *mx, unsigned *mn, cudaStream_t st)
{
    k_media_range<<<148 * 4, 256, 0, st>>>(g, md, mx, mn);
    return cudaGetLastError();
}

cudaError_t awp_launch_media_convert(const AwpMedia &src, const AwpMediaT &dst, int64_t n, cudaStream_t st)
{
    if (dst.type == AWP_STORE_BF16)
        k_media_convert<__nv_bfloat16><<<148 * 8, 256, 0, st>>>(src, dst.m[0], dst.m[1], dst.m[2], dst.m[3], dst.m[4],
                                                               dst.sc, n);
    else if (dst.type == AWP_STORE_F16)
        k_media_convert<__half><<<148 * 8, 256, 0, st>>>(src, dst.m[0], dst.m[1], dst.m[2], dst.m[3], dst.m[4],
                                                        dst.sc, n);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

template <class TM>
static MediaT<TM> media_view(const AwpMediaT &m)
{
    MediaT<TM> v;
    for (int a = 0; a < AM_N; ++a) {
        v.m[a] = (const TM *)m.m[a];
        v.inv[a] = m.sc.inv[a];
    }
    return v;
}

cudaError_t awp_launch_sg_coeffs(const AwpMediaT &md, int npts, const int *pt_idx, float *sg, cudaStream_t st)
{
    if (npts <= 0) return cudaSuccess;
    const int nb = (npts + 255) / 256;
    switch (md.type) {
    case AWP_STORE_BF16: k_sg_coeffs<__nv_bfloat16><<<nb, 256, 0, st>>>(media_view<__nv_bfloat16>(md), npts, pt_idx, sg); break;
    case AWP_STORE_F16: k_sg_coeffs<__half><<<nb, 256, 0, st>>>(media_view<__half>(md), npts, pt_idx, sg); break;
    default: k_sg_coeffs<float><<<nb, 256, 0, st>>>(media_view<float>(md), npts, pt_idx, sg); break;
    }
    return cudaGetLastError();
}

template <int NC>
static void comp_sets(const AwpStepArgs &s, AwpCompSet<NC> &a, AwpCompSet<NC> &b)
{
    for (int q = 0; q < NC; ++q) { a.c[q] = s.comp[q]; b.c[q] = s.comp_new[q]; }
}

template <int TY, int NC>
static size_t fused_smem() { return (size_t)FSLOT * 3 * NC * (FX + 4) * (TY + 4) * sizeof(float); }

static AwpWork make_work(const AwpGeom &g, int ty, int kchunk)
{
    AwpWork w;
    w.ntx = (g.nx + 31) / 32;
    w.nty = (g.ny + ty - 1) / ty;
    w.kchunk = kchunk;
    w.nzc = (g.nz + kchunk - 1) / kchunk;
    w.nitems = w.ntx * w.nty * w.nzc;
    return w;
}

/* persistent grid: every SM filled to its occupancy, capped by the items */
template <class K>
static int persistent_grid(K kernel, int threads, size_t smem, int nitems, int sm_limit)
{
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (sm_limit > 0 && sm_limit < nsm) nsm = sm_limit;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1) per = 1;
    const int grid = nsm * per;
    return grid < nitems ? grid : nitems;
}

template <int NC, class TM, class TR, int TY>
static cudaError_t launch_fused(const AwpStepArgs &s, const MediaT<TM> &md, const AwpCompSet<NC> &cs,
                                const AwpCompSet<NC> &cn, cudaStream_t st)
{
    dim3 b(FX, TY);
    const size_t smem = fused_smem<TY, NC>();
    static unsigned long long attr_done = 0;   /* per instantiation, bit per device */
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64 || !(attr_done & (1ull << dev))) {
        cudaError_t e = cudaFuncSetAttribute(k_fused<NC, TM, TR, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        if (dev < 64) attr_done |= 1ull << dev;
    }
    const AwpWork w = make_work(s.g, TY, s.kchunk);
    const int grid = persistent_grid(k_fused<NC, TM, TR, TY>, FX * TY, smem, w.nitems, s.sm_limit);
    k_fused<NC, TM, TR, TY><<<grid, b, smem, st>>>(s.g, md, cs, cn, s.cx, s.cy, s.cz, s.tau, s.dth, s.dt, s.dh1, w,
                                                   s.nve);
    return cudaGetLastError();
}

template <int NC, class TM, int UNR>
static cudaError_t launch_vel(const AwpStepArgs &s, const MediaT<TM> &md, const AwpCompSet<NC> &cs, int ty,
                              cudaStream_t st)
{
    const AwpWork w = make_work(s.g, ty, s.kchunk_sweep);
    const int grid = persistent_grid(k_vel<NC, TM, UNR>, 32 * ty, 0, w.nitems, s.sm_limit);
    k_vel<NC, TM, UNR><<<grid, dim3(32, ty), 0, st>>>(s.g, md, cs, s.cx, s.cy, s.cz, s.dth, w);
    return cudaGetLastError();
}

template <int NC, class TM, class TR, int UNR>
static cudaError_t launch_str(const AwpStepArgs &s, const MediaT<TM> &md, const AwpCompSet<NC> &cs, int ty,
                              cudaStream_t st)
{
    const AwpWork w = make_work(s.g, ty, s.kchunk_sweep);
    const int grid = persistent_grid(k_str<NC, TM, TR, UNR>, 32 * ty, 0, w.nitems, s.sm_limit);
    k_str<NC, TM, TR, UNR><<<grid, dim3(32, ty), 0, st>>>(s.g, md, cs, s.cx, s.cy, s.cz, s.tau, s.dth, s.dt, s.dh1,
                                                          w, s.nve);
    return cudaGetLastError();
}

template <int NC, class TM, class TR>
static cudaError_t launch_part_t(const AwpStepArgs &s, int part, cudaStream_t st)
{
    AwpCompSet<NC> cs, cn;
    comp_sets<NC>(s, cs, cn);
    const MediaT<TM> md = media_view<TM>(s.md);
    if (part == AWP_PART_VEL) {
        if (s.staged) return s.fma ? awp_launch_vel_staged_fma(s.staged, s, st) : awp_launch_vel_staged(s.staged, s, st);
        const int ty = s.ty == 4 ? 4 : 8;
        return s.unroll == 2 ? launch_vel<NC, TM, 2>(s, md, cs, ty, st) : launch_vel<NC, TM, 1>(s, md, cs, ty, st);
    } else if (part == AWP_PART_FSVEL) {
        dim3 b(32, 8);
        k_fsvel<NC, TM><<<plane_grid(s.g, b, 1), b, 0, st>>>(s.g, md, cs);
    } else if (part == AWP_PART_STR) {
        if (s.staged) return s.fma ? awp_launch_str_staged_fma(s.staged, s, st) : awp_launch_str_staged(s.staged, s, st);
        const int ty = s.ty == 4 ? 4 : 8;
        return s.unroll == 2 ? launch_str<NC, TM, TR, 2>(s, md, cs, ty, st) : launch_str<NC, TM, TR, 1>(s, md, cs, ty, st);
    } else if (part == AWP_PART_FUSED) {
        if (s.ty == 4) return launch_fused<NC, TM, TR, 4>(s, md, cs, cn, st);
        if (s.ty == 16) return launch_fused<NC, TM, TR, 16>(s, md, cs, cn, st);
        return launch_fused<NC, TM, TR, 8>(s, md, cs, cn, st);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int NC>
static cudaError_t launch_part_nc(const AwpStepArgs &s, int part, cudaStream_t st)
{
    /* (media storage, r1..r6 storage) pairs of awp_precision */
    if (s.md.type == AWP_STORE_BF16) return launch_part_t<NC, __nv_bfloat16, __nv_bfloat16>(s, part, st);
    if (s.md.type == AWP_STORE_F16) return launch_part_t<NC, __half, __nv_bfloat16>(s, part, st);
    if (s.rtype == AWP_STORE_BF16) return launch_part_t<NC, float, __nv_bfloat16>(s, part, st);
    if (s.rtype == AWP_STORE_BFP) return launch_part_t<NC, float, RBfp>(s, part, st);
    return launch_part_t<NC, float, float>(s, part, st);
}

cudaError_t awp_launch_part(const AwpStepArgs &s, int part, cudaStream_t st)
{
    switch (s.ncomp) {
    case 1: return launch_part_nc<1>(s, part, st);
    case 2: return launch_part_nc<2>(s, part, st);
    case 3: return launch_part_nc<3>(s, part, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t awp_launch_step(const AwpStepArgs &s, cudaStream_t st)
{
    if (s.fused) return awp_launch_part(s, AWP_PART_FUSED, st);
    for (int part = 0; part < 3; ++part) {
        cudaError_t e = awp_launch_part(s, part, st);
        /* NPC = 1: the PML zones recomputed after the velocity sweep (before
         * the free-surface velocity) and after the stress sweep */
        if (e == cudaSuccess && s.pml && part == AWP_PART_VEL) e = awp_launch_pml(*s.pml, 0, st);
        if (e == cudaSuccess && s.pml && part == AWP_PART_STR) e = awp_launch_pml(*s.pml, 1, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

/* ------------------------------------------------------------------ */
/* kinematic source (IFAULT=5)                                         */
/* ------------------------------------------------------------------ */

/* Unit double-couple moment tensor M = n d^T + d n^T from the fault normal n
 * and the slip direction d of a fault with strike `str`, dip and rake
 * (radians), after Aki & Richards, Quantitative Seismology (2002), section
 * 4.5.  The vectors are written in the AWP axes (x east, y north, z up):
 *   n = ( sin(dip) cos(str), -sin(dip) sin(str), cos(dip) )
 *   d = ( cos(rake) sin(str) - cos(dip) sin(rake) cos(str),
 *         cos(rake) cos(str) + cos(dip) sin(rake) sin(str),  sin(rake) sin(dip) )
 * Output order: xx yy zz xz yz xy. */
__device__ __forceinline__ void kin_mt(float str, float dip, float rake, float m[6])
{
    float ss, cs, sd, cd, sr, cr;
    sincosf(str, &ss, &cs);
    sincosf(dip, &sd, &cd);
    sincosf(rake, &sr, &cr);
    const float n[3] = {sd * cs, -(sd * ss), cd};
    const float d[3] = {cr * ss - cd * sr * cs, cr * cs + cd * sr * ss, sr * sd};
    m[0] = 2.f * n[0] * d[0];
    m[1] = 2.f * n[1] * d[1];
    m[2] = 2.f * n[2] * d[2];
    m[3] = n[0] * d[2] + n[2] * d[0];
    m[4] = n[1] * d[2] + n[2] * d[1];
    m[5] = n[0] * d[1] + n[1] * d[0];
}

/* Brune (1970) slip rate of unit slip for a rise time `rise`: with
 * w = 2 pi / rise and x = w t, rate(t) = w x exp(-x) for t > 0. */
__device__ __forceinline__ float kin_brune(float rise, float t)
{
    if (!(t > 0.f)) return 0.f;
    const float w = 6.28318530717958647692f / rise, x = w * t;
    return w * x * expf(-x);
}

/* Slip rate of unit slip of Liu, Archuleta & Hartzell (2006, BSSA 96) and of
 * its revision in Graves & Pitarka (2010, BSSA 100), both of one family set by
 * the tail weight c (0.3 and 0.2).  With t1 = 0.13 rise, t2 = rise - t1,
 * s = t / t1 and u = (t - t1) / t2 the shape is
 *   0.7 (1 - cos(pi s)) + 0.6 sin(pi s / 2)     0    <= t < t1
 *   1 - (1 - c) cos(pi s) + c cos(pi u)         t1   <= t < 2 t1
 *   c (1 + cos(pi u))                           2 t1 <= t < rise
 * and its integral over the rise time, (1.7 - c) t1 + 1.2 t1 / pi + c t2,
 * normalises it to unit area. */
__device__ __forceinline__ float kin_liu(float rise, float t, float c)
{
    if (!(t > 0.f) || !(t < rise)) return 0.f;
    const float t1 = 0.13f * rise, t2 = rise - t1;
    const float area = (1.7f - c) * t1 + 1.2f * t1 / 3.14159265358979323846f + c * t2;
    const float s = t / t1, u = (t - t1) / t2;
    float f;
    if (t < t1) f = 0.7f * (1.f - cospif(s)) + 0.6f * sinpif(0.5f * s);
    else if (t < 2.f * t1) f = 1.f - (1.f - c) * cospif(s) + c * cospif(u);
    else f = c * (1.f + cospif(u));
    return f / area;
}

/* stress increments of every subfault at step n (= *step + 1), one thread per
 * subfault: rows [type slip t_rupture t_rise area .] [strike dip rake . . .] */
__global__ void k_kin_contrib(AwpPostArgs a)
{
    const int q = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.ncomp || j >= a.src[q].nsrc) return;
    const float *r0 = a.src[q].stf + (size_t)j * 12, *r1 = r0 + 6;
    const float atime = (*a.step + 1) * a.dt;
    float out[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (atime > r0[2]) {
        const int type = (int)r0[0];
        float m[6];
        const float deg = 3.14159265358979323846f / 180.f;
        kin_mt(r1[0] * deg, r1[1] * deg, r1[2] * deg, m);
        float stf = 0.f;
        if (type == 1) stf = kin_brune(r0[3], atime - r0[2]);
        else if (type == 2) stf = kin_liu(r0[3], atime - r0[2], 0.3f);
        else if (type == 3) stf = kin_liu(r0[3], atime - r0[2], 0.2f);
        const int *ijk = a.src[q].ijk + 3 * j;
        const int c = a.g.idx(ijk[0], ijk[1], ijk[2]);
        float mu;
        switch (a.media_type) {
        case 1: mu = __bfloat162float(((const __nv_bfloat16 *)a.mu)[c]); break;
        case 2: mu = __half2float(((const __half *)a.mu)[c]) * a.mu_inv; break;
        default: mu = ((const float *)a.mu)[c];
        }
        stf *= r0[1] * r0[4] / mu;
        stf *= a.vtst;
        for (int v = 0; v < 6; ++v) out[v] = stf * m[v];
    }
    float *o = a.kin[q] + (size_t)j * 6;
    for (int v = 0; v < 6; ++v) o[v] = out[v];
}

/* applies the increments in subfault order (one thread per component), so
 * subfaults that share a cell add up in a fixed order */
__global__ void k_kin_apply(AwpPostArgs a)
{
    const int q = threadIdx.x;
    if (q >= a.ncomp) return;
    AwpComp &cp = a.comp[q];
    for (int j = 0; j < a.src[q].nsrc; ++j) {
        const int *ijk = a.src[q].ijk + 3 * j;
        const int c = a.g.idx(ijk[0], ijk[1], ijk[2]);
        const float *d = a.kin[q] + (size_t)j * 6;
        cp.f[AF_XX][c] = cp.f[AF_XX][c] - d[0];
        cp.f[AF_YY][c] = cp.f[AF_YY][c] - d[1];
        cp.f[AF_ZZ][c] = cp.f[AF_ZZ][c] - d[2];
        cp.f[AF_XZ][c] = cp.f[AF_XZ][c] - d[3];
        cp.f[AF_YZ][c] = cp.f[AF_YZ][c] - d[4];
        cp.f[AF_XY][c] = cp.f[AF_XY][c] - d[5];
    }
}

cudaError_t awp_launch_post(const AwpPostArgs &a, int initial, cudaStream_t st)
{
    if (a.kinematic && !initial) {
        int nmax = 0;
        for (int q = 0; q < a.ncomp; ++q) nmax = a.src[q].nsrc > nmax ? a.src[q].nsrc : nmax;
        if (nmax > 0) {
            k_kin_contrib<<<dim3((nmax + 127) / 128, a.ncomp), 128, 0, st>>>(a);
            k_kin_apply<<<1, 32, 0, st>>>(a);
        }
    }
    k_post<<<1, 32, 0, st>>>(a, initial);
    return cudaGetLastError();
}

/* RWG order of SGT file images, per point [6][nt]: XX <- YY, YY <- XX, ZZ,
 * XY, XZ <- -YZ, YZ <- -XZ, every value first scaled by -2 for the z-force
 * run (SgtHead/src/reformat_awp_mpi.c:85-122).  Scaling by -2 and -1 is
 * exact in FP32, so the result matches the reference's double products. */
__global__ void k_sgt_rwg(const float *__restrict__ in, float *__restrict__ out, int64_t total, int nt, int zsrc)
{
    const int64_t per = (int64_t)6 * nt;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = e / per;
        const int r = (int)(e - p * per);
        const int c = r / nt, t = r - c * nt;
        const int src = c == 0 ? 1 : (c == 1 ? 0 : (c == 4 ? 5 : (c == 5 ? 4 : c)));
        float v = in[p * per + (int64_t)src * nt + t];
        if (zsrc) v = -2.0f * v;
        if (c >= 4) v = -1.0f * v;
        out[e] = v;
    }
}

cudaError_t awp_launch_sgt_rwg(const float *in, float *out, int64_t npts, int nt, int zsrc, cudaStream_t st)
{
    const int64_t total = npts * 6 * (int64_t)nt;
    if (total <= 0) return cudaSuccess;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_sgt_rwg<<<(unsigned)blocks, 256, 0, st>>>(in, out, total, nt, zsrc);
    return cudaGetLastError();
}

/* RWG velocity volumes to the AWP media layout, one z-slab of n levels
 * (SgtHead/src/reformat_velocity.c:30-80): input [3][ny][n][nx] (p, s, d;
 * x fastest, then z, then y; km/s and g/cm^3), output [n][nx][ny][3] (y
 * fastest; m/s and kg/m^3, values times 1000).  A 32 x 32 (x, y) tile of all
 * three variables goes through shared memory so reads and writes coalesce.
 * The float product is the exact product rounded once, as the reference's
 * double product stored to float. */
__global__ void __launch_bounds__(256) k_rwg_slab(const float *__restrict__ rwg, float *__restrict__ awp, int nx,
                                                  int ny, int n)
{
    __shared__ float t[3][32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32, kk = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int v = 0; v < 3; ++v)
        for (int jj = ty; jj < 32; jj += 8) {
            const int i = i0 + tx, j = j0 + jj;
            if (i < nx && j < ny) t[v][jj][tx] = rwg[(((size_t)v * ny + j) * n + kk) * nx + i];
        }
    __syncthreads();
    /* one output row per x: 32 y values x 3 variables, contiguous */
    for (int ii = ty; ii < 32; ii += 8) {
        const int i = i0 + ii;
        if (i >= nx) continue;
        float *row = awp + (((size_t)kk * nx + i) * ny + j0) * 3;
        const int nyr = min(32, ny - j0);
        for (int e = tx; e < 3 * nyr; e += 32) {
            const int jj = e / 3, v = e - 3 * jj;
            row[e] = t[v][jj][ii] * 1000.0f;
        }
    }
}

cudaError_t awp_launch_rwg_slab(const float *rwg, float *awp, int nx, int ny, int n, cudaStream_t st)
{
    if (nx <= 0 || ny <= 0 || n <= 0) return cudaSuccess;
    k_rwg_slab<<<dim3((nx + 31) / 32, (ny + 31) / 32, n), dim3(32, 8), 0, st>>>(rwg, awp, nx, ny, n);
    return cudaGetLastError();
}

cudaError_t awp_launch_sgt(const AwpSgtArgs &a, cudaStream_t st)
{
    const int n = a.npts * a.ncomp;
    if (n <= 0) return cudaSuccess;
    k_sgt<<<(n + 255) / 256, 256, 0, st>>>(a);
    return cudaGetLastError();
}
