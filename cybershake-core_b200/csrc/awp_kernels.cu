/*
 * awp_kernels.cu -- sm_100a kernels of the AWP-ODC-SGT stepper (two-sweep form).
 *
 * Arithmetic follows the Fortran statement by statement with the same
 * evaluation order; this translation unit is compiled with --fmad=false so
 * every product and sum is rounded once, as in the FP32 CPU reference, and the
 * FP32 stepper reproduces it bit for bit.
 *
 * Kernels:
 *   k_media_interior  structure.f:449-533   media -> compliances + Q transform
 *   k_media_ghosts    structure.f:563-707   padmedia / afsmedia
 *   k_media_homo      structure.f:709-765   inihomo
 *   k_sg_coeffs       pmcl3d.f:1158-1171    sg1 sg2 sg3 at the SGT points
 *   k_vel<NC>         operator.f:92-244 + cerjan.f:292-330   velocity sweep
 *   k_fsvel<NC>       operator.f:246-306    free-surface velocity images
 *   k_str<NC>         viscoop.f:49-191 + cerjan.f:249-290 + operator.f:575-612
 *   k_post            source.f:812-913, pmcl3d.f:1379-1385, 1478-1479
 *   k_sgt             pmcl3d.f:1537-1557    SGT gather into the file image
 * NC = number of unit-force components stepped together (they share media).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "awp_internal.h"
#include "awp_kernels.h"

#define C1 (9.0f / 8.0f)
#define C2 (-(1.0f / 24.0f))

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

/* pmcl3d.f:1166-1168, evaluated at the SGT points only. */
__global__ void k_sg_coeffs(AwpGeom g, AwpMedia md, int npts, const int *__restrict__ pt_idx, float *sg)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= npts) return;
    const int c = pt_idx[n];
    const float lam = md.m[AM_LAM][c], mu = md.m[AM_MU][c];
    sg[3 * n] = (1.0f / lam + 1.0f / mu) / (1.0f / mu * (3.0f / lam + 2.0f / mu));
    sg[3 * n + 1] = -(1.0f / lam / (2.0f / mu * (3.0f / lam + 2.0f / mu)));
    sg[3 * n + 2] = mu;
}

/* ------------------------------------------------------------------ */
/* velocity sweep                                                      */
/* ------------------------------------------------------------------ */

template <int NC>
__global__ void __launch_bounds__(256)
k_vel(AwpGeom g, const float *__restrict__ d1, AwpCompSet<NC> cs,
      const float *__restrict__ cx, const float *__restrict__ cy, const float *__restrict__ cz,
      float dth, int kchunk)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.nx || j > g.ny) return;
    /* z chunks are aligned to the top so the top chunk always holds the
     * levels nz-2..nz that the fused fstr reads back */
    const int k1 = g.nz - ((int)gridDim.z - 1 - (int)blockIdx.z) * kchunk;
    const int k0 = max(1, k1 - kchunk + 1);
    const int sy = g.px, sz = g.plane;
    const float cxy = cx[i] * cy[j];
    for (int k = k0; k <= k1; ++k) {
        const int c = g.idx(i, j, k);
        const float da = d1[c], db = d1[c - sy], dc = d1[c - sz], dd = d1[c - sy - sz];
        const float de = d1[c + 1], df = d1[c + 1 - sz], dg = d1[c + 1 - sy];
        /* operator.f:120-121, 171-172, 224-225 */
        const float fu = dth / (0.25f * ((da + db) + (dc + dd)));
        const float fv = dth / (0.25f * ((da + de) + (dc + df)));
        const float fw = dth / (0.25f * ((da + de) + (db + dg)));
        const float crj = cxy * cz[k];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            float *__restrict__ u1 = cs.c[q].f[AF_U];
            float *__restrict__ v1 = cs.c[q].f[AF_V];
            float *__restrict__ w1 = cs.c[q].f[AF_W];
            const float *__restrict__ xx = cs.c[q].f[AF_XX];
            const float *__restrict__ yy = cs.c[q].f[AF_YY];
            const float *__restrict__ zz = cs.c[q].f[AF_ZZ];
            const float *__restrict__ xy = cs.c[q].f[AF_XY];
            const float *__restrict__ xz = cs.c[q].f[AF_XZ];
            const float *__restrict__ yz = cs.c[q].f[AF_YZ];
            const float u = u1[c] + fu * (
                C1 * (xx[c] - xx[c - 1]) + C2 * (xx[c + 1] - xx[c - 2]) +
                C1 * (xy[c] - xy[c - sy]) + C2 * (xy[c + sy] - xy[c - 2 * sy]) +
                C1 * (xz[c] - xz[c - sz]) + C2 * (xz[c + sz] - xz[c - 2 * sz]));
            const float v = v1[c] + fv * (
                C1 * (xy[c + 1] - xy[c]) + C2 * (xy[c + 2] - xy[c - 1]) +
                C1 * (yy[c + sy] - yy[c]) + C2 * (yy[c + 2 * sy] - yy[c - sy]) +
                C1 * (yz[c] - yz[c - sz]) + C2 * (yz[c + sz] - yz[c - 2 * sz]));
            const float w = w1[c] + fw * (
                C1 * (xz[c + 1] - xz[c]) + C2 * (xz[c + 2] - xz[c - 1]) +
                C1 * (yz[c] - yz[c - sy]) + C2 * (yz[c + sy] - yz[c - 2 * sy]) +
                C1 * (zz[c + sz] - zz[c]) + C2 * (zz[c + 2 * sz] - zz[c - sz]));
            /* Cerjan: the factor is exactly 1 outside the sponge zones */
            u1[c] = u * crj;
            v1[c] = v * crj;
            w1[c] = w * crj;
        }
    }
}

/* fvelxy then fvelz.  Each thread recomputes the two neighbouring fvelxy
 * values fvelz needs, so one launch covers both routines. */
template <int NC>
__global__ void k_fsvel(AwpGeom g, const float *__restrict__ lam, const float *__restrict__ mu, AwpCompSet<NC> cs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.nx || j > g.ny) return;
    const int nz = g.nz;
    const int c = g.idx(i, j, nz), sy = g.px, sz = g.plane;
    const float xl = 1.0f / lam[c];
    const float xl2m = 2.0f / mu[c] + xl;
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

/* ------------------------------------------------------------------ */
/* stress + memory-variable sweep                                      */
/* ------------------------------------------------------------------ */

template <int NC>
__global__ void __launch_bounds__(256)
k_str(AwpGeom g, AwpMedia md, AwpCompSet<NC> cs,
      const float *__restrict__ cx, const float *__restrict__ cy, const float *__restrict__ cz,
      const float *__restrict__ tau, float dth, float dt, float dh1, int kchunk, int nve, int fuse_fstr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.nx || j > g.ny) return;
    /* z chunks are aligned to the top so the top chunk always holds the
     * levels nz-2..nz that the fused fstr reads back */
    const int k1 = g.nz - ((int)gridDim.z - 1 - (int)blockIdx.z) * kchunk;
    const int k0 = max(1, k1 - kchunk + 1);
    const int sy = g.px, sz = g.plane;
    const float *__restrict__ lam = md.m[AM_LAM];
    const float *__restrict__ mu = md.m[AM_MU];
    const float *__restrict__ qp = md.m[AM_QP];
    const float *__restrict__ qs = md.m[AM_QS];
    const float cxy = cx[i] * cy[j];
    const int itxy = ((j & 1) << 1) | (i & 1);
    for (int k = k0; k <= k1; ++k) {
        const int c = g.idx(i, j, k);
        const int it = (((g.nz + 1 - k) & 1) << 2) | itxy;   /* viscoop.f:93-101 */
        const float vx1 = tau[it], vx2 = tau[8 + it];
        /* 8-cell harmonic / arithmetic averages, viscoop.f:104-124 */
        float xl = 8.0f / (lam[c] + lam[c + 1] + lam[c - sy] + lam[c + 1 - sy] +
                           lam[c - sz] + lam[c + 1 - sz] + lam[c - sy - sz] + lam[c + 1 - sy - sz]);
        const float xm = 8.0f / (mu[c] + mu[c + 1] + mu[c - sy] + mu[c + 1 - sy] +
                                 mu[c - sz] + mu[c + 1 - sz] + mu[c - sy - sz] + mu[c + 1 - sy - sz]);
        float qpa = 0.f, qsa = 0.f;
        if (nve == 1) {
            qpa = 0.125f * (qp[c] + qp[c + 1] + qp[c - sy] + qp[c + 1 - sy] +
                            qp[c - sz] + qp[c + 1 - sz] + qp[c - sy - sz] + qp[c + 1 - sy - sz]);
            qsa = 0.125f * (qs[c] + qs[c + 1] + qs[c - sy] + qs[c + 1 - sy] +
                            qs[c - sz] + qs[c + 1 - sz] + qs[c - sy - sz] + qs[c + 1 - sy - sz]);
        }
        const float xmu4 = 2.0f / (mu[c] + mu[c - sz]);
        const float xmu5 = 2.0f / (mu[c] + mu[c - sy]);
        const float xmu6 = 2.0f / (mu[c] + mu[c + 1]);
        const float crj = cxy * cz[k];
        if (nve == 1) {
            xl = xl + 2.0f * xm;
            const float aas4 = 0.5f * (qs[c] + qs[c - sz]);
            const float aas5 = 0.5f * (qs[c] + qs[c - sy]);
            const float aas6 = 0.5f * (qs[c] + qs[c + 1]);
            const float vh1 = -(xm * qsa);
            const float vh2_r4 = -(aas4 * xmu4 / 2.0f);
            const float vh2_r5 = -(aas5 * xmu5 / 2.0f);
            const float vh2_r6 = -(aas6 * xmu6 / 2.0f);
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const float *__restrict__ u1 = cs.c[q].f[AF_U];
                const float *__restrict__ v1 = cs.c[q].f[AF_V];
                const float *__restrict__ w1 = cs.c[q].f[AF_W];
                float *__restrict__ xx = cs.c[q].f[AF_XX];
                float *__restrict__ yy = cs.c[q].f[AF_YY];
                float *__restrict__ zz = cs.c[q].f[AF_ZZ];
                float *__restrict__ xy = cs.c[q].f[AF_XY];
                float *__restrict__ xz = cs.c[q].f[AF_XZ];
                float *__restrict__ yz = cs.c[q].f[AF_YZ];
                float *__restrict__ r1 = cs.c[q].f[AF_R1];
                float *__restrict__ r2 = cs.c[q].f[AF_R2];
                float *__restrict__ r3 = cs.c[q].f[AF_R3];
                float *__restrict__ r4 = cs.c[q].f[AF_R4];
                float *__restrict__ r5 = cs.c[q].f[AF_R5];
                float *__restrict__ r6 = cs.c[q].f[AF_R6];
                const float vt1 = C1 * (u1[c + 1] - u1[c]) + C2 * (u1[c + 2] - u1[c - 1]);
                const float vt2 = C1 * (v1[c] - v1[c - sy]) + C2 * (v1[c + sy] - v1[c - 2 * sy]);
                const float vt3 = C1 * (w1[c] - w1[c - sz]) + C2 * (w1[c + sz] - w1[c - 2 * sz]);
                const float vt4 = C1 * (u1[c + sy] - u1[c]) + C2 * (u1[c + 2 * sy] - u1[c - sy]) +
                                  C1 * (v1[c] - v1[c - 1]) + C2 * (v1[c + 1] - v1[c - 2]);
                const float vt5 = C1 * (u1[c + sz] - u1[c]) + C2 * (u1[c + 2 * sz] - u1[c - sz]) +
                                  C1 * (w1[c] - w1[c - 1]) + C2 * (w1[c + 1] - w1[c - 2]);
                const float vt6 = C1 * (v1[c + sz] - v1[c]) + C2 * (v1[c + 2 * sz] - v1[c - sz]);
                const float vt7 = C1 * (w1[c + sy] - w1[c]) + C2 * (w1[c + 2 * sy] - w1[c - sy]);
                const float vtmp = xl * (vt1 + vt2 + vt3);
                const float va1 = -(qpa * xl * dh1 * (vt1 + vt2 + vt3) / 2.0f);
                const float o1 = r1[c], o2 = r2[c], o3 = r3[c], o4 = r4[c], o5 = r5[c], o6 = r6[c];
                float sxx = xx[c] + dth * (vtmp - 2.0f * xm * (vt2 + vt3)) + dt * o1;
                float syy = yy[c] + dth * (vtmp - 2.0f * xm * (vt1 + vt3)) + dt * o2;
                float szz = zz[c] + dth * (vtmp - 2.0f * xm * (vt1 + vt2)) + dt * o3;
                float sxy = xy[c] + xmu4 * dth * vt4 + dt * o4;
                float sxz = xz[c] + xmu5 * dth * vt5 + dt * o5;
                float syz = yz[c] + xmu6 * (dth * vt6 + dth * vt7) + dt * o6;
                const float n1 = (vx2 * o1 - vh1 * (vt2 + vt3) * dh1 + va1) * vx1;
                const float n2 = (vx2 * o2 - vh1 * (vt1 + vt3) * dh1 + va1) * vx1;
                const float n3 = (vx2 * o3 - vh1 * (vt1 + vt2) * dh1 + va1) * vx1;
                const float n4 = (vx2 * o4 + vh2_r4 * dh1 * vt4) * vx1;
                const float n5 = (vx2 * o5 + vh2_r5 * dh1 * vt5) * vx1;
                const float n6 = (vx2 * o6 + vh2_r6 * dh1 * (vt6 + vt7)) * vx1;
                r1[c] = n1; r2[c] = n2; r3[c] = n3; r4[c] = n4; r5[c] = n5; r6[c] = n6;
                sxx = sxx + dt * n1;
                syy = syy + dt * n2;
                szz = szz + dt * n3;
                sxy = sxy + dt * n4;
                sxz = sxz + dt * n5;
                syz = syz + dt * n6;
                xx[c] = sxx * crj; yy[c] = syy * crj; zz[c] = szz * crj;
                xy[c] = sxy * crj; xz[c] = sxz * crj; yz[c] = syz * crj;
            }
        } else {
            /* elastic, operator.f:348-571 */
            const float a = xl + 2.0f * xm, b = xl;
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const float *__restrict__ u1 = cs.c[q].f[AF_U];
                const float *__restrict__ v1 = cs.c[q].f[AF_V];
                const float *__restrict__ w1 = cs.c[q].f[AF_W];
                float *__restrict__ xx = cs.c[q].f[AF_XX];
                float *__restrict__ yy = cs.c[q].f[AF_YY];
                float *__restrict__ zz = cs.c[q].f[AF_ZZ];
                float *__restrict__ xy = cs.c[q].f[AF_XY];
                float *__restrict__ xz = cs.c[q].f[AF_XZ];
                float *__restrict__ yz = cs.c[q].f[AF_YZ];
                const float u_a = C1 * (u1[c + 1] - u1[c]), u_b = C2 * (u1[c + 2] - u1[c - 1]);
                const float v_a = C1 * (v1[c] - v1[c - sy]), v_b = C2 * (v1[c + sy] - v1[c - 2 * sy]);
                const float w_a = C1 * (w1[c] - w1[c - sz]), w_b = C2 * (w1[c + sz] - w1[c - 2 * sz]);
                const float sxx = xx[c] + dth * a * (u_a + u_b) + dth * b * (v_a + v_b + w_a + w_b);
                const float syy = yy[c] + dth * a * (v_a + v_b) + dth * b * (u_a + u_b + w_a + w_b);
                const float szz = zz[c] + dth * a * (w_a + w_b) + dth * b * (u_a + u_b + v_a + v_b);
                const float sxy = xy[c] + dth * xmu4 * (C1 * (u1[c + sy] - u1[c]) + C2 * (u1[c + 2 * sy] - u1[c - sy]) +
                                                        C1 * (v1[c] - v1[c - 1]) + C2 * (v1[c + 1] - v1[c - 2]));
                const float sxz = xz[c] + dth * xmu5 * (C1 * (u1[c + sz] - u1[c]) + C2 * (u1[c + 2 * sz] - u1[c - sz]) +
                                                        C1 * (w1[c] - w1[c - 1]) + C2 * (w1[c + 1] - w1[c - 2]));
                const float syz = yz[c] + dth * xmu6 * (C1 * (v1[c + sz] - v1[c]) + C2 * (v1[c + 2 * sz] - v1[c - sz]) +
                                                        C1 * (w1[c + sy] - w1[c]) + C2 * (w1[c + 2 * sy] - w1[c - sy]));
                xx[c] = sxx * crj; yy[c] = syy * crj; zz[c] = szz * crj;
                xy[c] = sxy * crj; xz[c] = sxz * crj; yz[c] = syz * crj;
            }
        }
    }
    if (fuse_fstr && k1 == g.nz) {
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
    if (q < a.ncomp && sample <= a.nst) {
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
                cp.f[AF_U][c] = cp.f[AF_U][c] + axx * a.vtst / a.d1[c];
                break;
            case 2:
                cp.f[AF_V][c] = cp.f[AF_V][c] + ayy * a.vtst / a.d1[c];
                break;
            case 3:
                cp.f[AF_W][c] = cp.f[AF_W][c] + azz * a.vtst / a.d1[c];
                break;
            case -2:
                cp.f[AF_U][c] = cp.f[AF_U][c] + axx * a.vtst / a.d1[c];
                cp.f[AF_V][c] = cp.f[AF_V][c] + ayy * a.vtst / a.d1[c];
                cp.f[AF_W][c] = cp.f[AF_W][c] + azz * a.vtst / a.d1[c];
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

cudaError_t awp_launch_media_homo(const AwpGeom &g, const AwpMedia &md, float lam, float mu, float d1, cudaStream_t st)
{
    dim3 b(32, 8);
    dim3 gr((g.nx + 2 + b.x - 1) / b.x, (g.ny + 2 + b.y - 1) / b.y, g.nz + 2);
    k_media_homo<<<gr, b, 0, st>>>(g, md, lam, mu, d1);
    return cudaGetLastError();
}

cudaError_t awp_launch_sg_coeffs(const AwpGeom &g, const AwpMedia &md, int npts, const int *pt_idx, float *sg,
                                 cudaStream_t st)
{
    if (npts <= 0) return cudaSuccess;
    k_sg_coeffs<<<(npts + 255) / 256, 256, 0, st>>>(g, md, npts, pt_idx, sg);
    return cudaGetLastError();
}

template <int NC>
static cudaError_t launch_step_nc(const AwpStepArgs &s, cudaStream_t st)
{
    AwpCompSet<NC> cs;
    for (int q = 0; q < NC; ++q) cs.c[q] = s.comp[q];
    dim3 b(32, 8);
    const int nzb = (s.g.nz + s.kchunk - 1) / s.kchunk;
    k_vel<NC><<<plane_grid(s.g, b, nzb), b, 0, st>>>(s.g, s.md.m[AM_D1], cs, s.cx, s.cy, s.cz, s.dth, s.kchunk);
    k_fsvel<NC><<<plane_grid(s.g, b, 1), b, 0, st>>>(s.g, s.md.m[AM_LAM], s.md.m[AM_MU], cs);
    k_str<NC><<<plane_grid(s.g, b, nzb), b, 0, st>>>(s.g, s.md, cs, s.cx, s.cy, s.cz, s.tau, s.dth, s.dt, s.dh1,
                                                     s.kchunk, s.nve, 1);
    return cudaGetLastError();
}

cudaError_t awp_launch_step(const AwpStepArgs &s, cudaStream_t st)
{
    switch (s.ncomp) {
    case 1: return launch_step_nc<1>(s, st);
    case 2: return launch_step_nc<2>(s, st);
    case 3: return launch_step_nc<3>(s, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t awp_launch_post(const AwpPostArgs &a, int initial, cudaStream_t st)
{
    k_post<<<1, 32, 0, st>>>(a, initial);
    return cudaGetLastError();
}

cudaError_t awp_launch_sgt(const AwpSgtArgs &a, cudaStream_t st)
{
    const int n = a.npts * a.ncomp;
    if (n <= 0) return cudaSuccess;
    k_sgt<<<(n + 255) / 256, 256, 0, st>>>(a);
    return cudaGetLastError();
}
