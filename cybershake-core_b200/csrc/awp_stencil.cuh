/*
 * awp_stencil.cuh -- the per-cell arithmetic of the stepper, shared by the
 * two-sweep kernels and the fused kernel so every stepper evaluates the same
 * expressions in the same order (operator.f:92-244, viscoop.f:49-191,
 * operator.f:348-571, cerjan.f:292-330).
 *
 * Storage types: media arrays (lam, mu, d1, qp, qs) are TM = float, bf16 or
 * binary16 (scaled by a power of two, so the scaling is exact); the memory
 * variables r1..r6 are TR = float or bf16.  Every value is widened to FP32
 * before any arithmetic.
 */
#ifndef AWP_STENCIL_CUH
#define AWP_STENCIL_CUH

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "awp_internal.h"

/* Work items of the persistent steppers: (x tile, y tile, z chunk), x
 * fastest so that blocks running together hold neighbouring tiles.  Every
 * block walks items blockIdx.x, +gridDim.x, ...  z chunks are aligned to the
 * top, so the top chunk always holds the levels nz-2..nz that fstr reads. */
struct AwpWork {
    int ntx, nty, nzc, kchunk, nitems;
};

__device__ __forceinline__ void work_item(const AwpGeom &g, const AwpWork &w, int item, int &bx, int &by, int &k0,
                                          int &k1)
{
    bx = item % w.ntx;
    const int t = item / w.ntx;
    by = t % w.nty;
    const int bz = t / w.nty;
    k1 = g.nz - (w.nzc - 1 - bz) * w.kchunk;
    k0 = max(1, k1 - w.kchunk + 1);
}

#define C1 (9.0f / 8.0f)
#define C2 (-(1.0f / 24.0f))

/* Stores go to global memory through __stwb (a global store with the
 * default write-back policy): some kernels keep their array pointers in a
 * shared-memory table, and a store through such a pointer would otherwise be
 * a generic one. */
template <class T> struct Store;
template <> struct Store<float> {
    static __device__ __forceinline__ float ld(const float *p, int c, float) { return p[c]; }
    static __device__ __forceinline__ void st(float *p, int c, float v, float) { __stwb(p + c, v); }
};
template <> struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16 *p, int c, float) { return __bfloat162float(p[c]); }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, int c, float v, float) { __stwb(p + c, __float2bfloat16_rn(v)); }
};
/* binary16 arrays hold value * 2^e; ld multiplies by inv = 2^-e (exact) */
template <> struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half *p, int c, float inv) { return __half2float(p[c]) * inv; }
    static __device__ __forceinline__ void st(__half *p, int c, float v, float scale) { __stwb(p + c, __float2half_rn(v * scale)); }
};

/* 16-bit block floating point of r1..r6 (AWP_STORE_BFP; the rule is stated
 * in awp_internal.h).  RBfp is the storage tag of the steppers' templates. */
struct RBfp {};

/* encodes three values; returns the exponent byte */
__device__ __forceinline__ uint32_t bfp_enc3(float a, float b, float c, short &ma, short &mb, short &mc)
{
    const float mx = fmaxf(fabsf(a), fmaxf(fabsf(b), fabsf(c)));
    const uint32_t e = __float_as_uint(mx) >> 23;
    if (e < AWP_BFP_EMIN) {
        ma = mb = mc = 0;
        return 0u;
    }
    const float up = __uint_as_float((268u - e) << 23);
    ma = (short)__float2int_rn(fminf(fmaxf(a * up, -32767.f), 32767.f));
    mb = (short)__float2int_rn(fminf(fmaxf(b * up, -32767.f), 32767.f));
    mc = (short)__float2int_rn(fminf(fmaxf(c * up, -32767.f), 32767.f));
    return e;
}

/* decodes three values of exponent byte e */
__device__ __forceinline__ void bfp_dec3(uint32_t e, short ma, short mb, short mc, float &a, float &b, float &c)
{
    const float down = __uint_as_float((max(e, AWP_BFP_EMIN) - 14u) << 23);
    a = (float)ma * down;
    b = (float)mb * down;
    c = (float)mc * down;
}

/* the six memory variables of a cell from their storage (m: the mantissa
 * arrays at the cell, stride apart; x: the exponent word) */
__device__ __forceinline__ void bfp_load6(const short *m, int stride, uint32_t x, float r[6])
{
    bfp_dec3(x & 0xffu, m[0], m[stride], m[2 * stride], r[0], r[1], r[2]);
    bfp_dec3(x >> 8, m[3 * stride], m[4 * stride], m[5 * stride], r[3], r[4], r[5]);
}

/* memory variables r1..r6 of one cell in global memory, by storage type */
template <class TR>
struct RVars {
    static __device__ __forceinline__ void ld(const AwpComp &o, int c, float r[6])
    {
#pragma unroll
        for (int a = 0; a < 6; ++a) r[a] = Store<TR>::ld((const TR *)o.f[AF_R1 + a], c, 1.0f);
    }
    static __device__ __forceinline__ void st(const AwpComp &o, int c, const float r[6])
    {
#pragma unroll
        for (int a = 0; a < 6; ++a) Store<TR>::st((TR *)o.f[AF_R1 + a], c, r[a], 1.0f);
    }
};
template <>
struct RVars<RBfp> {
    static __device__ __forceinline__ void ld(const AwpComp &o, int c, float r[6])
    {
        const uint32_t x = ((const unsigned short *)o.f[AF_RX])[c];
        bfp_dec3(x & 0xffu, ((const short *)o.f[AF_R1])[c], ((const short *)o.f[AF_R2])[c],
                 ((const short *)o.f[AF_R3])[c], r[0], r[1], r[2]);
        bfp_dec3(x >> 8, ((const short *)o.f[AF_R4])[c], ((const short *)o.f[AF_R5])[c],
                 ((const short *)o.f[AF_R6])[c], r[3], r[4], r[5]);
    }
    static __device__ __forceinline__ void st(const AwpComp &o, int c, const float r[6])
    {
        short m[6];
        const uint32_t e0 = bfp_enc3(r[0], r[1], r[2], m[0], m[1], m[2]);
        const uint32_t e1 = bfp_enc3(r[3], r[4], r[5], m[3], m[4], m[5]);
#pragma unroll
        for (int a = 0; a < 6; ++a) __stwb((short *)o.f[AF_R1 + a] + c, m[a]);
        __stwb((unsigned short *)o.f[AF_RX] + c, (unsigned short)(e0 | (e1 << 8)));
    }
};

/* typed view of the media arrays */
template <class TM>
struct MediaT {
    const TM *m[AM_N];
    float inv[AM_N];
    __device__ __forceinline__ float operator()(int a, int c) const { return Store<TM>::ld(m[a], c, inv[a]); }
};

/* ------------------------------------------------------------------ */
/* velocity update of one cell (all NC components)                    */
/* ------------------------------------------------------------------ */

/* d1 averages of operator.f:120-121, 171-172, 224-225 -> dth/d, from the
 * seven d1 values around the cell: a (0,0,0) b (0,-1,0) c (0,0,-1)
 * d (0,-1,-1) e (1,0,0) f (1,0,-1) g (1,-1,0) */
__device__ __forceinline__ void vel_factors7(float da, float db, float dc, float dd, float de, float df, float dg,
                                             float dth, float &fu, float &fv, float &fw)
{
    fu = dth / (0.25f * ((da + db) + (dc + dd)));
    fv = dth / (0.25f * ((da + de) + (dc + df)));
    fw = dth / (0.25f * ((da + de) + (db + dg)));
}

template <class TM>
__device__ __forceinline__ void vel_factors(const MediaT<TM> &md, int c, int sy, int sz, float dth,
                                            float &fu, float &fv, float &fw)
{
    const float da = md(AM_D1, c), db = md(AM_D1, c - sy), dc = md(AM_D1, c - sz), dd = md(AM_D1, c - sy - sz);
    const float de = md(AM_D1, c + 1), df = md(AM_D1, c + 1 - sz), dg = md(AM_D1, c + 1 - sy);
    vel_factors7(da, db, dc, dd, de, df, dg, dth, fu, fv, fw);
}

/* stress indices of the accessors below */
enum { S_XX = 0, S_YY = 1, S_ZZ = 2, S_XY = 3, S_XZ = 4, S_YZ = 5 };

/* new (u, v, w) of one component, before the sponge factor; A::s(f, dx, dy,
 * dz) is stress f at the offset (operator.f:122-132, 173-183, 226-236) */
template <class A>
__device__ __forceinline__ void vel_one_t(const A &S, float u0, float v0, float w0, float fu, float fv, float fw,
                                          float &u, float &v, float &w)
{
    u = u0 + fu * (
        C1 * (S.s(S_XX, 0, 0, 0) - S.s(S_XX, -1, 0, 0)) + C2 * (S.s(S_XX, 1, 0, 0) - S.s(S_XX, -2, 0, 0)) +
        C1 * (S.s(S_XY, 0, 0, 0) - S.s(S_XY, 0, -1, 0)) + C2 * (S.s(S_XY, 0, 1, 0) - S.s(S_XY, 0, -2, 0)) +
        C1 * (S.s(S_XZ, 0, 0, 0) - S.s(S_XZ, 0, 0, -1)) + C2 * (S.s(S_XZ, 0, 0, 1) - S.s(S_XZ, 0, 0, -2)));
    v = v0 + fv * (
        C1 * (S.s(S_XY, 1, 0, 0) - S.s(S_XY, 0, 0, 0)) + C2 * (S.s(S_XY, 2, 0, 0) - S.s(S_XY, -1, 0, 0)) +
        C1 * (S.s(S_YY, 0, 1, 0) - S.s(S_YY, 0, 0, 0)) + C2 * (S.s(S_YY, 0, 2, 0) - S.s(S_YY, 0, -1, 0)) +
        C1 * (S.s(S_YZ, 0, 0, 0) - S.s(S_YZ, 0, 0, -1)) + C2 * (S.s(S_YZ, 0, 0, 1) - S.s(S_YZ, 0, 0, -2)));
    w = w0 + fw * (
        C1 * (S.s(S_XZ, 1, 0, 0) - S.s(S_XZ, 0, 0, 0)) + C2 * (S.s(S_XZ, 2, 0, 0) - S.s(S_XZ, -1, 0, 0)) +
        C1 * (S.s(S_YZ, 0, 0, 0) - S.s(S_YZ, 0, -1, 0)) + C2 * (S.s(S_YZ, 0, 1, 0) - S.s(S_YZ, 0, -2, 0)) +
        C1 * (S.s(S_ZZ, 0, 0, 1) - S.s(S_ZZ, 0, 0, 0)) + C2 * (S.s(S_ZZ, 0, 0, 2) - S.s(S_ZZ, 0, 0, -1)));
}

/* stresses of one component in global memory */
struct GStr {
    const float *__restrict__ f[6];
    int c, sy, sz;
    __device__ __forceinline__ float s(int a, int dx, int dy, int dz) const { return f[a][c + dx + dy * sy + dz * sz]; }
};

__device__ __forceinline__ void vel_one(const AwpComp &o, int c, int sy, int sz, float fu, float fv, float fw,
                                        float &u, float &v, float &w)
{
    const GStr S{{o.f[AF_XX], o.f[AF_YY], o.f[AF_ZZ], o.f[AF_XY], o.f[AF_XZ], o.f[AF_YZ]}, c, sy, sz};
    vel_one_t(S, o.f[AF_U][c], o.f[AF_V][c], o.f[AF_W][c], fu, fv, fw, u, v, w);
}

/* ------------------------------------------------------------------ */
/* stress + memory variables of one cell                              */
/* ------------------------------------------------------------------ */

/* cell coefficients shared by all components (viscoop.f:104-124, 151-167) */
struct StrCoef {
    float xl, xm, qpa, vh1, xmu4, xmu5, xmu6, vh2_r4, vh2_r5, vh2_r6, vx1, vx2;
};

/* A::m(a, dx, dy, dz) is media array a at the offset */
template <class A>
__device__ __forceinline__ StrCoef str_coef_t(const A &M, int nve, float vx1, float vx2)
{
    StrCoef k;
    k.xl = 8.0f / (M.m(AM_LAM, 0, 0, 0) + M.m(AM_LAM, 1, 0, 0) + M.m(AM_LAM, 0, -1, 0) + M.m(AM_LAM, 1, -1, 0) +
                   M.m(AM_LAM, 0, 0, -1) + M.m(AM_LAM, 1, 0, -1) + M.m(AM_LAM, 0, -1, -1) + M.m(AM_LAM, 1, -1, -1));
    k.xm = 8.0f / (M.m(AM_MU, 0, 0, 0) + M.m(AM_MU, 1, 0, 0) + M.m(AM_MU, 0, -1, 0) + M.m(AM_MU, 1, -1, 0) +
                   M.m(AM_MU, 0, 0, -1) + M.m(AM_MU, 1, 0, -1) + M.m(AM_MU, 0, -1, -1) + M.m(AM_MU, 1, -1, -1));
    const float mu0 = M.m(AM_MU, 0, 0, 0);
    k.xmu4 = 2.0f / (mu0 + M.m(AM_MU, 0, 0, -1));
    k.xmu5 = 2.0f / (mu0 + M.m(AM_MU, 0, -1, 0));
    k.xmu6 = 2.0f / (mu0 + M.m(AM_MU, 1, 0, 0));
    k.vx1 = vx1;
    k.vx2 = vx2;
    if (nve == 1) {
        k.qpa = 0.125f * (M.m(AM_QP, 0, 0, 0) + M.m(AM_QP, 1, 0, 0) + M.m(AM_QP, 0, -1, 0) + M.m(AM_QP, 1, -1, 0) +
                          M.m(AM_QP, 0, 0, -1) + M.m(AM_QP, 1, 0, -1) + M.m(AM_QP, 0, -1, -1) + M.m(AM_QP, 1, -1, -1));
        const float qsa = 0.125f * (M.m(AM_QS, 0, 0, 0) + M.m(AM_QS, 1, 0, 0) + M.m(AM_QS, 0, -1, 0) +
                                    M.m(AM_QS, 1, -1, 0) + M.m(AM_QS, 0, 0, -1) + M.m(AM_QS, 1, 0, -1) +
                                    M.m(AM_QS, 0, -1, -1) + M.m(AM_QS, 1, -1, -1));
        k.xl = k.xl + 2.0f * k.xm;
        const float qs0 = M.m(AM_QS, 0, 0, 0);
        const float aas4 = 0.5f * (qs0 + M.m(AM_QS, 0, 0, -1));
        const float aas5 = 0.5f * (qs0 + M.m(AM_QS, 0, -1, 0));
        const float aas6 = 0.5f * (qs0 + M.m(AM_QS, 1, 0, 0));
        k.vh1 = -(k.xm * qsa);
        k.vh2_r4 = -(aas4 * k.xmu4 / 2.0f);
        k.vh2_r5 = -(aas5 * k.xmu5 / 2.0f);
        k.vh2_r6 = -(aas6 * k.xmu6 / 2.0f);
    } else {
        k.qpa = k.vh1 = k.vh2_r4 = k.vh2_r5 = k.vh2_r6 = 0.f;
    }
    return k;
}

/* media in global memory around cell c */
template <class TM>
struct GMed {
    const MediaT<TM> &md;
    int c, sy, sz;
    __device__ __forceinline__ float m(int a, int dx, int dy, int dz) const { return md(a, c + dx + dy * sy + dz * sz); }
};

template <class TM>
__device__ __forceinline__ StrCoef str_coef(const MediaT<TM> &md, int c, int sy, int sz, int nve,
                                            float vx1, float vx2)
{
    const GMed<TM> M{md, c, sy, sz};
    return str_coef_t(M, nve, vx1, vx2);
}

/* velocity differences of viscoop.f:126-134; A provides u/v/w at offsets */
struct VelDiff {
    float vt1, vt2, vt3, vt4, vt5, vt6, vt7;
};

template <class A>
__device__ __forceinline__ VelDiff vel_diff(const A &V)
{
    VelDiff d;
    d.vt1 = C1 * (V.u(1, 0, 0) - V.u(0, 0, 0)) + C2 * (V.u(2, 0, 0) - V.u(-1, 0, 0));
    d.vt2 = C1 * (V.v(0, 0, 0) - V.v(0, -1, 0)) + C2 * (V.v(0, 1, 0) - V.v(0, -2, 0));
    d.vt3 = C1 * (V.w(0, 0, 0) - V.w(0, 0, -1)) + C2 * (V.w(0, 0, 1) - V.w(0, 0, -2));
    d.vt4 = C1 * (V.u(0, 1, 0) - V.u(0, 0, 0)) + C2 * (V.u(0, 2, 0) - V.u(0, -1, 0)) +
            C1 * (V.v(0, 0, 0) - V.v(-1, 0, 0)) + C2 * (V.v(1, 0, 0) - V.v(-2, 0, 0));
    d.vt5 = C1 * (V.u(0, 0, 1) - V.u(0, 0, 0)) + C2 * (V.u(0, 0, 2) - V.u(0, 0, -1)) +
            C1 * (V.w(0, 0, 0) - V.w(-1, 0, 0)) + C2 * (V.w(1, 0, 0) - V.w(-2, 0, 0));
    d.vt6 = C1 * (V.v(0, 0, 1) - V.v(0, 0, 0)) + C2 * (V.v(0, 0, 2) - V.v(0, 0, -1));
    d.vt7 = C1 * (V.w(0, 1, 0) - V.w(0, 0, 0)) + C2 * (V.w(0, 2, 0) - V.w(0, -1, 0));
    return d;
}

struct Stress6 {
    float xx, yy, zz, xy, xz, yz;
};

/* viscoelastic update (viscoop.f:136-185): old stresses s, old memory
 * variables r[6] (overwritten with the new ones), returns the new stresses
 * before the sponge factor */
__device__ __forceinline__ Stress6 str_visco(const StrCoef &k, const VelDiff &d, const Stress6 &s, float r[6],
                                             float dth, float dt, float dh1)
{
    const float vtmp = k.xl * (d.vt1 + d.vt2 + d.vt3);
    const float va1 = -(k.qpa * k.xl * dh1 * (d.vt1 + d.vt2 + d.vt3) / 2.0f);
    Stress6 o;
    o.xx = s.xx + dth * (vtmp - 2.0f * k.xm * (d.vt2 + d.vt3)) + dt * r[0];
    o.yy = s.yy + dth * (vtmp - 2.0f * k.xm * (d.vt1 + d.vt3)) + dt * r[1];
    o.zz = s.zz + dth * (vtmp - 2.0f * k.xm * (d.vt1 + d.vt2)) + dt * r[2];
    o.xy = s.xy + k.xmu4 * dth * d.vt4 + dt * r[3];
    o.xz = s.xz + k.xmu5 * dth * d.vt5 + dt * r[4];
    o.yz = s.yz + k.xmu6 * (dth * d.vt6 + dth * d.vt7) + dt * r[5];
    r[0] = (k.vx2 * r[0] - k.vh1 * (d.vt2 + d.vt3) * dh1 + va1) * k.vx1;
    r[1] = (k.vx2 * r[1] - k.vh1 * (d.vt1 + d.vt3) * dh1 + va1) * k.vx1;
    r[2] = (k.vx2 * r[2] - k.vh1 * (d.vt1 + d.vt2) * dh1 + va1) * k.vx1;
    r[3] = (k.vx2 * r[3] + k.vh2_r4 * dh1 * d.vt4) * k.vx1;
    r[4] = (k.vx2 * r[4] + k.vh2_r5 * dh1 * d.vt5) * k.vx1;
    r[5] = (k.vx2 * r[5] + k.vh2_r6 * dh1 * (d.vt6 + d.vt7)) * k.vx1;
    o.xx = o.xx + dt * r[0];
    o.yy = o.yy + dt * r[1];
    o.zz = o.zz + dt * r[2];
    o.xy = o.xy + dt * r[3];
    o.xz = o.xz + dt * r[4];
    o.yz = o.yz + dt * r[5];
    return o;
}

/* elastic update (operator.f:389-426, 464-470, 509-515, 559-565) */
template <class A>
__device__ __forceinline__ Stress6 str_elastic(const StrCoef &k, const A &V, const Stress6 &s, float dth)
{
    const float a = k.xl + 2.0f * k.xm, b = k.xl;
    const float u_a = C1 * (V.u(1, 0, 0) - V.u(0, 0, 0)), u_b = C2 * (V.u(2, 0, 0) - V.u(-1, 0, 0));
    const float v_a = C1 * (V.v(0, 0, 0) - V.v(0, -1, 0)), v_b = C2 * (V.v(0, 1, 0) - V.v(0, -2, 0));
    const float w_a = C1 * (V.w(0, 0, 0) - V.w(0, 0, -1)), w_b = C2 * (V.w(0, 0, 1) - V.w(0, 0, -2));
    Stress6 o;
    o.xx = s.xx + dth * a * (u_a + u_b) + dth * b * (v_a + v_b + w_a + w_b);
    o.yy = s.yy + dth * a * (v_a + v_b) + dth * b * (u_a + u_b + w_a + w_b);
    o.zz = s.zz + dth * a * (w_a + w_b) + dth * b * (u_a + u_b + v_a + v_b);
    o.xy = s.xy + dth * k.xmu4 * (C1 * (V.u(0, 1, 0) - V.u(0, 0, 0)) + C2 * (V.u(0, 2, 0) - V.u(0, -1, 0)) +
                                  C1 * (V.v(0, 0, 0) - V.v(-1, 0, 0)) + C2 * (V.v(1, 0, 0) - V.v(-2, 0, 0)));
    o.xz = s.xz + dth * k.xmu5 * (C1 * (V.u(0, 0, 1) - V.u(0, 0, 0)) + C2 * (V.u(0, 0, 2) - V.u(0, 0, -1)) +
                                  C1 * (V.w(0, 0, 0) - V.w(-1, 0, 0)) + C2 * (V.w(1, 0, 0) - V.w(-2, 0, 0)));
    o.yz = s.yz + dth * k.xmu6 * (C1 * (V.v(0, 0, 1) - V.v(0, 0, 0)) + C2 * (V.v(0, 0, 2) - V.v(0, 0, -1)) +
                                  C1 * (V.w(0, 1, 0) - V.w(0, 0, 0)) + C2 * (V.w(0, 2, 0) - V.w(0, -1, 0)));
    return o;
}

/* velocity accessor over global arrays (two-sweep stress kernel) */
struct GVel {
    const float *__restrict__ U;
    const float *__restrict__ Vv;
    const float *__restrict__ W;
    int c, sy, sz;
    __device__ __forceinline__ float u(int dx, int dy, int dz) const { return U[c + dx + dy * sy + dz * sz]; }
    __device__ __forceinline__ float v(int dx, int dy, int dz) const { return Vv[c + dx + dy * sy + dz * sz]; }
    __device__ __forceinline__ float w(int dx, int dy, int dz) const { return W[c + dx + dy * sy + dz * sz]; }
};

#endif
