/*
 * awp_synth.cu -- reciprocity seismogram synthesis on the device: the SGT
 * set resident in HBM, every variation of a rupture synthesised in one pass.
 *
 * Work split (one "term" = variation x rupture point x slip component):
 *   host (awp_synth_plan.c): bracketing SGT points, mechanism coefficients,
 *     shifts, dt-scaled slip rates -- O(1) per term;
 *   k_synth_gf: per term and output sample, the mechanism-weighted,
 *     rotated, tapered and shifted sum over the bracketing SGT points
 *     (mech_sgt + timeshift_sgt, DirectSynth/src/jbsim/sgt3d_subs.c:1173-1422)
 *     into a term buffer u[slot][3][ntout];
 *   k_synth_conv: per variation, component and block of output samples, the
 *     convolution of every term with its slip rate, accumulated in rupture
 *     point order (srf_stf / do_cnvlv, jbsim/srf_rupm.c:148-151,
 *     jbsim/stf_subs.c:6-40).
 * The terms of a batch are laid out point-major (all variations of a point
 * next to each other) so that the SGT rows of a point are read from HBM once
 * and served from L2 to the other variations.  Points are taken in chunks
 * whose terms fit the term buffer; the seismograms stay in device memory
 * between chunks.
 *
 * Compiled with --fmad=false: every multiply and add rounds once, in the
 * reference's order, so the seismograms equal the C reference's bit for bit.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <omp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <chrono>
#include <vector>

#include "awp_synth_internal.h"

extern "C" void awp_set_error_text(const char *msg);

namespace {

awp_status fail(awp_status st, const char *fmt, ...)
{
    char b[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b, sizeof b, fmt, ap);
    va_end(ap);
    awp_set_error_text(b);
    return st;
}

#define SCU(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(AWP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

constexpr int GF_THREADS = 256;
constexpr int CV_THREADS = 128;
constexpr int CV_BLOCK = CV_THREADS * 8;   /* output samples of one convolution CTA */

__constant__ float c_taper[SY_TAPLEN];

/* ---- kernel 1: per term, the shifted sum of the bracketing SGTs --------- */

/* u holds UC component traces per slot: vertical, north, east when the SGTs
 * have three components, else north and east only -- with no z SGT the
 * vertical trace is +0 throughout (zero rows times a zero amplitude, added
 * to +0), and so is its convolution, which the zeroed seismogram already
 * holds. */

template <int NC>
__device__ __forceinline__ void gf_load(const float *__restrict__ b, int nt, float *a, float *y, float *z)
{
#pragma unroll
    for (int r = 0; r < 6; r++) {
        a[r] = __ldg(b + (size_t)r * nt);
        y[r] = NC > 1 ? __ldg(b + (size_t)(6 + r) * nt) : 0.0f;
        z[r] = NC > 2 ? __ldg(b + (size_t)(12 + r) * nt) : 0.0f;
    }
}

/* sgt3d_subs.c:1393-1406: left-to-right sums, amplitude last, then the
 * rotation to north / east */
__device__ __forceinline__ void gf_combine(const float *a, const float *y, const float *z, const float *k, float &gv,
                                           float &gn, float &ge)
{
    const float sx = k[SY_XAMP] * (a[0] * k[SY_MXX] + a[1] * k[SY_MYY] + a[2] * k[SY_MZZ] + a[3] * k[SY_MXY] +
                                   a[4] * k[SY_MXZ] + a[5] * k[SY_MYZ]);
    const float sy = k[SY_YAMP] * (y[0] * k[SY_MXX] + y[1] * k[SY_MYY] + y[2] * k[SY_MZZ] + y[3] * k[SY_MXY] +
                                   y[4] * k[SY_MXZ] + y[5] * k[SY_MYZ]);
    const float sz = k[SY_ZAMP] * (z[0] * k[SY_MXX] + z[1] * k[SY_MYY] + z[2] * k[SY_MZZ] + z[3] * k[SY_MXY] +
                                   z[4] * k[SY_MXZ] + z[5] * k[SY_MYZ]);
    ge = sx * k[SY_SINA] + sy * k[SY_COSA];
    gn = sx * k[SY_COSA] - sy * k[SY_SINA];
    gv = -sz;
}

/* terms whose rupture point sits between SGT points (2-4 brackets): one
 * block per (listed slot, 256 output samples), every output sample written */
template <int NC, int UC>
__global__ void __launch_bounds__(GF_THREADS) k_synth_gf(const float *__restrict__ sgt, int nt, int tapst,
                                                         const awp_synth_gterm *__restrict__ gt,
                                                         const int *__restrict__ slot_term,
                                                         const int *__restrict__ slots, int ntout,
                                                         float *__restrict__ u)
{
    __shared__ awp_synth_gterm g;
    const int slot = slots[blockIdx.x];
    if (threadIdx.x == 0) g = gt[slot_term[slot]];
    __syncthreads();
    const int i = blockIdx.y * GF_THREADS + threadIdx.x;
    if (i >= ntout) return;
    float uv = 0.0f, un = 0.0f, ue = 0.0f;
    for (int ig = 0; ig < g.nsgt; ig++) {
        if (i < g.lo[ig] || i >= g.hi[ig]) continue;
        const int j = i - g.shift[ig];
        float a[6], y[6], z[6], gv, gn, ge;
        gf_load<NC>(sgt + (size_t)g.pt[ig] * (6 * NC) * nt + j, nt, a, y, z);
        gf_combine(a, y, z, g.c[ig], gv, gn, ge);
        if (j > tapst) {                   /* sgt3d_subs.c:1206-1212 */
            const float f = c_taper[j - tapst];
            gv = f * gv;
            gn = f * gn;
            ge = f * ge;
        }
        uv = uv + gv;                      /* sgt3d_subs.c:1237-1254 */
        un = un + gn;
        ue = ue + ge;
    }
    float *o = u + (size_t)slot * UC * ntout + i;
    if (UC == 3) *o = uv, o += ntout;
    o[0] = un;
    o[ntout] = ue;
}

/* rupture points with an exact SGT match: one block per (point, 256 SGT
 * samples).  Each thread loads its SGT sample once and applies every term of
 * the point (all variations and slip components) to it, writing output
 * sample j + shift of each term inside the term's coverage; samples outside
 * it are +0 and the convolution supplies them.  The terms' coefficients are
 * staged in shared memory 64 at a time. */
constexpr int GF1_TERMS = 64;

template <int NC, int UC>
__global__ void __launch_bounds__(GF_THREADS) k_synth_gf1(const float *__restrict__ sgt, int nt, int tapst,
                                                          const awp_synth_gterm *__restrict__ gt,
                                                          const int *__restrict__ slot_term,
                                                          const int4 *__restrict__ groups, int ntout,
                                                          float *__restrict__ u)
{
    __shared__ float4 rec[GF1_TERMS][4];
    const int4 grp = groups[blockIdx.y];               /* SGT point, first slot, slots */
    const int j = blockIdx.x * GF_THREADS + threadIdx.x;
    float a[6], y[6], z[6];
    float f = 1.0f;
    if (j < nt) {
        gf_load<NC>(sgt + (size_t)grp.x * (6 * NC) * nt + j, nt, a, y, z);
        if (j > tapst) f = c_taper[j - tapst];         /* sgt3d_subs.c:1206-1212; 1 * g is g */
    }
    for (int t0 = 0; t0 < grp.z; t0 += GF1_TERMS) {
        const int nterm = grp.z - t0 < GF1_TERMS ? grp.z - t0 : GF1_TERMS;
        __syncthreads();
        for (int e = threadIdx.x; e < nterm * 16; e += GF_THREADS) {
            const int tt = e >> 4, w = e & 15;
            const awp_synth_gterm *g = gt + slot_term[grp.y + t0 + tt];
            float v = 0.0f;
            if (w < SY_NC) v = g->c[0][w];
            else if (w == SY_NC) v = __int_as_float(g->shift[0]);
            else if (w == SY_NC + 1) v = __int_as_float(g->lo[0]);
            else if (w == SY_NC + 2) v = __int_as_float(g->hi[0]);
            reinterpret_cast<float *>(rec[tt])[w] = v;
        }
        __syncthreads();
        if (j >= nt) continue;
        for (int tt = 0; tt < nterm; tt++) {
            float k[16];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float4 r = rec[tt][q];
                k[4 * q] = r.x, k[4 * q + 1] = r.y, k[4 * q + 2] = r.z, k[4 * q + 3] = r.w;
            }
            const int i = j + __float_as_int(k[SY_NC]);
            if (i < __float_as_int(k[SY_NC + 1]) || i >= __float_as_int(k[SY_NC + 2])) continue;
            float gv, gn, ge;
            gf_combine(a, y, z, k, gv, gn, ge);
            float *o = u + (size_t)(grp.y + t0 + tt) * UC * ntout + i;
            if (UC == 3) *o = 0.0f + f * gv, o += ntout;    /* sgt3d_subs.c:1237-1254 */
            o[0] = 0.0f + f * gn;
            o[ntout] = 0.0f + f * ge;
        }
    }
}

/* ---- kernel 2: slip-rate convolution, terms in rupture-point order ------- */

__device__ __forceinline__ void cp_async4(float *dst, const float *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

/* Each CTA owns CV_BLOCK consecutive output samples (8 per thread) of one
 * component of one variation and walks the variation's terms in
 * rupture-point order.  The window of term n + 1 (its trace around the block
 * and its slip rate) is copied into the other shared buffer with cp.async
 * while term n is convolved; term records are read two terms ahead.
 *
 * Inside a term, thread samples W[j] = window[8 tid + j] feed its outputs
 * q = 0..7 at lag k through W[q + m], m = n8 - 1 - k.  Lags go in groups of
 * eight (m = 8g+7 .. 8g, g descending): a group needs W[8g .. 8g+14], held
 * as lo = W[8g..8g+7] and hi = W[8g+8..8g+15], and loads the next group's lo
 * while it computes.  Three register sets take the lo / hi / next roles in
 * turn (the loop is unrolled three times), so no window value is moved.
 * W[8g + j] sits in shared row j at column tid + g (rows STRIDE apart,
 * STRIDE = 4 mod 32), so the loads of a warp hit 32 banks and their offsets
 * are immediates. */
template <int STRIDE, int UC>
__global__ void __launch_bounds__(CV_THREADS) k_synth_conv(const float *__restrict__ u,
                                                           const int2 *__restrict__ range,
                                                           const awp_synth_cterm *__restrict__ ct,
                                                           const float *__restrict__ stfpool, int ntout, int ns8,
                                                           float *__restrict__ seis)
{
    static_assert(STRIDE % 32 == 4, "stride");
    extern __shared__ __align__(16) float sm[];
    const int buf = ns8 + 8 * STRIDE;                  /* floats per buffer: slip rate, then window */
    const int v = blockIdx.z, cu = blockIdx.y, t0 = blockIdx.x * CV_BLOCK, tid = threadIdx.x;
    const int base = t0 + tid * 8;
    float *out = seis + ((size_t)v * 3 + cu + 3 - UC) * ntout;
    float s[8];
#pragma unroll
    for (int q = 0; q < 8; q++) s[q] = base + q < ntout ? out[base + q] : 0.0f;
    const int2 rg = range[v];

    auto issue = [&](const awp_synth_cterm &t, float *b) {
        const int n8 = (t.nstf + 7) & ~7;
        for (int k = tid; k < n8; k += CV_THREADS) cp_async4(b + k, stfpool + t.stf + (k < t.nstf ? k : 0), k < t.nstf);
        const float *tr = u + ((size_t)t.slot * UC + cu) * ntout;
        const int w0 = t0 - (n8 - 1), wl = CV_BLOCK + n8;
        /* window sample y = tid + 128 i: row tid & 7, column tid / 8 + 16 i */
        float *win = b + ns8 + (tid & 7) * STRIDE + (tid >> 3);
        for (int y = tid; y < wl; y += CV_THREADS, win += CV_THREADS / 8) {
            const int x = w0 + y;
            const bool ok = x >= t.lo && x < t.hi;
            cp_async4(win, tr + (ok ? x : 0), ok);
        }
    };

    /* one group of eight lags with lo = L, hi = H; loads the next lo into N.
     * At g = 0 the load of N reads column tid - 1 (for tid = 0 the float just
     * before the window, in this buffer's slip-rate area): in bounds, unused. */
    auto group = [&](float(&acc)[8], const float(&L)[8], const float(&H)[8], float(&N)[8], const float *stf,
                     const float *col, int k0) {
        const float4 fa = *reinterpret_cast<const float4 *>(stf + k0);
        const float4 fb = *reinterpret_cast<const float4 *>(stf + k0 + 4);
        const float f[8] = {fa.x, fa.y, fa.z, fa.w, fb.x, fb.y, fb.z, fb.w};
#pragma unroll
        for (int j = 0; j < 8; j++) N[j] = col[j * STRIDE - 1];
#pragma unroll
        for (int kk = 0; kk < 8; kk++)
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int j = q + 7 - kk;                   /* W[q + m], m = 8g + 7 - kk */
                acc[q] = acc[q] + f[kk] * (j < 8 ? L[j] : H[j - 8]);
            }
    };

    awp_synth_cterm cur{}, nxt{}, nn{};
    if (rg.x < rg.y) {
        cur = ct[rg.x];
        issue(cur, sm);
    }
    cp_async_commit();
    if (rg.x + 1 < rg.y) nxt = ct[rg.x + 1];
    for (int n = rg.x; n < rg.y; n++) {
        float *b = sm + ((n - rg.x) & 1) * buf;
        if (n + 2 < rg.y) nn = ct[n + 2];
        if (n + 1 < rg.y) issue(nxt, sm + ((n + 1 - rg.x) & 1) * buf);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        /* acc_q = sum over k of stf[k] * u[base + q - k], k ascending
         * (stf_subs.c:25-33).  Slip-rate samples past nstf are zero and
         * window samples outside the written trace are zero: those products
         * add +-0 to an accumulator that starts at +0 and so leave it as the
         * reference's shorter sum leaves it. */
        const int n8 = (cur.nstf + 7) & ~7;
        int g = n8 / 8 - 1;
        const float *col = b + ns8 + tid + g;               /* column of group g in row 0 */
        float acc[8], X[8], Y[8], Z[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            acc[q] = 0.0f;
            Y[q] = col[q * STRIDE + 1];
            X[q] = col[q * STRIDE];
        }
        /* groups g, g - 1, g - 2 cover lags n8 - 8 - 8 g .. n8 + 15 - 8 g */
        for (; g >= 2; g -= 3, col -= 3) {
            group(acc, X, Y, Z, b, col, n8 - 8 - 8 * g);
            group(acc, Z, X, Y, b, col - 1, n8 - 8 * g);
            group(acc, Y, Z, X, b, col - 2, n8 + 8 - 8 * g);
        }
        if (g >= 0) group(acc, X, Y, Z, b, col, n8 - 8 - 8 * g);
        if (g >= 1) group(acc, Z, X, Y, b, col - 1, n8 - 8 * g);
#pragma unroll
        for (int q = 0; q < 8; q++) s[q] = s[q] + acc[q];     /* stf_subs.c:34-36 */
        __syncthreads();
        cur = nxt;
        nxt = nn;
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
        if (base + q < ntout) out[base + q] = s[q];
}

/* window row strides (4 mod 32); a stride holds slip rates of
 * n8 <= 8 (STRIDE - 1) - CV_BLOCK + 1 samples */
constexpr int CV_STRIDES[4] = {164, 260, 644, 1668};

size_t cv_smem_bytes(int ns8, int st) { return sizeof(float) * 2 * ((size_t)ns8 + 8 * (size_t)st); }

int cv_stride_for(int ns8)
{
    for (int st : CV_STRIDES)
        if (8 * (st - 1) - CV_BLOCK + 1 >= ns8 && cv_smem_bytes(ns8, st) <= 227 * 1024) return st;
    return 0;
}


template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t want)
    {
        if (want <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc((void **)&p, want * sizeof(T) + 16);
        if (e == cudaSuccess) n = want;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

template <class T>
struct HBuf {                      /* pinned host staging, grown on demand */
    T *p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t want)
    {
        if (want <= n) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaHostAlloc((void **)&p, want * sizeof(T) + 16, cudaHostAllocDefault);
        if (e == cudaSuccess) n = want;
        return e;
    }
    void release()
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
};

/* one chunk's terms on both sides: pinned host arrays the plan fills and
 * the device copies the kernels read, with the trace buffer; two stages
 * alternate so that chunk c + 1 is planned and copied while chunk c runs */
struct Stage {
    HBuf<awp_synth_gterm> gt;
    HBuf<awp_synth_cterm> ct;
    HBuf<float> stf;
    HBuf<int> slot_term, tl, multi;
    HBuf<int2> range;
    HBuf<int4> groups;
    DBuf<awp_synth_gterm> d_gt;
    DBuf<awp_synth_cterm> d_ct;
    DBuf<float> d_stf, d_u;
    DBuf<int> d_slot_term, d_multi;
    DBuf<int2> d_range;
    DBuf<int4> d_groups;
    cudaEvent_t h2d = nullptr;     /* host arrays copied: the host may refill them    */
    cudaEvent_t gf = nullptr;      /* traces written: the convolution may read them    */
    cudaEvent_t conv = nullptr;    /* convolution done: the device arrays may be refilled */
    bool pending = false;
    void release()
    {
        gt.release(), ct.release(), stf.release(), slot_term.release(), tl.release(), multi.release();
        range.release(), groups.release();
        d_gt.release(), d_ct.release(), d_stf.release(), d_u.release(), d_slot_term.release(), d_multi.release();
        d_range.release(), d_groups.release();
        for (cudaEvent_t e : {h2d, gf, conv})
            if (e) cudaEventDestroy(e);
        h2d = gf = conv = nullptr;
    }
};

/* a rupture variation: its own copy of the points and samples, or the
 * caller's arrays (borrowed while the variation is listed) */
struct Variation {
    int id;
    std::vector<awp_srf_point> own_pts;
    std::vector<float> own_pool;
    const awp_srf_point *pts;
    int np;
    const float *pool;
    long long npool;
};

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct awp_synth {
    awp_synth_params p;
    cudaStream_t stream = nullptr;   /* convolutions, seismogram copies */
    cudaStream_t cstream = nullptr;  /* host-to-device copies of chunk terms */
    cudaStream_t gstream = nullptr;  /* SGT combination kernels */
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    /* SGT set */
    awp_sgtmaster m{};
    std::vector<awp_sgtindex> ix;
    std::vector<awp_sgtheader> hd;
    int ncomp = 0;
    float *d_sgt = nullptr;
    /* variations and results */
    std::vector<Variation> vars;
    std::vector<float> seis;
    int nseis = 0;
    awp_synth_info info{};
    /* run buffers */
    DBuf<float> d_seis;
    Stage stage[2];
    HBuf<float> h_seis;
    std::vector<cudaEvent_t> cev;  /* per chunk: around the combination, around the convolution */
    size_t u_cap_bytes = (size_t)2 << 30;
};

static awp_status synth_set_sgt_common(awp_synth *s, const awp_sgtmaster *m, const awp_sgtindex *ix,
                                       const awp_sgtheader *hd, int ncomp)
{
    if (!s || !m || !ix || !hd) return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: null argument");
    if (ncomp < 1 || ncomp > 3) return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: ncomp must be 1..3");
    if (m->globnp < 1 || m->nt < 1) return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: empty SGT set");
    for (int i = 0; i < m->globnp; i++) {
        if (hd[i].nt != hd[0].nt || hd[i].dt != hd[0].dt)
            return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: SGT points differ in nt or dt");
        if (i && ix[i].indx <= ix[i - 1].indx)
            return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: SGT index not sorted by indx");
    }
    if (hd[0].nt != m->nt) return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: header nt differs from the master nt");
    if (!(ix[0].h > 0.0f) || !(hd[0].dt > 0.0f))
        return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: grid spacing and SGT sample interval must be > 0");
    s->m = *m;
    s->ix.assign(ix, ix + m->globnp);
    s->hd.assign(hd, hd + m->globnp);
    /* the x headers stand for every component: synth.c:545-557 */
    for (auto &h : s->hd) {
        if (ncomp >= 2) h.ymom = h.xmom;
        if (ncomp == 3) h.zmom = h.xmom;
    }
    s->ncomp = ncomp;
    return AWP_OK;
}

extern "C" awp_status awp_synth_create(const awp_synth_params *p, awp_synth **out)
{
    if (!p || !out) return fail(AWP_ERR_PARAM, "awp_synth_create: null argument");
    *out = nullptr;
    if (!(p->dtout > 0.0f)) return fail(AWP_ERR_PARAM, "awp_synth_create: dtout must be > 0");
    if (p->rv_batch < 0) return fail(AWP_ERR_PARAM, "awp_synth_create: rv_batch must be >= 0");
    SCU(cudaSetDevice(p->device));
    awp_synth *s = new awp_synth();
    s->p = *p;
    if (const char *e = getenv("AWP_SYNTH_UBUF_MB")) {
        const long mb = atol(e);
        if (mb > 0) s->u_cap_bytes = (size_t)mb << 20;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->gstream, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&s->ev[i]);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
        e = cudaEventCreateWithFlags(&s->stage[i].h2d, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->stage[i].gf, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->stage[i].conv, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        awp_synth_destroy(s);
        return fail(AWP_ERR_CUDA, "awp_synth_create: %s", cudaGetErrorString(e));
    }
    *out = s;
    return AWP_OK;
}

extern "C" void awp_synth_destroy(awp_synth *s)
{
    if (!s) return;
    cudaSetDevice(s->p.device);
    for (cudaStream_t st : {s->stream, s->cstream, s->gstream})
        if (st) cudaStreamSynchronize(st);
    if (s->d_sgt) cudaFree(s->d_sgt);
    s->d_seis.release();
    for (auto &st : s->stage) st.release();
    s->h_seis.release();
    for (auto &e : s->cev) cudaEventDestroy(e);
    for (auto &e : s->ev)
        if (e) cudaEventDestroy(e);
    for (cudaStream_t st : {s->stream, s->cstream, s->gstream})
        if (st) cudaStreamDestroy(st);
    delete s;
}

extern "C" awp_status awp_synth_set_sgt(awp_synth *s, const awp_sgtmaster *m, const awp_sgtindex *ix,
                                        const awp_sgtheader *hd, int ncomp, const float *x, const float *y,
                                        const float *z)
{
    awp_status st = synth_set_sgt_common(s, m, ix, hd, ncomp);
    if (st != AWP_OK) return st;
    const float *src[3] = {x, y, z};
    for (int q = 0; q < ncomp; q++)
        if (!src[q]) return fail(AWP_ERR_PARAM, "awp_synth_set_sgt: component %d data missing", q);
    SCU(cudaSetDevice(s->p.device));
    if (s->d_sgt) cudaFree(s->d_sgt);
    s->d_sgt = nullptr;
    const size_t np = (size_t)m->globnp, row = (size_t)6 * m->nt;
    SCU(cudaMalloc((void **)&s->d_sgt, np * ncomp * row * sizeof(float)));
    /* [point][component][6][nt]: one strided copy per component */
    for (int q = 0; q < ncomp; q++)
        SCU(cudaMemcpy2DAsync(s->d_sgt + q * row, ncomp * row * sizeof(float), src[q], row * sizeof(float),
                              row * sizeof(float), np, cudaMemcpyHostToDevice, s->stream));
    SCU(cudaStreamSynchronize(s->stream));
    s->info.ncomp = ncomp;
    return AWP_OK;
}

static awp_status read_file(const char *path, size_t off, size_t bytes, void *dst)
{
    FILE *f = fopen(path, "rb");
    if (!f) return fail(AWP_ERR_IO, "cannot open %s", path);
    int ok = fseeko(f, (off_t)off, SEEK_SET) == 0 && fread(dst, 1, bytes, f) == bytes;
    fclose(f);
    return ok ? AWP_OK : fail(AWP_ERR_IO, "%s: short read (%zu bytes at %zu)", path, bytes, off);
}

struct HeadFile {
    awp_sgtmaster m;
    std::vector<awp_sgtindex> ix;
    std::vector<awp_sgtheader> hd;
};

static awp_status read_head(const char *path, HeadFile &h)
{
    awp_status st = read_file(path, 0, sizeof h.m, &h.m);
    if (st != AWP_OK) return st;
    if (h.m.globnp < 1 || h.m.globnp > (1 << 28) || h.m.nt < 1)
        return fail(AWP_ERR_IO, "%s: implausible SGT master record (globnp %d, nt %d)", path, h.m.globnp, h.m.nt);
    h.ix.resize(h.m.globnp);
    h.hd.resize(h.m.globnp);
    st = read_file(path, sizeof h.m, sizeof(awp_sgtindex) * h.ix.size(), h.ix.data());
    if (st == AWP_OK)
        st = read_file(path, sizeof h.m + sizeof(awp_sgtindex) * h.ix.size(), sizeof(awp_sgtheader) * h.hd.size(),
                       h.hd.data());
    return st;
}

extern "C" awp_status awp_synth_load_sgt_files(awp_synth *s, const char *xhead, const char *xdata, const char *yhead,
                                               const char *ydata, const char *zhead, const char *zdata)
{
    if (!s || !xhead || !xdata) return fail(AWP_ERR_PARAM, "awp_synth_load_sgt_files: x component required");
    if ((yhead == nullptr) != (ydata == nullptr) || (zhead == nullptr) != (zdata == nullptr))
        return fail(AWP_ERR_PARAM, "awp_synth_load_sgt_files: header and data come in pairs");
    if (!yhead && zhead)
        return fail(AWP_ERR_PARAM, "awp_synth_load_sgt_files: z without y is not a supported set (jbsim3d.c:641)");
    HeadFile h[3];
    const char *heads[3] = {xhead, yhead, zhead}, *datas[3] = {xdata, ydata, zdata};
    int ncomp = 0;
    for (int q = 0; q < 3 && heads[q]; q++, ncomp++) {
        awp_status st = read_head(heads[q], h[q]);
        if (st != AWP_OK) return st;
        if (h[q].m.globnp != h[0].m.globnp || h[q].m.nt != h[0].m.nt)
            return fail(AWP_ERR_PARAM, "%s: point count or nt differs from the x component", heads[q]);
    }
    /* moments must agree (sgt_handler.c:226-242) */
    if (ncomp >= 2 && h[0].hd[0].xmom != h[1].hd[0].ymom)
        return fail(AWP_ERR_PARAM, "X-moment and Y-moment are not the same");
    if (ncomp == 3 && h[0].hd[0].xmom != h[2].hd[0].zmom)
        return fail(AWP_ERR_PARAM, "X-moment and Z-moment are not the same");
    const size_t bytes = (size_t)h[0].m.globnp * 6 * h[0].m.nt * sizeof(float);
    std::vector<float> data[3];
    for (int q = 0; q < ncomp; q++) {
        data[q].resize(bytes / sizeof(float));
        awp_status st = read_file(datas[q], 0, bytes, data[q].data());
        if (st != AWP_OK) return st;
    }
    return awp_synth_set_sgt(s, &h[0].m, h[0].ix.data(), h[0].hd.data(), ncomp, data[0].data(),
                             ncomp > 1 ? data[1].data() : nullptr, ncomp > 2 ? data[2].data() : nullptr);
}

static awp_status add_variation(awp_synth *s, int rup_var_id, const awp_srf_point *pts, int np, const float *pool,
                                long long npool, bool borrow)
{
    if (!s || (np > 0 && !pts) || (npool > 0 && !pool) || np < 0 || npool < 0)
        return fail(AWP_ERR_PARAM, "awp_synth_add_variation: bad argument");
    if (!s->vars.empty() && s->vars[0].np != np)
        return fail(AWP_ERR_PARAM, "awp_synth_add_variation: %d points, the rupture has %d", np, s->vars[0].np);
    for (int i = 0; i < np; i++) {
        const awp_srf_point &a = pts[i];
        const int n[3] = {a.nt1, a.nt2, a.nt3};
        const long long o[3] = {a.stf1, a.stf2, a.stf3};
        for (int q = 0; q < 3; q++)
            if (n[q] < 0 || (n[q] > 0 && (o[q] < 0 || o[q] + n[q] > npool)))
                return fail(AWP_ERR_PARAM, "awp_synth_add_variation: point %d slip-rate samples outside the pool", i);
    }
    s->vars.emplace_back();
    Variation &v = s->vars.back();
    v.id = rup_var_id;
    v.np = np;
    v.npool = npool;
    if (borrow) {
        v.pts = pts;
        v.pool = pool;
    } else {
        v.own_pts.assign(pts, pts + np);
        v.own_pool.assign(pool, pool + npool);
        v.pts = v.own_pts.data();
        v.pool = v.own_pool.data();
    }
    return AWP_OK;
}

extern "C" awp_status awp_synth_add_variation(awp_synth *s, int rup_var_id, const awp_srf_point *pts, int np,
                                              const float *pool, long long npool)
{
    return add_variation(s, rup_var_id, pts, np, pool, npool, false);
}

extern "C" awp_status awp_synth_add_variation_borrowed(awp_synth *s, int rup_var_id, const awp_srf_point *pts,
                                                       int np, const float *pool, long long npool)
{
    return add_variation(s, rup_var_id, pts, np, pool, npool, true);
}

extern "C" awp_status awp_synth_add_srf_file(awp_synth *s, int rup_var_id, const char *path, int binary)
{
    if (!s) return fail(AWP_ERR_PARAM, "awp_synth_add_srf_file: null synth");
    awp_srf_point *pts = nullptr;
    float *pool = nullptr;
    int np = 0;
    long long npool = 0;
    awp_status st = awp_srf_read(path, binary, &pts, &np, &pool, &npool);
    if (st != AWP_OK) return st;
    st = awp_synth_add_variation(s, rup_var_id, pts, np, pool, npool);
    free(pts);
    free(pool);
    return st;
}

extern "C" awp_status awp_synth_clear_variations(awp_synth *s)
{
    if (!s) return fail(AWP_ERR_PARAM, "awp_synth_clear_variations: null synth");
    s->vars.clear();
    return AWP_OK;
}

/* jbsim3d.c:436-447: working length and output length */
static void synth_lengths(const awp_synth *s, int *ntsum, int *ntout)
{
    int maxnt = s->hd[0].nt;
    const float mindt = s->hd[0].dt, dtout = s->p.dtout;
    if (dtout < mindt) maxnt = (int)(maxnt * mindt / dtout);
    int n = 2;
    while (n < 4 * maxnt) n *= 2;
    *ntsum = n;
    *ntout = s->p.ntout > 0 ? s->p.ntout : n;
}

template <int STRIDE, int UC>
static cudaError_t launch_conv_t(dim3 grid, size_t smem, cudaStream_t st, const float *u, const int2 *range,
                                 const awp_synth_cterm *ct, const float *stf, int ntout, int ns8, float *seis)
{
    cudaError_t e =
        cudaFuncSetAttribute(k_synth_conv<STRIDE, UC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_synth_conv<STRIDE, UC><<<grid, CV_THREADS, smem, st>>>(u, range, ct, stf, ntout, ns8, seis);
    return cudaGetLastError();
}

/* one convolution launch: nb variations, uc components */
static cudaError_t launch_conv(int stride, int uc, int nb, int ntout, int ns8, cudaStream_t st, const float *u,
                               const int2 *range, const awp_synth_cterm *ct, const float *stf, float *seis)
{
    const size_t smem = cv_smem_bytes(ns8, stride);
    const dim3 g((unsigned)((ntout + CV_BLOCK - 1) / CV_BLOCK), (unsigned)uc, (unsigned)nb);
#define CONV_CASE(I)                                                                                      \
    if (stride == CV_STRIDES[I])                                                                          \
        return uc == 3 ? launch_conv_t<CV_STRIDES[I], 3>(g, smem, st, u, range, ct, stf, ntout, ns8, seis) \
                       : launch_conv_t<CV_STRIDES[I], 2>(g, smem, st, u, range, ct, stf, ntout, ns8, seis);
    CONV_CASE(0)
    CONV_CASE(1)
    CONV_CASE(2)
    CONV_CASE(3)
#undef CONV_CASE
    return cudaErrorInvalidValue;
}

template <int NC, int UC>
static cudaError_t launch_gf_nc(int ngroups, int nmulti, int nt, int ntout, cudaStream_t st, const float *sgt,
                                const awp_synth_gterm *gt, const int *slot_term, const int4 *groups,
                                const int *multi, float *u)
{
    if (ngroups) {
        const dim3 g((unsigned)((nt + GF_THREADS - 1) / GF_THREADS), (unsigned)ngroups);
        k_synth_gf1<NC, UC><<<g, GF_THREADS, 0, st>>>(sgt, nt, nt - SY_TAPLEN, gt, slot_term, groups, ntout, u);
    }
    if (nmulti) {
        const dim3 g((unsigned)nmulti, (unsigned)((ntout + GF_THREADS - 1) / GF_THREADS));
        k_synth_gf<NC, UC><<<g, GF_THREADS, 0, st>>>(sgt, nt, nt - SY_TAPLEN, gt, slot_term, multi, ntout, u);
    }
    return cudaGetLastError();
}

static cudaError_t launch_gf(int ncomp, int ngroups, int nmulti, int nt, int ntout, cudaStream_t st,
                             const float *sgt, const awp_synth_gterm *gt, const int *slot_term, const int4 *groups,
                             const int *multi, float *u)
{
    if (ncomp == 1) return launch_gf_nc<1, 2>(ngroups, nmulti, nt, ntout, st, sgt, gt, slot_term, groups, multi, u);
    if (ncomp == 2) return launch_gf_nc<2, 2>(ngroups, nmulti, nt, ntout, st, sgt, gt, slot_term, groups, multi, u);
    return launch_gf_nc<3, 3>(ngroups, nmulti, nt, ntout, st, sgt, gt, slot_term, groups, multi, u);
}

static cudaError_t events_for(awp_synth *s, int n)
{
    while ((int)s->cev.size() < n) {
        cudaEvent_t ev;
        cudaError_t e = cudaEventCreate(&ev);
        if (e != cudaSuccess) return e;
        s->cev.push_back(ev);
    }
    return cudaSuccess;
}

/* Work order: variations in batches (rv_batch, default all of them); inside
 * a batch the rupture points in chunks.  A chunk is planned on the host (all
 * its variations in parallel), copied, combined (k_synth_gf) and convolved
 * into the batch's seismograms (k_synth_conv); the host plans chunk c + 1
 * while the device runs chunk c.  Chunks hold whole points, at most the
 * term buffer's capacity and about a quarter of the batch. */
extern "C" awp_status awp_synth_run(awp_synth *s)
{
    if (!s) return fail(AWP_ERR_PARAM, "awp_synth_run: null synth");
    if (!s->d_sgt) return fail(AWP_ERR_STATE, "awp_synth_run: no SGT set loaded");
    if (s->vars.empty()) return fail(AWP_ERR_STATE, "awp_synth_run: no rupture variation added");
    SCU(cudaSetDevice(s->p.device));
    double t_plan = now_s();
    const int np = s->vars[0].np, nv = (int)s->vars.size();
    int ntsum, ntout;
    synth_lengths(s, &ntsum, &ntout);
    const int nt = s->m.nt;

    /* site and rupture points in the SGT grid, bracketing SGT points
     * (synth.c:35-80) */
    awp_synth_geo geo;
    awp_status st = awp_synth_geo_init(&s->m, &geo);
    if (st != AWP_OK) return st;
    const float h = s->ix[0].h;
    awp_sgtindex stat;
    awp_synth_get_indx(&geo, s->p.slon, s->p.slat, 0.0f, h, &stat);
    std::vector<awp_synth_bracket> br(np);
    int non_exact = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : non_exact)
    for (int ip = 0; ip < np; ip++) {
        const awp_srf_point &a = s->vars[0].pts[ip];
        awp_sgtindex eq;
        awp_synth_get_indx(&geo, a.lon, a.lat, a.dep, h, &eq);
        awp_synth_find_sgt(s->ix.data(), (int)s->ix.size(), &eq, &stat, &br[ip]);
        non_exact += br[ip].nsgt != 1;
    }
    std::vector<char> used(s->ix.size(), 0);
    for (auto &b : br)
        for (int g = 0; g < b.nsgt; g++) used[b.pos[g]] = 1;
    int nm = 0;
    for (char c : used) nm += c;

    float taper[SY_TAPLEN];
    awp_synth_taper(nt, taper);
    SCU(cudaMemcpyToSymbolAsync(c_taper, taper, sizeof taper, 0, cudaMemcpyHostToDevice, s->stream));

    awp_synth_plan_ctx cx;
    cx.hd = s->hd.data();
    cx.br = br.data();
    cx.np = np;
    cx.nt = nt;
    cx.ntsum = ntsum;
    cx.ntout = ntout;
    cx.dtout = s->p.dtout;
    cx.tstart = s->p.tstart;
    cx.taper = taper;

    /* per variation and point: terms and slip-rate samples (prefix sums) */
    std::vector<long long> tpre((size_t)nv * (np + 1)), spre((size_t)nv * (np + 1));
    int maxnstf = 1;
#pragma omp parallel for schedule(static) reduction(max : maxnstf)
    for (int v = 0; v < nv; v++) {
        long long t = 0, n = 0;
        for (int ip = 0; ip < np; ip++) {
            tpre[(size_t)v * (np + 1) + ip] = t;
            spre[(size_t)v * (np + 1) + ip] = n;
            const awp_srf_point &a = s->vars[v].pts[ip];
            t += (a.nt1 > 0) + (a.nt2 > 0) + (a.nt3 > 0);
            n += (a.nt1 > 0 ? a.nt1 : 0) + (a.nt2 > 0 ? a.nt2 : 0) + (a.nt3 > 0 ? a.nt3 : 0);
            maxnstf = a.nt1 > maxnstf ? a.nt1 : maxnstf;
            maxnstf = a.nt2 > maxnstf ? a.nt2 : maxnstf;
            maxnstf = a.nt3 > maxnstf ? a.nt3 : maxnstf;
        }
        tpre[(size_t)v * (np + 1) + np] = t;
        spre[(size_t)v * (np + 1) + np] = n;
    }
    maxnstf = maxnstf < ntout ? maxnstf : ntout;      /* longer ones are refused by the plan */
    const int batch = s->p.rv_batch > 0 ? s->p.rv_batch : nv;

    /* chunk boundaries per batch: whole points, terms <= cap */
    const int uc = s->ncomp == 3 ? 3 : 2;             /* component traces kept per term */
    const size_t slot_bytes = (size_t)uc * ntout * sizeof(float);
    const long long ucap = (long long)(s->u_cap_bytes / slot_bytes) > 0 ? (long long)(s->u_cap_bytes / slot_bytes) : 1;
    struct Chunk {
        int v0, nb, p0, p1;
        long long terms, samples;
    };
    std::vector<Chunk> chunks;
    long long max_terms = 1, max_stf = 1;
    for (int v0 = 0; v0 < nv; v0 += batch) {
        const int nb = v0 + batch <= nv ? batch : nv - v0;
        long long total = 0;
        for (int v = v0; v < v0 + nb; v++) total += tpre[(size_t)v * (np + 1) + np];
        /* at least four chunks (to overlap the plan with the device) of equal
         * size, none above the term buffer; the first one an eighth of that,
         * so that the device starts while the host plans the rest */
        long long nch = (total + ucap - 1) / ucap;
        nch = nch < 4 ? 4 : nch;
        const long long full_target = (total + nch - 1) / nch;
        long long target = (full_target + 7) / 8;
        for (int p0 = 0; p0 < np; target = full_target) {
            long long t = 0, n = 0;
            int p1 = p0;
            while (p1 < np) {
                long long dt = 0, dn = 0;
                for (int v = v0; v < v0 + nb; v++) {
                    const size_t o = (size_t)v * (np + 1) + p1;
                    dt += tpre[o + 1] - tpre[o];
                    dn += spre[o + 1] - spre[o];
                }
                if (p1 > p0 && t + dt > target) break;
                t += dt, n += dn, p1++;
            }
            chunks.push_back({v0, nb, p0, p1, t, n});
            max_terms = t > max_terms ? t : max_terms;
            max_stf = n > max_stf ? n : max_stf;
            p0 = p1;
        }
    }
    if (max_terms >= (1LL << 31)) return fail(AWP_ERR_PARAM, "awp_synth_run: too many terms in one chunk");

    cudaError_t e = cudaSuccess;
    e = e ? e : s->d_seis.reserve((size_t)nv * 3 * ntout);
    e = e ? e : s->h_seis.reserve((size_t)nv * 3 * ntout);
    for (auto &sg : s->stage) {
        e = e ? e : sg.gt.reserve((size_t)max_terms);
        e = e ? e : sg.ct.reserve((size_t)max_terms);
        e = e ? e : sg.stf.reserve((size_t)max_stf + 8);
        e = e ? e : sg.slot_term.reserve((size_t)max_terms);
        e = e ? e : sg.tl.reserve((size_t)max_terms);
        e = e ? e : sg.range.reserve((size_t)batch);
        e = e ? e : sg.multi.reserve((size_t)max_terms);
        e = e ? e : sg.groups.reserve((size_t)np);
        e = e ? e : sg.d_gt.reserve((size_t)max_terms);
        e = e ? e : sg.d_ct.reserve((size_t)max_terms);
        e = e ? e : sg.d_stf.reserve((size_t)max_stf + 8);
        e = e ? e : sg.d_slot_term.reserve((size_t)max_terms);
        e = e ? e : sg.d_range.reserve((size_t)batch);
        e = e ? e : sg.d_multi.reserve((size_t)max_terms);
        e = e ? e : sg.d_groups.reserve((size_t)np);
        e = e ? e : sg.d_u.reserve((size_t)max_terms * uc * ntout);
    }
    if (e != cudaSuccess) return fail(AWP_ERR_OOM, "awp_synth_run: buffers: %s", cudaGetErrorString(e));

    const int ns8 = (maxnstf + 7) & ~7;
    const int stride = cv_stride_for(ns8);
    if (!stride) return fail(AWP_ERR_PARAM, "awp_synth_run: slip-rate functions too long (%d samples)", maxnstf);

    s->nseis = 0;
    s->info = awp_synth_info{};
    s->info.ncomp = s->ncomp;
    s->info.ntout = ntout;
    s->info.ntsum = ntsum;
    s->info.nsgt_points = nm;
    s->info.non_exact = non_exact;
    double plan_s = now_s() - t_plan;
    int launches = 0, nk = 0;     /* chunks launched; chunk j is timed by events 4j .. 4j + 3 */

    /* streams: copies on cstream, combination on gstream, convolution on
     * stream.  Chunk c (stage c & 1): copy after the convolution of chunk
     * c - 2 released the stage; combine after the copy; convolve after the
     * combination (and, on its stream, after chunk c - 1). */
    SCU(cudaEventRecord(s->ev[0], s->stream));
    SCU(cudaMemsetAsync(s->d_seis.p, 0, (size_t)nv * 3 * ntout * sizeof(float), s->stream));
    SCU(cudaEventRecord(s->ev[2], s->stream));
    SCU(cudaStreamWaitEvent(s->cstream, s->ev[2], 0));
    SCU(cudaStreamWaitEvent(s->gstream, s->ev[2], 0));
    for (auto &sg : s->stage) sg.pending = false;
    std::vector<long long> toff, soff, pbase;
    std::vector<int> pslot;
    for (size_t ic = 0; ic < chunks.size(); ic++) {
        t_plan = now_s();
        const Chunk &C = chunks[ic];
        const int nb = C.nb, p0 = C.p0, p1 = C.p1, npc = p1 - p0;
        Stage &S = s->stage[ic & 1];
        if (S.pending) SCU(cudaEventSynchronize(S.h2d));   /* its copies of two chunks ago are done */
        S.pending = false;
        /* chunk-local term numbering: variation-major (each variation's terms
         * contiguous, in point order); slots: point-major */
        toff.assign(nb + 1, 0);
        soff.assign(nb + 1, 0);
        for (int b = 0; b < nb; b++) {
            const size_t o = (size_t)(C.v0 + b) * (np + 1);
            toff[b + 1] = toff[b] + tpre[o + p1] - tpre[o + p0];
            soff[b + 1] = soff[b] + spre[o + p1] - spre[o + p0];
        }
        const long long nterm = toff[nb];
        std::vector<long long> macs(nb, 0);
        std::vector<awp_status> pst(nb, AWP_OK);
#pragma omp parallel for schedule(dynamic, 1)
        for (int b = 0; b < nb; b++) {
            const Variation &v = s->vars[C.v0 + b];
            long long nterms = 0, nused = 0;
            pst[b] = awp_synth_plan_variation(&cx, v.pts, v.pool, v.npool, p0, p1,
                                              S.gt.p + toff[b], S.ct.p + toff[b], S.stf.p + soff[b], soff[b],
                                              &nterms, &nused, &macs[b]);
        }
        for (int b = 0; b < nb; b++)
            if (pst[b] != AWP_OK) {
                /* the error text is per thread: plan the variation again here */
                for (cudaStream_t q : {s->stream, s->cstream, s->gstream}) SCU(cudaStreamSynchronize(q));
                for (auto &sg : s->stage) sg.pending = false;
                const Variation &v = s->vars[C.v0 + b];
                long long a1, a2, a3;
                return awp_synth_plan_variation(&cx, v.pts, v.pool, v.npool, p0, p1,
                                                S.gt.p + toff[b], S.ct.p + toff[b], S.stf.p + soff[b], soff[b], &a1,
                                                &a2, &a3);
            }
        for (int b = 0; b < nb; b++) s->info.macs += macs[b] * uc;
        s->info.terms += nterm;
        for (int k = 0; k < 8; k++) S.stf.p[soff[nb] + k] = 0.0f;
        /* slots of point ip start at pslot[ip - p0]; a point's slots hold its
         * variations in order */
        pslot.assign(npc + 1, 0);
        for (int i = 0; i < npc; i++) {
            long long n = 0;
            for (int b = 0; b < nb; b++) {
                const size_t o = (size_t)(C.v0 + b) * (np + 1) + p0 + i;
                n += tpre[o + 1] - tpre[o];
            }
            pslot[i + 1] = pslot[i] + (int)n;
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < npc; i++) {
            long long sl = pslot[i];
            for (int b = 0; b < nb; b++) {
                const size_t o = (size_t)(C.v0 + b) * (np + 1);
                const long long a0 = toff[b] + tpre[o + p0 + i] - tpre[o + p0];
                const long long a1 = a0 + tpre[o + p0 + i + 1] - tpre[o + p0 + i];
                for (long long t = a0; t < a1; t++, sl++) {
                    S.slot_term.p[sl] = (int)t;
                    S.tl.p[t] = (int)sl;
                }
            }
        }
        for (long long t = 0; t < nterm; t++) S.ct.p[t].slot = S.tl.p[t];
        for (int b = 0; b < nb; b++) S.range.p[b] = make_int2((int)toff[b], (int)toff[b + 1]);
        /* exactly matched points go to the per-point kernel, the others'
         * slots to the per-term one */
        int ngroups = 0, nmulti = 0;
        for (int i = 0; i < npc; i++) {
            const int n = pslot[i + 1] - pslot[i];
            if (!n) continue;
            const awp_synth_bracket &bk = br[p0 + i];
            if (bk.nsgt == 1) S.groups.p[ngroups++] = make_int4(bk.pos[0], pslot[i], n, 0);
            else
                for (int k = pslot[i]; k < pslot[i + 1]; k++) S.multi.p[nmulti++] = k;
        }
        plan_s += now_s() - t_plan;

        if (nterm) {
            cudaStream_t cs = s->cstream;
            if (ic >= 2) SCU(cudaStreamWaitEvent(cs, S.conv, 0));
            SCU(cudaMemcpyAsync(S.d_gt.p, S.gt.p, nterm * sizeof(awp_synth_gterm), cudaMemcpyHostToDevice, cs));
            SCU(cudaMemcpyAsync(S.d_ct.p, S.ct.p, nterm * sizeof(awp_synth_cterm), cudaMemcpyHostToDevice, cs));
            SCU(cudaMemcpyAsync(S.d_slot_term.p, S.slot_term.p, nterm * sizeof(int), cudaMemcpyHostToDevice, cs));
            SCU(cudaMemcpyAsync(S.d_stf.p, S.stf.p, (soff[nb] + 8) * sizeof(float), cudaMemcpyHostToDevice, cs));
            SCU(cudaMemcpyAsync(S.d_range.p, S.range.p, (size_t)nb * sizeof(int2), cudaMemcpyHostToDevice, cs));
            if (ngroups)
                SCU(cudaMemcpyAsync(S.d_groups.p, S.groups.p, (size_t)ngroups * sizeof(int4), cudaMemcpyHostToDevice, cs));
            if (nmulti) SCU(cudaMemcpyAsync(S.d_multi.p, S.multi.p, (size_t)nmulti * sizeof(int), cudaMemcpyHostToDevice, cs));
        }
        SCU(cudaEventRecord(S.h2d, s->cstream));
        S.pending = true;
        float *seis_b = s->d_seis.p + (size_t)C.v0 * 3 * ntout;
        if (nterm) {
            SCU(events_for(s, 4 * (nk + 1)));
            SCU(cudaStreamWaitEvent(s->gstream, S.h2d, 0));
            if (ic >= 2) SCU(cudaStreamWaitEvent(s->gstream, S.conv, 0));   /* chunk c - 2 read these traces */
            SCU(cudaEventRecord(s->cev[4 * nk], s->gstream));
            SCU(launch_gf(s->ncomp, ngroups, nmulti, nt, ntout, s->gstream, s->d_sgt, S.d_gt.p, S.d_slot_term.p,
                          S.d_groups.p, S.d_multi.p, S.d_u.p));
            SCU(cudaEventRecord(s->cev[4 * nk + 1], s->gstream));
            SCU(cudaEventRecord(S.gf, s->gstream));
            SCU(cudaStreamWaitEvent(s->stream, S.gf, 0));
            SCU(cudaEventRecord(s->cev[4 * nk + 2], s->stream));
            e = launch_conv(stride, uc, nb, ntout, ns8, s->stream, S.d_u.p, S.d_range.p, S.d_ct.p, S.d_stf.p, seis_b);
            SCU(e);
            SCU(cudaEventRecord(s->cev[4 * nk + 3], s->stream));
            SCU(cudaEventRecord(S.conv, s->stream));
            nk++;
            launches += (ngroups > 0) + (nmulti > 0) + 1;
        }
    }
    /* every variation's seismograms, including those of a rupture without
     * points or without slip (zeros from the memset) */
    SCU(cudaMemcpyAsync(s->h_seis.p, s->d_seis.p, (size_t)nv * 3 * ntout * sizeof(float), cudaMemcpyDeviceToHost,
                        s->stream));
    SCU(cudaEventRecord(s->ev[1], s->stream));
    SCU(cudaEventSynchronize(s->ev[1]));
    SCU(cudaStreamSynchronize(s->cstream));
    SCU(cudaStreamSynchronize(s->gstream));
    for (auto &sg : s->stage) sg.pending = false;
    float ms = 0.0f;
    SCU(cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]));
    double gf_s = 0.0, conv_s = 0.0;
    for (int j = 0; j < nk; j++) {
        float a = 0.0f, c = 0.0f;
        SCU(cudaEventElapsedTime(&a, s->cev[4 * j], s->cev[4 * j + 1]));
        SCU(cudaEventElapsedTime(&c, s->cev[4 * j + 2], s->cev[4 * j + 3]));
        gf_s += a * 1e-3;
        conv_s += c * 1e-3;
    }
    s->seis.assign(s->h_seis.p, s->h_seis.p + (size_t)nv * 3 * ntout);
    s->nseis = nv;
    s->info.nvariations = nv;
    s->info.seconds_plan = plan_s;
    s->info.seconds_device = ms * 1e-3;
    s->info.seconds_conv = conv_s;
    s->info.seconds_gf = gf_s;
    s->info.gpu_launches = launches;
    return AWP_OK;
}

extern "C" awp_status awp_synth_seismograms(awp_synth *s, float *out, size_t n)
{
    if (!s || !out) return fail(AWP_ERR_PARAM, "awp_synth_seismograms: null argument");
    if (!s->nseis) return fail(AWP_ERR_STATE, "awp_synth_seismograms: nothing synthesised yet");
    if (n < s->seis.size()) return fail(AWP_ERR_PARAM, "awp_synth_seismograms: buffer holds %zu floats, need %zu", n,
                                        s->seis.size());
    memcpy(out, s->seis.data(), s->seis.size() * sizeof(float));
    return AWP_OK;
}

/* component flags of the seisheader (DirectSynth/src/direct_synth.c) */
enum { SEIS_X = 1, SEIS_Y = 2, SEIS_Z = 4 };

extern "C" awp_status awp_synth_write_grm(awp_synth *s, const char *path, const awp_seisheader *tmpl)
{
    if (!s || !path || !tmpl) return fail(AWP_ERR_PARAM, "awp_synth_write_grm: null argument");
    if (!s->nseis) return fail(AWP_ERR_STATE, "awp_synth_write_grm: nothing synthesised yet");
    const int ntout = s->info.ntout;
    /* jbsim3d.c:619-656: x,y,z -> [v n e]; x,y -> [n e]; x -> [n] */
    int comps, off, len;
    if (s->ncomp == 3) comps = SEIS_X | SEIS_Y | SEIS_Z, off = 0, len = 3;
    else if (s->ncomp == 2) comps = SEIS_X | SEIS_Y, off = 1, len = 2;
    else comps = SEIS_X, off = 1, len = 1;
    FILE *f = fopen(path, "wb");
    if (!f) return fail(AWP_ERR_IO, "cannot create %s", path);
    int ok = 1;
    for (int v = 0; v < s->nseis && ok; v++) {
        awp_seisheader h = *tmpl;
        h.rup_var_id = s->vars[v].id;
        h.dt = s->p.dtout;
        h.nt = ntout;
        h.comps = comps;
        ok = fwrite(&h, sizeof h, 1, f) == 1 &&
             fwrite(s->seis.data() + ((size_t)v * 3 + off) * ntout, sizeof(float), (size_t)len * ntout, f) ==
                 (size_t)len * ntout;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? AWP_OK : fail(AWP_ERR_IO, "%s: write failed", path);
}

extern "C" awp_status awp_synth_get_info(awp_synth *s, awp_synth_info *out)
{
    if (!s || !out) return fail(AWP_ERR_PARAM, "awp_synth_get_info: null argument");
    *out = s->info;
    return AWP_OK;
}
