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
constexpr int CV_Q = 8;                   /* consecutive outputs per thread  */
constexpr int CV_BLOCK = CV_THREADS * CV_Q;

__constant__ float c_taper[SY_TAPLEN];

/* ---- kernel 1: per term, the shifted sum of the bracketing SGTs --------- */

template <int NC>
__device__ __forceinline__ void gf_sample(const float *__restrict__ b, int nt, const float *k, float &gv, float &gn,
                                          float &ge)
{
    float a[6], y[6], z[6];
#pragma unroll
    for (int r = 0; r < 6; r++) {
        a[r] = __ldg(b + (size_t)r * nt);
        y[r] = NC > 1 ? __ldg(b + (size_t)(6 + r) * nt) : 0.0f;
        z[r] = NC > 2 ? __ldg(b + (size_t)(12 + r) * nt) : 0.0f;
    }
    /* sgt3d_subs.c:1393-1406: left-to-right sums, amplitude last */
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

template <int NC>
__global__ void __launch_bounds__(GF_THREADS) k_synth_gf(const float *__restrict__ sgt, int nt, int tapst,
                                                         const awp_synth_gterm *__restrict__ gt,
                                                         const int *__restrict__ slot_term, long long slot0,
                                                         int ntout, float *__restrict__ u)
{
    __shared__ awp_synth_gterm g;
    const long long slot = blockIdx.x;
    if (threadIdx.x == 0) g = gt[slot_term[slot0 + slot]];
    __syncthreads();
    const int i = blockIdx.y * GF_THREADS + threadIdx.x;
    if (i >= ntout) return;
    float uv = 0.0f, un = 0.0f, ue = 0.0f;
    for (int ig = 0; ig < g.nsgt; ig++) {
        if (i < g.lo[ig] || i >= g.hi[ig]) continue;
        const int j = i - g.shift[ig];
        float gv, gn, ge;
        gf_sample<NC>(sgt + (size_t)g.pt[ig] * (6 * NC) * nt + j, nt, g.c[ig], gv, gn, ge);
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
    float *o = u + (size_t)slot * 3 * ntout + i;
    o[0] = uv;
    o[ntout] = un;
    o[2 * (size_t)ntout] = ue;
}

/* ---- kernel 2: slip-rate convolution, terms in rupture-point order ------- */

/* shared-memory position of window sample y: Q interleaved rows, so that the
 * one new sample each thread loads per step (y = 8 * tid + const) hits 32
 * different banks; the row stride is 4 mod 32 for the same reason on fill */
__device__ __forceinline__ int cv_pos(int y, int stride) { return (y & (CV_Q - 1)) * stride + (y >> 3); }

__global__ void __launch_bounds__(CV_THREADS) k_synth_conv(const float *__restrict__ u, const int *__restrict__ tl,
                                                           const int2 *__restrict__ range, long long slot0,
                                                           const int *__restrict__ slot_term,
                                                           const awp_synth_cterm *__restrict__ ct,
                                                           const float *__restrict__ stfpool, int ntout, int stride,
                                                           int maxnstf, float *__restrict__ seis)
{
    extern __shared__ float sm[];
    float *stf = sm;                                   /* maxnstf rounded to 4 */
    float *win = sm + ((maxnstf + 3) & ~3);
    const int v = blockIdx.z, c = blockIdx.y, t0 = blockIdx.x * CV_BLOCK, tid = threadIdx.x;
    const int base = t0 + tid * CV_Q;
    float *out = seis + ((size_t)v * 3 + c) * ntout;
    float s[CV_Q];
#pragma unroll
    for (int q = 0; q < CV_Q; q++) s[q] = base + q < ntout ? out[base + q] : 0.0f;
    const int2 rg = range[v];
    for (int n = rg.x; n < rg.y; n++) {
        const int slot = tl[n];
        const awp_synth_cterm t = ct[slot_term[slot]];
        const int nstf = t.nstf;
        const float *uu = u + ((size_t)(slot - slot0) * 3 + c) * ntout;
        const int w0 = t0 - (nstf - 1), wl = CV_BLOCK + nstf - 1;
        __syncthreads();
        for (int k = tid; k < nstf; k += CV_THREADS) stf[k] = stfpool[t.stf + k];
        for (int y = tid; y < wl; y += CV_THREADS) {
            const int x = w0 + y;
            win[cv_pos(y, stride)] = x >= 0 && x < ntout ? uu[x] : 0.0f;
        }
        __syncthreads();
        /* acc_q = sum over k of stf[k] * u[base + q - k], k ascending
         * (stf_subs.c:25-33); window samples before the trace are zero and
         * add +-0 to an accumulator that starts at +0, which leaves it as the
         * reference's shorter sum leaves it */
        float acc[CV_Q], w[CV_Q];
#pragma unroll
        for (int q = 0; q < CV_Q; q++) {
            acc[q] = 0.0f;
            w[q] = win[cv_pos(tid * CV_Q + q + nstf - 1, stride)];
        }
        for (int k = 0; k < nstf; k++) {
            const float f = stf[k];
#pragma unroll
            for (int q = 0; q < CV_Q; q++) acc[q] = acc[q] + f * w[q];
#pragma unroll
            for (int q = CV_Q - 1; q > 0; q--) w[q] = w[q - 1];
            const int y = tid * CV_Q + nstf - 2 - k;
            w[0] = y >= 0 ? win[cv_pos(y, stride)] : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < CV_Q; q++) s[q] = s[q] + acc[q];     /* stf_subs.c:34-36 */
    }
#pragma unroll
    for (int q = 0; q < CV_Q; q++)
        if (base + q < ntout) out[base + q] = s[q];
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

struct Variation {
    int id;
    std::vector<awp_srf_point> pts;
    std::vector<float> pool;
};

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct awp_synth {
    awp_synth_params p;
    cudaStream_t stream = nullptr;
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
    DBuf<awp_synth_gterm> d_gt;
    DBuf<awp_synth_cterm> d_ct;
    DBuf<float> d_stf, d_u, d_seis;
    DBuf<int> d_slot_term, d_tl;
    DBuf<int2> d_range;
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
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&s->ev[i]);
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
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->d_sgt) cudaFree(s->d_sgt);
    s->d_gt.release();
    s->d_ct.release();
    s->d_stf.release();
    s->d_u.release();
    s->d_seis.release();
    s->d_slot_term.release();
    s->d_tl.release();
    s->d_range.release();
    for (auto &e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
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

extern "C" awp_status awp_synth_add_variation(awp_synth *s, int rup_var_id, const awp_srf_point *pts, int np,
                                              const float *pool, long long npool)
{
    if (!s || (np > 0 && !pts) || (npool > 0 && !pool) || np < 0 || npool < 0)
        return fail(AWP_ERR_PARAM, "awp_synth_add_variation: bad argument");
    if (!s->vars.empty() && (int)s->vars[0].pts.size() != np)
        return fail(AWP_ERR_PARAM, "awp_synth_add_variation: %d points, the rupture has %d", np,
                    (int)s->vars[0].pts.size());
    for (int i = 0; i < np; i++) {
        const awp_srf_point &a = pts[i];
        const int n[3] = {a.nt1, a.nt2, a.nt3};
        const long long o[3] = {a.stf1, a.stf2, a.stf3};
        for (int q = 0; q < 3; q++)
            if (n[q] < 0 || (n[q] > 0 && (o[q] < 0 || o[q] + n[q] > npool)))
                return fail(AWP_ERR_PARAM, "awp_synth_add_variation: point %d slip-rate samples outside the pool", i);
    }
    Variation v;
    v.id = rup_var_id;
    v.pts.assign(pts, pts + np);
    v.pool.assign(pool, pool + npool);
    s->vars.push_back(std::move(v));
    return AWP_OK;
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

extern "C" awp_status awp_synth_run(awp_synth *s)
{
    if (!s) return fail(AWP_ERR_PARAM, "awp_synth_run: null synth");
    if (!s->d_sgt) return fail(AWP_ERR_STATE, "awp_synth_run: no SGT set loaded");
    if (s->vars.empty()) return fail(AWP_ERR_STATE, "awp_synth_run: no rupture variation added");
    SCU(cudaSetDevice(s->p.device));
    const double tp0 = now_s();
    const int np = (int)s->vars[0].pts.size(), nv = (int)s->vars.size();
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

    s->seis.assign((size_t)nv * 3 * ntout, 0.0f);
    s->nseis = 0;
    s->info = awp_synth_info{};
    s->info.ncomp = s->ncomp;
    s->info.ntout = ntout;
    s->info.ntsum = ntsum;
    s->info.nsgt_points = nm;
    s->info.non_exact = non_exact;
    double plan_s = now_s() - tp0, dev_s = 0.0, conv_s = 0.0;
    int launches = 0;

    const int batch = s->p.rv_batch > 0 ? s->p.rv_batch : nv;
    for (int v0 = 0; v0 < nv; v0 += batch) {
        const double tb = now_s();
        const int nb = v0 + batch <= nv ? batch : nv - v0;
        /* per variation: terms and samples, then the plan in parallel */
        std::vector<long long> toff(nb + 1, 0), soff(nb + 1, 0);
        for (int b = 0; b < nb; b++) {
            const Variation &v = s->vars[v0 + b];
            long long ns = 0;
            for (auto &a : v.pts) ns += (a.nt1 > 0 ? a.nt1 : 0) + (a.nt2 > 0 ? a.nt2 : 0) + (a.nt3 > 0 ? a.nt3 : 0);
            toff[b + 1] = toff[b] + awp_synth_count_terms(v.pts.data(), np);
            soff[b + 1] = soff[b] + ns;
        }
        const long long nterm = toff[nb];
        if (nterm >= (1LL << 31)) return fail(AWP_ERR_PARAM, "awp_synth_run: too many terms in one batch; set rv_batch");
        std::vector<awp_synth_gterm> gt((size_t)nterm);
        std::vector<awp_synth_cterm> ctv((size_t)nterm);
        std::vector<float> stf((size_t)soff[nb] + 1);
        std::vector<long long> macs(nb, 0);
        std::vector<awp_status> pst(nb, AWP_OK);
#pragma omp parallel for schedule(dynamic, 1)
        for (int b = 0; b < nb; b++) {
            const Variation &v = s->vars[v0 + b];
            long long nterms = 0, nused = 0;
            pst[b] = awp_synth_plan_variation(&cx, v.pts.data(), v.pool.data(), (long long)v.pool.size(),
                                              gt.data() + toff[b], ctv.data() + toff[b], stf.data() + soff[b], soff[b],
                                              &nterms, &nused, &macs[b]);
        }
        for (int b = 0; b < nb; b++)
            if (pst[b] != AWP_OK) {
                /* the error text is per thread: plan the variation again here */
                const Variation &v = s->vars[v0 + b];
                long long a, c, d;
                return awp_synth_plan_variation(&cx, v.pts.data(), v.pool.data(), (long long)v.pool.size(),
                                                gt.data() + toff[b], ctv.data() + toff[b], stf.data() + soff[b],
                                                soff[b], &a, &c, &d);
            }
        for (int b = 0; b < nb; b++) s->info.macs += macs[b];
        s->info.terms += nterm;

        /* point-major slot order: slot -> term; each variation's slots in
         * point order (its term list for the convolution) */
        std::vector<long long> pstart((size_t)nb * (np + 1));
        for (int b = 0; b < nb; b++) {
            const Variation &v = s->vars[v0 + b];
            long long t = toff[b];
            for (int ip = 0; ip < np; ip++) {
                pstart[(size_t)b * (np + 1) + ip] = t;
                const awp_srf_point &a = v.pts[ip];
                t += (a.nt1 > 0) + (a.nt2 > 0) + (a.nt3 > 0);
            }
            pstart[(size_t)b * (np + 1) + np] = t;
        }
        std::vector<int> slot_term((size_t)nterm), tl((size_t)nterm), pslot(np + 1);
        long long sl = 0;
        for (int ip = 0; ip < np; ip++) {
            pslot[ip] = (int)sl;
            for (int b = 0; b < nb; b++) {
                const long long a0 = pstart[(size_t)b * (np + 1) + ip], a1 = pstart[(size_t)b * (np + 1) + ip + 1];
                for (long long t = a0; t < a1; t++) {
                    slot_term[sl] = (int)t;
                    tl[t] = (int)sl;          /* term t of variation b sits in slot sl */
                    sl++;
                }
            }
        }
        pslot[np] = (int)sl;
        /* a variation's terms are contiguous and in point order, so tl
         * indexed by term is each variation's slot list */
        int maxnstf = 1;
        for (auto &c : ctv) maxnstf = c.nstf > maxnstf ? c.nstf : maxnstf;

        const size_t slot_bytes = (size_t)3 * ntout * sizeof(float);
        long long cap = (long long)(s->u_cap_bytes / slot_bytes);
        if (cap < 1) cap = 1;
        long long maxslots = 0;
        for (int ip = 0; ip < np; ip++)
            maxslots = pslot[ip + 1] - pslot[ip] > maxslots ? pslot[ip + 1] - pslot[ip] : maxslots;
        if (maxslots > cap) cap = maxslots;   /* one point's terms always fit */
        const long long ucap = cap < nterm ? cap : (nterm > 0 ? nterm : 1);

        cudaError_t e = cudaSuccess;
        e = e ? e : s->d_gt.reserve((size_t)nterm);
        e = e ? e : s->d_ct.reserve((size_t)nterm);
        e = e ? e : s->d_stf.reserve(stf.size());
        e = e ? e : s->d_slot_term.reserve((size_t)nterm);
        e = e ? e : s->d_tl.reserve((size_t)nterm);
        e = e ? e : s->d_range.reserve((size_t)nb);
        e = e ? e : s->d_u.reserve((size_t)ucap * 3 * ntout);
        e = e ? e : s->d_seis.reserve((size_t)nb * 3 * ntout);
        if (e != cudaSuccess) return fail(AWP_ERR_OOM, "awp_synth_run: device buffers: %s", cudaGetErrorString(e));
        plan_s += now_s() - tb;

        SCU(cudaEventRecord(s->ev[0], s->stream));
        if (nterm) {
            SCU(cudaMemcpyAsync(s->d_gt.p, gt.data(), gt.size() * sizeof(awp_synth_gterm), cudaMemcpyHostToDevice,
                                s->stream));
            SCU(cudaMemcpyAsync(s->d_ct.p, ctv.data(), ctv.size() * sizeof(awp_synth_cterm), cudaMemcpyHostToDevice,
                                s->stream));
            SCU(cudaMemcpyAsync(s->d_slot_term.p, slot_term.data(), slot_term.size() * sizeof(int),
                                cudaMemcpyHostToDevice, s->stream));
            SCU(cudaMemcpyAsync(s->d_tl.p, tl.data(), tl.size() * sizeof(int), cudaMemcpyHostToDevice, s->stream));
        }
        SCU(cudaMemcpyAsync(s->d_stf.p, stf.data(), stf.size() * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        SCU(cudaMemsetAsync(s->d_seis.p, 0, (size_t)nb * 3 * ntout * sizeof(float), s->stream));

        /* convolution launch shape */
        const int stride = ((((CV_BLOCK + maxnstf - 1) + CV_Q - 1) / CV_Q + 1 + 27) / 32) * 32 + 4;
        const size_t cv_smem = sizeof(float) * (((maxnstf + 3) & ~3) + (size_t)CV_Q * stride);
        if (cv_smem > 227 * 1024) return fail(AWP_ERR_PARAM, "awp_synth_run: slip-rate functions too long");
        SCU(cudaFuncSetAttribute(k_synth_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cv_smem));
        std::vector<int2> range(nb);
        float conv_ms = 0.0f;
        for (int p0 = 0; p0 < np;) {
            int p1 = p0;
            while (p1 < np && pslot[p1 + 1] - pslot[p0] <= ucap) p1++;
            if (p1 == p0) p1 = p0 + 1;
            const long long s0 = pslot[p0], ns = pslot[p1] - pslot[p0];
            if (ns > 0) {
                const dim3 g1((unsigned)ns, (unsigned)((ntout + GF_THREADS - 1) / GF_THREADS));
                if (s->ncomp == 1)
                    k_synth_gf<1><<<g1, GF_THREADS, 0, s->stream>>>(s->d_sgt, nt, nt - SY_TAPLEN, s->d_gt.p,
                                                                    s->d_slot_term.p, s0, ntout, s->d_u.p);
                else if (s->ncomp == 2)
                    k_synth_gf<2><<<g1, GF_THREADS, 0, s->stream>>>(s->d_sgt, nt, nt - SY_TAPLEN, s->d_gt.p,
                                                                    s->d_slot_term.p, s0, ntout, s->d_u.p);
                else
                    k_synth_gf<3><<<g1, GF_THREADS, 0, s->stream>>>(s->d_sgt, nt, nt - SY_TAPLEN, s->d_gt.p,
                                                                    s->d_slot_term.p, s0, ntout, s->d_u.p);
                SCU(cudaGetLastError());
                for (int b = 0; b < nb; b++)
                    range[b] = make_int2((int)pstart[(size_t)b * (np + 1) + p0], (int)pstart[(size_t)b * (np + 1) + p1]);
                SCU(cudaMemcpyAsync(s->d_range.p, range.data(), nb * sizeof(int2), cudaMemcpyHostToDevice, s->stream));
                SCU(cudaEventRecord(s->ev[2], s->stream));
                const dim3 g2((unsigned)((ntout + CV_BLOCK - 1) / CV_BLOCK), 3, (unsigned)nb);
                k_synth_conv<<<g2, CV_THREADS, cv_smem, s->stream>>>(s->d_u.p, s->d_tl.p, s->d_range.p, s0,
                                                                      s->d_slot_term.p, s->d_ct.p, s->d_stf.p, ntout,
                                                                      stride, maxnstf, s->d_seis.p);
                SCU(cudaGetLastError());
                SCU(cudaEventRecord(s->ev[3], s->stream));
                /* the range table is rewritten by the next chunk */
                SCU(cudaEventSynchronize(s->ev[3]));
                float ms = 0.0f;
                SCU(cudaEventElapsedTime(&ms, s->ev[2], s->ev[3]));
                conv_ms += ms;
                launches += 2;
            }
            p0 = p1;
        }
        SCU(cudaMemcpyAsync(s->seis.data() + (size_t)v0 * 3 * ntout, s->d_seis.p, (size_t)nb * 3 * ntout * sizeof(float),
                            cudaMemcpyDeviceToHost, s->stream));
        SCU(cudaEventRecord(s->ev[1], s->stream));
        SCU(cudaEventSynchronize(s->ev[1]));
        float ms = 0.0f;
        SCU(cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]));
        dev_s += ms * 1e-3;
        conv_s += conv_ms * 1e-3;
    }
    s->nseis = nv;
    s->info.nvariations = nv;
    s->info.seconds_plan = plan_s;
    s->info.seconds_device = dev_s;
    s->info.seconds_conv = conv_s;
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
