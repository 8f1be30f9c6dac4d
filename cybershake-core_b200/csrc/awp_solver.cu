/*
 * awp_solver.cu -- C ABI of libawpsgt: solver object, device memory, media
 * ingest, time loop orchestration (CUDA graphs), SGT output.
 *
 * Host-side set-up restates, for the device layout of awp_internal.h:
 *   relax.f:4-39 (tausub), viscoop.f:79-88 (tau1/tau2), cerjan.f:4-247 (1-D
 *   sponge factors), structure.f:461-468 (Q-band constants), source.f:834-835,
 *   station.f:31-80 (point location), pmcl3d.f:1589-1601 (file offsets).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <new>

#include "awp_internal.h"
#include "awp_kernels.h"
#include "../../include/awp_sgt.h"

static thread_local char g_err[512];

static awp_status set_err(awp_status st, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return st;
}

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_err(e_ == cudaErrorMemoryAllocation ? AWP_ERR_OOM : AWP_ERR_CUDA,           \
                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);   \
    } while (0)

struct awp_solver {
    awp_params p;
    AwpGeom g;
    cudaStream_t stream;
    AwpComp comp[AWP_MAX_COMP];
    AwpMedia md;
    float *cx, *cy, *cz;
    float *tau;
    int *step;
    int *ext;
    float *chkj[AWP_MAX_COMP];
    int nsrc[AWP_MAX_COMP];
    int *src_ijk[AWP_MAX_COMP];
    float *src_stf[AWP_MAX_COMP];
    int npts;
    int *pt_idx;
    float *sg;
    float *sgt_file[AWP_MAX_COMP];
    int64_t sgt_file_floats;
    int64_t nt_file;
    int nsamp_written;
    int steps_done;
    int started;
    int media_loaded;
    int kchunk;
    float vtst, vtst1, dth, dh1;
    float ext_host[6];
    cudaEvent_t ev0, ev1;
    double loop_seconds;
    int64_t loop_steps;
    cudaGraphExec_t graph;
    int graph_steps;
    double device_bytes;
};

/* ------------------------------------------------------------------ */
/* small helpers                                                       */
/* ------------------------------------------------------------------ */

extern "C" const char *awp_last_error(void) { return g_err; }

extern "C" void awp_set_error_text(const char *msg) { snprintf(g_err, sizeof g_err, "%s", msg); }

extern "C" const char *awp_status_string(awp_status st)
{
    switch (st) {
    case AWP_OK: return "AWP_OK";
    case AWP_ERR_IO: return "AWP_ERR_IO";
    case AWP_ERR_PARAM: return "AWP_ERR_PARAM";
    case AWP_ERR_OOM: return "AWP_ERR_OOM";
    case AWP_ERR_CUDA: return "AWP_ERR_CUDA";
    case AWP_ERR_UNSTABLE: return "AWP_ERR_UNSTABLE";
    case AWP_ERR_TIMEOUT: return "AWP_ERR_TIMEOUT";
    case AWP_ERR_STATE: return "AWP_ERR_STATE";
    case AWP_ERR_BUSY: return "AWP_ERR_BUSY";
    case AWP_ERR_CANCELLED: return "AWP_ERR_CANCELLED";
    }
    return "AWP_ERR_UNKNOWN";
}

extern "C" void awp_free(void *p) { free(p); }

extern "C" void awp_params_default(awp_params *p)
{
    memset(p, 0, sizeof *p);
    p->nx = 224; p->ny = 224; p->nz = 1024;
    p->dh = 200.0f; p->dt = 0.01f;
    p->nt = (int)(20.0f / 0.01f) + 1;
    p->nd = 20; p->arbc = 0.92f;
    p->fl = 0.005f; p->fh = 5.0f; p->fp = 2.5f;
    p->socalq = 1; p->nve = 1; p->mediastart = 1; p->nvar = 3; p->idyna = 0;
    p->nst = 91; p->ntiskp_sgt = 1; p->write_step = 10;
    p->ncomp = 1; p->igreen[0] = 1; p->igreen[1] = 2; p->igreen[2] = 3;
    p->precision = AWP_PREC_F32; p->kernel = AWP_KERNEL_AUTO; p->device = 0;
    p->monitor_every = 0;
}

static AwpGeom make_geom(const awp_params *p)
{
    AwpGeom g;
    g.nx = p->nx; g.ny = p->ny; g.nz = p->nz;
    g.px = ((p->nx + AWP_XO + 2) + 7) / 8 * 8;
    g.py = p->ny + 4;
    g.plane = g.px * g.py;
    g.vol = (int64_t)g.plane * (p->nz + 4);
    return g;
}

static int64_t nt_file_of(const awp_params *p)
{
    return ((int64_t)(p->nt / p->write_step) * p->write_step) / p->ntiskp_sgt;
}

static int64_t file_floats_of(const awp_params *p, int npts)
{
    int64_t ntf = nt_file_of(p);
    int64_t n = (int64_t)npts * 6 * ntf;
    int nsamp = p->nt / p->ntiskp_sgt;
    int nchunk = nsamp / p->write_step;
    if (npts > 0 && nchunk > 0) {
        int64_t last = (int64_t)(npts - 1) * 6 * ntf + 5 * ntf + (int64_t)(nchunk - 1) * p->write_step + p->write_step;
        if (last > n) n = last;
    }
    return n;
}

extern "C" double awp_bytes_per_cell_update(const awp_params *p)
{
    const int nc = p->ncomp < 1 ? 1 : p->ncomp;
    const double mb = (p->precision == AWP_PREC_F32) ? 4.0 : 2.0;   /* media word  */
    const double rb = (p->precision == AWP_PREC_F32) ? 4.0 : 2.0;   /* r1..r6 word */
    const int nmedia = (p->nve == 1) ? 5 : 3;
    const int nr = (p->nve == 1) ? 12 : 0;          /* r1..r6 read + write       */
    /* two sweeps: velocity R 9 W 3 ; stress R 9 (u v w + 6 stresses) W 6 ; r R+W */
    const double state = 12 * 4.0 + 15 * 4.0 + nr * rb;
    return (nc * state + nmedia * mb) / nc;
}

static int choose_kchunk(const AwpGeom &g)
{
    const int bxy = ((g.nx + 31) / 32) * ((g.ny + 7) / 8);
    int nzb = (148 * 8 + bxy - 1) / bxy;
    if (nzb < 1) nzb = 1;
    int kc = (g.nz + nzb - 1) / nzb;
    if (kc < 8) kc = 8;
    if (kc > g.nz) kc = g.nz;
    return kc;
}

extern "C" int64_t awp_footprint_bytes(const awp_params *p, int npts)
{
    AwpGeom g = make_geom(p);
    const int nc = p->ncomp < 1 ? 1 : p->ncomp;
    int64_t b = (int64_t)g.vol * 4 * (AWP_NF_STATE * nc + AM_N);
    b += file_floats_of(p, npts) * 4 * nc;
    b += (int64_t)p->nt * 12 * nc;
    b += (int64_t)npts * 16;
    b += 64ll << 20;   /* media staging slab + small buffers */
    return b;
}

/* sponge factor of a face, cerjan.f:52 and :76 (float arithmetic) */
static float crj_low(float alpha, int nd, int g)
{
    float a = alpha * (float)(nd - g + 1);
    return expf(-(a * a));
}
static float crj_high(float alpha, int nd, int n, int g)
{
    float a = alpha * (float)(nd - (n - g));
    return expf(-(a * a));
}

static void free_all(awp_solver *s)
{
    if (!s) return;
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (int q = 0; q < AWP_MAX_COMP; q++) {
        for (int f = 0; f < AWP_NF_STATE; f++) cudaFree(s->comp[q].f[f]);
        cudaFree(s->chkj[q]);
        cudaFree(s->src_ijk[q]);
        cudaFree(s->src_stf[q]);
        cudaFree(s->sgt_file[q]);
    }
    for (int m = 0; m < AM_N; m++) cudaFree(s->md.m[m]);
    cudaFree(s->cx); cudaFree(s->cy); cudaFree(s->cz);
    cudaFree(s->tau); cudaFree(s->step); cudaFree(s->ext);
    cudaFree(s->pt_idx); cudaFree(s->sg);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
}

static awp_status dalloc(awp_solver *s, void **ptr, size_t bytes)
{
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        *ptr = NULL;
        return set_err(AWP_ERR_OOM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    s->device_bytes += (double)bytes;
    return AWP_OK;
}

static awp_status check_params(const awp_params *p)
{
    if (p->nx < 8 || p->ny < 8 || p->nz < 8) return set_err(AWP_ERR_PARAM, "grid %dx%dx%d too small (min 8)", p->nx, p->ny, p->nz);
    if (!(p->dh > 0) || !(p->dt > 0)) return set_err(AWP_ERR_PARAM, "DH and DT must be positive");
    if (p->nt < 1) return set_err(AWP_ERR_PARAM, "nt must be >= 1");
    if (p->nd < 1 || !(p->arbc > 0 && p->arbc < 1)) return set_err(AWP_ERR_PARAM, "ND >= 1 and 0 < ARBC < 1 required");
    if (p->ncomp < 1 || p->ncomp > AWP_MAX_COMP) return set_err(AWP_ERR_PARAM, "ncomp must be 1..3");
    if (p->ntiskp_sgt < 1 || p->write_step < 1) return set_err(AWP_ERR_PARAM, "NTISKP_SGT and WRITE_STEP must be >= 1");
    if (p->nst < 0) return set_err(AWP_ERR_PARAM, "NST must be >= 0");
    if (p->nvar != 3 && p->nvar != 5 && p->nvar != 8) return set_err(AWP_ERR_PARAM, "NVAR must be 3, 5 or 8");
    if (p->nve != 0 && p->nve != 1) return set_err(AWP_ERR_PARAM, "NVE must be 0 or 1");
    if (p->precision != AWP_PREC_F32) return set_err(AWP_ERR_PARAM, "precision %d not available in this build", p->precision);
    if (p->nve == 1 && !(p->fl > 0 && p->fh > p->fl && p->fp > 0)) return set_err(AWP_ERR_PARAM, "Q band needs 0 < FL < FH and FP > 0");
    for (int q = 0; q < p->ncomp; q++) {
        int ig = p->igreen[q];
        if (!(ig == -2 || ig == -1 || (ig >= 1 && ig <= 6))) return set_err(AWP_ERR_PARAM, "IGREEN %d not supported", ig);
    }
    AwpGeom g = make_geom(p);
    if (g.vol >= (int64_t)1 << 31) return set_err(AWP_ERR_PARAM, "grid too large for 32-bit field indexing");
    return AWP_OK;
}

/* ------------------------------------------------------------------ */
/* create / destroy                                                    */
/* ------------------------------------------------------------------ */

extern "C" awp_status awp_create(const awp_params *pin, awp_solver **out)
{
    *out = NULL;
    awp_status st = check_params(pin);
    if (st != AWP_OK) return st;
    CU(cudaSetDevice(pin->device));
    awp_solver *s = new (std::nothrow) awp_solver();
    if (!s) return set_err(AWP_ERR_OOM, "host allocation failed");
    memset(s, 0, sizeof *s);
    s->p = *pin;
    s->g = make_geom(pin);
    const awp_params *p = &s->p;
    const size_t vb = (size_t)s->g.vol * sizeof(float);
#define TRY(x) do { awp_status t_ = (x); if (t_ != AWP_OK) { free_all(s); delete s; return t_; } } while (0)
#define TRYCU(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { free_all(s); delete s; \
    return set_err(AWP_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); } } while (0)
    TRYCU(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    TRYCU(cudaEventCreate(&s->ev0));
    TRYCU(cudaEventCreate(&s->ev1));
    for (int q = 0; q < p->ncomp; q++)
        for (int f = 0; f < AWP_NF_STATE; f++) {
            if (p->nve == 0 && f >= AF_R1) continue;
            TRY(dalloc(s, (void **)&s->comp[q].f[f], vb));
            TRYCU(cudaMemsetAsync(s->comp[q].f[f], 0, vb, s->stream));
        }
    for (int m = 0; m < AM_N; m++) {
        TRY(dalloc(s, (void **)&s->md.m[m], vb));
        TRYCU(cudaMemsetAsync(s->md.m[m], 0, vb, s->stream));
    }
    /* sponge factors (cerjan.f:19-242): separable, both lateral faces and
     * the bottom damped, the free surface not */
    {
        float alpha = sqrtf(-logf(p->arbc)) / (float)p->nd;
        const int n3[3] = {p->nx, p->ny, p->nz};
        float *dst[3];
        for (int a = 0; a < 3; a++) {
            float *h = (float *)calloc((size_t)n3[a] + 2, sizeof(float));
            for (int i = 1; i <= n3[a]; i++) {
                float f = 1.0f;
                if (i <= p->nd) f = f * crj_low(alpha, p->nd, i);
                if (a < 2 && i >= n3[a] - p->nd + 1) f = f * crj_high(alpha, p->nd, n3[a], i);
                h[i] = f;
            }
            TRY(dalloc(s, (void **)&dst[a], sizeof(float) * ((size_t)n3[a] + 2)));
            cudaError_t e = cudaMemcpy(dst[a], h, sizeof(float) * ((size_t)n3[a] + 2), cudaMemcpyHostToDevice);
            free(h);
            if (a == 0) s->cx = dst[a]; else if (a == 1) s->cy = dst[a]; else s->cz = dst[a];
            TRYCU(e);
        }
    }
    TRY(dalloc(s, (void **)&s->tau, 16 * sizeof(float)));
    TRY(dalloc(s, (void **)&s->step, sizeof(int)));
    TRYCU(cudaMemsetAsync(s->step, 0, sizeof(int), s->stream));
    TRY(dalloc(s, (void **)&s->ext, 8 * sizeof(int)));
    for (int q = 0; q < p->ncomp; q++) {
        TRY(dalloc(s, (void **)&s->chkj[q], sizeof(float) * 3 * (size_t)p->nt));
        TRYCU(cudaMemsetAsync(s->chkj[q], 0, sizeof(float) * 3 * (size_t)p->nt, s->stream));
    }
    s->dth = p->dt / p->dh;
    s->dh1 = 1.0f / p->dh;
    s->vtst = p->dt / (p->dh * p->dh * p->dh);     /* source.f:834-835 */
    s->vtst1 = 1.0f / (p->dh * p->dh);
    s->kchunk = choose_kchunk(s->g);
    s->nt_file = nt_file_of(p);
    s->nsamp_written = ((p->nt / p->ntiskp_sgt) / p->write_step) * p->write_step;
    TRYCU(cudaStreamSynchronize(s->stream));
#undef TRY
#undef TRYCU
    *out = s;
    return AWP_OK;
}

extern "C" awp_status awp_destroy(awp_solver *s)
{
    if (!s) return AWP_OK;
    cudaSetDevice(s->p.device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_all(s);
    delete s;
    return AWP_OK;
}

/* ------------------------------------------------------------------ */
/* media                                                               */
/* ------------------------------------------------------------------ */

/* tausub (relax.f:15-36) and tau1/tau2 (viscoop.f:79-88), float arithmetic;
 * layout [itz][ity][itx] for tau1 then tau2 */
static awp_status upload_tau(awp_solver *s, float taumin, float taumax)
{
    static const int tautem[2][2][2] = {{{1, 6}, {7, 4}}, {{8, 3}, {2, 5}}};
    float h[16];
    const float dt1 = 1.0f / s->p.dt;
    for (int z = 0; z < 2; z++)
        for (int y = 0; y < 2; y++)
            for (int x = 0; x < 2; x++) {
                float tmp = (float)tautem[z][y][x];
                tmp = (tmp - 0.5f) / 8.0f;
                tmp = 2.0f * tmp - 1.0f;
                float tau = expf(0.5f * (logf(taumax * taumin) + logf(taumax / taumin) * tmp));
                h[(z * 2 + y) * 2 + x] = 1.0f / ((tau * dt1) + (1.0f / 2.0f));
                h[8 + (z * 2 + y) * 2 + x] = (tau * dt1) - (1.0f / 2.0f);
            }
    CU(cudaMemcpyAsync(s->tau, h, sizeof h, cudaMemcpyHostToDevice, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return AWP_OK;
}

static awp_status finish_media(awp_solver *s)
{
    int e[8];
    CU(cudaMemcpyAsync(e, s->ext, sizeof e, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    /* ext: vp_min vs_min rho_min vp_max vs_max rho_max */
    memcpy(&s->ext_host[0], &e[0], 4); memcpy(&s->ext_host[1], &e[3], 4);
    memcpy(&s->ext_host[2], &e[1], 4); memcpy(&s->ext_host[3], &e[4], 4);
    memcpy(&s->ext_host[4], &e[2], 4); memcpy(&s->ext_host[5], &e[5], 4);
    s->media_loaded = 1;
    if (s->npts > 0) {
        CU(awp_launch_sg_coeffs(s->g, s->md, s->npts, s->pt_idx, s->sg, s->stream));
        CU(cudaStreamSynchronize(s->stream));
    }
    return AWP_OK;
}

typedef int (*slab_reader)(void *ctx, float *dst, int zf0, int nzs, size_t floats_per_level);

static awp_status load_media_common(awp_solver *s, slab_reader rd, void *ctx)
{
    const awp_params *p = &s->p;
    CU(cudaSetDevice(p->device));
    if (s->started) return set_err(AWP_ERR_STATE, "media must be loaded before the first step (or after awp_reset)");
    const float pi = 4.0f * atanf(1.0f);
    if (p->mediastart == 0) {
        /* inihomo, structure.f:725-762 */
        float vp, vs, dd;
        if (p->idyna == 1) { vp = 6000.f; vs = 3464.f; dd = 2670.f; }
        else { vp = 4800.f; vs = 2800.f; dd = 2500.f; }
        const float lam = 1.0f / (dd * (vp * vp - 2.0f * vs * vs));
        const float mu = 1.0f / (dd * vs * vs);
        CU(awp_launch_media_homo(s->g, s->md, lam, mu, dd, s->stream));
        int e[8];
        float fv[6] = {vp, vs, dd, vp, vs, dd};
        memcpy(e, fv, sizeof fv);
        CU(cudaMemcpyAsync(s->ext, e, sizeof e, cudaMemcpyHostToDevice, s->stream));
        if (p->nve == 1) {
            awp_status st = upload_tau(s, 1.0f / (2 * pi * p->fh), 1.0f / (2 * pi * p->fl));
            if (st != AWP_OK) return st;
        }
        return finish_media(s);
    }
    int var_offset = (p->nvar == 8) ? 3 : 0;
    const float w0 = 2 * pi * p->fp, ww1 = 2 * pi * p->fl, w2 = 2 * pi * p->fh;
    const float taumax = 1.0f / ww1, taumin = 1.0f / w2;
    const float tmp1 = 2.0f / pi * (logf(taumax / taumin));
    const float tmp2 = 2.0f / pi * logf(w0 * taumin);
    const float lw = logf(w2 / w0);
    {
        int e[8];
        const float big = 99999.f, zero = 0.f;
        for (int q = 0; q < 3; q++) { memcpy(&e[q], &big, 4); memcpy(&e[3 + q], &zero, 4); }
        e[6] = e[7] = 0;
        CU(cudaMemcpyAsync(s->ext, e, sizeof e, cudaMemcpyHostToDevice, s->stream));
    }
    const size_t per_level = (size_t)p->nx * p->ny * p->nvar;
    int nzs = (int)((64ull << 20) / (per_level * sizeof(float)));
    if (nzs < 1) nzs = 1;
    if (nzs > p->nz) nzs = p->nz;
    float *hbuf = NULL, *dbuf = NULL;
    CU(cudaMallocHost((void **)&hbuf, per_level * nzs * sizeof(float)));
    cudaError_t e = cudaMalloc((void **)&dbuf, per_level * nzs * sizeof(float));
    if (e != cudaSuccess) { cudaFreeHost(hbuf); return set_err(AWP_ERR_OOM, "media staging: %s", cudaGetErrorString(e)); }
    awp_status st = AWP_OK;
    for (int z0 = 0; z0 < p->nz && st == AWP_OK; z0 += nzs) {
        const int n = (z0 + nzs <= p->nz) ? nzs : p->nz - z0;
        if (cudaStreamSynchronize(s->stream) != cudaSuccess) { st = set_err(AWP_ERR_CUDA, "media stream"); break; }
        if (rd(ctx, hbuf, z0, n, per_level) != 0) { st = set_err(AWP_ERR_IO, "media: short read at level %d", z0); break; }
        e = cudaMemcpyAsync(dbuf, hbuf, per_level * n * sizeof(float), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess)
            e = awp_launch_media_interior(s->g, s->md, dbuf, z0, n, p->nvar, var_offset, p->socalq, p->nve,
                                          pi, lw, tmp1, tmp2, s->ext, s->stream);
        if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "media upload: %s", cudaGetErrorString(e));
    }
    if (st == AWP_OK) {
        e = awp_launch_media_ghosts(s->g, s->md, p->nve, s->stream);
        if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "media ghosts: %s", cudaGetErrorString(e));
    }
    cudaStreamSynchronize(s->stream);
    cudaFree(dbuf);
    cudaFreeHost(hbuf);
    if (st != AWP_OK) return st;
    if (p->nve == 1) {
        st = upload_tau(s, taumin, taumax);
        if (st != AWP_OK) return st;
    }
    return finish_media(s);
}

struct mem_ctx { const float *base; };
static int mem_reader(void *ctx, float *dst, int zf0, int nzs, size_t per_level)
{
    const mem_ctx *m = (const mem_ctx *)ctx;
    memcpy(dst, m->base + per_level * (size_t)zf0, per_level * (size_t)nzs * sizeof(float));
    return 0;
}
struct file_ctx { FILE *f; };
static int file_reader(void *ctx, float *dst, int zf0, int nzs, size_t per_level)
{
    file_ctx *fc = (file_ctx *)ctx;
    (void)zf0;
    size_t n = per_level * (size_t)nzs;
    return fread(dst, sizeof(float), n, fc->f) == n ? 0 : -1;
}

extern "C" awp_status awp_load_media(awp_solver *s, const float *media)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    if (s->p.mediastart != 0 && !media) return set_err(AWP_ERR_PARAM, "media array required when MEDIARESTART != 0");
    mem_ctx m = {media};
    return load_media_common(s, mem_reader, &m);
}

extern "C" awp_status awp_load_media_file(awp_solver *s, const char *path)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    if (s->p.mediastart == 0) return load_media_common(s, mem_reader, NULL);
    FILE *f = fopen(path, "rb");
    if (!f) return set_err(AWP_ERR_IO, "cannot open media file %s", path);
    file_ctx fc = {f};
    awp_status st = load_media_common(s, file_reader, &fc);
    fclose(f);
    return st;
}

/* ------------------------------------------------------------------ */
/* sources and points                                                  */
/* ------------------------------------------------------------------ */

extern "C" awp_status awp_set_source(awp_solver *s, int comp, int nsrc, const int *xyz, const float *stf)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    const awp_params *p = &s->p;
    if (comp < 0 || comp >= p->ncomp) return set_err(AWP_ERR_PARAM, "component %d out of range", comp);
    if (nsrc < 0 || (nsrc > 0 && (!xyz || !stf))) return set_err(AWP_ERR_PARAM, "bad source arrays");
    if (s->started) return set_err(AWP_ERR_STATE, "sources must be set before the first step");
    /* bounds check of source.f:176-187, reported instead of stopping */
    for (int m = 0; m < nsrc; m++) {
        if (xyz[3 * m] < 1 || xyz[3 * m] > p->nx) return set_err(AWP_ERR_PARAM, "X source coordinate %d is outside range 1-%d", xyz[3 * m], p->nx);
        if (xyz[3 * m + 1] < 1 || xyz[3 * m + 1] > p->ny) return set_err(AWP_ERR_PARAM, "Y source coordinate %d is outside range 1-%d", xyz[3 * m + 1], p->ny);
        if (xyz[3 * m + 2] < 1 || xyz[3 * m + 2] > p->nz) return set_err(AWP_ERR_PARAM, "Z source coordinate %d is outside range 1-%d", xyz[3 * m + 2], p->nz);
    }
    CU(cudaSetDevice(p->device));
    cudaFree(s->src_ijk[comp]); s->src_ijk[comp] = NULL;
    cudaFree(s->src_stf[comp]); s->src_stf[comp] = NULL;
    s->nsrc[comp] = nsrc;
    if (nsrc == 0) return AWP_OK;
    int *ijk = (int *)malloc(sizeof(int) * 3 * (size_t)nsrc);
    for (int m = 0; m < nsrc; m++) {
        ijk[3 * m] = xyz[3 * m];
        ijk[3 * m + 1] = xyz[3 * m + 1];
        ijk[3 * m + 2] = p->nz + 1 - xyz[3 * m + 2];
    }
    awp_status st = dalloc(s, (void **)&s->src_ijk[comp], sizeof(int) * 3 * (size_t)nsrc);
    if (st == AWP_OK) st = dalloc(s, (void **)&s->src_stf[comp], sizeof(float) * 6 * (size_t)nsrc * (size_t)(p->nst > 0 ? p->nst : 1));
    if (st == AWP_OK) {
        cudaError_t e = cudaMemcpy(s->src_ijk[comp], ijk, sizeof(int) * 3 * (size_t)nsrc, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && p->nst > 0)
            e = cudaMemcpy(s->src_stf[comp], stf, sizeof(float) * 6 * (size_t)nsrc * (size_t)p->nst, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "source upload: %s", cudaGetErrorString(e));
    }
    free(ijk);
    return st;
}

extern "C" awp_status awp_set_points(awp_solver *s, int npts, const int *xyz)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    const awp_params *p = &s->p;
    if (npts < 0 || (npts > 0 && !xyz)) return set_err(AWP_ERR_PARAM, "bad point arrays");
    if (s->started) return set_err(AWP_ERR_STATE, "points must be set before the first step");
    for (int n = 0; n < npts; n++) {
        if (xyz[3 * n] < 1 || xyz[3 * n] > p->nx || xyz[3 * n + 1] < 1 || xyz[3 * n + 1] > p->ny ||
            xyz[3 * n + 2] < 1 || xyz[3 * n + 2] > p->nz)
            return set_err(AWP_ERR_PARAM, "SGT point %d (%d,%d,%d) outside the grid", n, xyz[3 * n], xyz[3 * n + 1], xyz[3 * n + 2]);
    }
    CU(cudaSetDevice(p->device));
    cudaFree(s->pt_idx); s->pt_idx = NULL;
    cudaFree(s->sg); s->sg = NULL;
    for (int q = 0; q < AWP_MAX_COMP; q++) { cudaFree(s->sgt_file[q]); s->sgt_file[q] = NULL; }
    s->npts = npts;
    s->sgt_file_floats = file_floats_of(p, npts);
    if (npts == 0) return AWP_OK;
    int *idx = (int *)malloc(sizeof(int) * (size_t)npts);
    for (int n = 0; n < npts; n++)   /* station.f:42-52: k = nz - z + 1 */
        idx[n] = s->g.idx(xyz[3 * n], xyz[3 * n + 1], p->nz - xyz[3 * n + 2] + 1);
    awp_status st = dalloc(s, (void **)&s->pt_idx, sizeof(int) * (size_t)npts);
    if (st == AWP_OK) st = dalloc(s, (void **)&s->sg, sizeof(float) * 3 * (size_t)npts);
    for (int q = 0; q < p->ncomp && st == AWP_OK; q++) {
        st = dalloc(s, (void **)&s->sgt_file[q], sizeof(float) * (size_t)(s->sgt_file_floats > 0 ? s->sgt_file_floats : 1));
        if (st == AWP_OK && cudaMemset(s->sgt_file[q], 0, sizeof(float) * (size_t)(s->sgt_file_floats > 0 ? s->sgt_file_floats : 1)) != cudaSuccess)
            st = set_err(AWP_ERR_CUDA, "memset SGT file image");
    }
    if (st == AWP_OK && cudaMemcpy(s->pt_idx, idx, sizeof(int) * (size_t)npts, cudaMemcpyHostToDevice) != cudaSuccess)
        st = set_err(AWP_ERR_CUDA, "point upload");
    free(idx);
    if (st == AWP_OK && s->media_loaded) {
        cudaError_t e = awp_launch_sg_coeffs(s->g, s->md, s->npts, s->pt_idx, s->sg, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "sg coefficients: %s", cudaGetErrorString(e));
    }
    return st;
}

extern "C" int64_t awp_sgt_file_floats(const awp_solver *s) { return s ? s->sgt_file_floats : 0; }

/* ------------------------------------------------------------------ */
/* time loop                                                           */
/* ------------------------------------------------------------------ */

static void fill_args(awp_solver *s, AwpStepArgs &a, AwpPostArgs &pa, AwpSgtArgs &sa)
{
    const awp_params *p = &s->p;
    memset(&a, 0, sizeof a);
    a.g = s->g; a.md = s->md; a.ncomp = p->ncomp;
    for (int q = 0; q < p->ncomp; q++) a.comp[q] = s->comp[q];
    a.cx = s->cx; a.cy = s->cy; a.cz = s->cz; a.tau = s->tau;
    a.dth = s->dth; a.dt = p->dt; a.dh1 = s->dh1; a.kchunk = s->kchunk; a.nve = p->nve;

    memset(&pa, 0, sizeof pa);
    pa.g = s->g; pa.ncomp = p->ncomp; pa.nst = p->nst; pa.nt = p->nt;
    pa.vtst = s->vtst; pa.vtst1 = s->vtst1;
    const int q0 = p->nd + 2;
    pa.probe = (q0 <= p->nx && q0 <= p->ny && q0 <= p->nz) ? q0 : 0;
    pa.step = s->step;
    pa.d1 = s->md.m[AM_D1];
    for (int q = 0; q < p->ncomp; q++) {
        pa.chkj[q] = s->chkj[q];
        pa.src[q].igreen = p->igreen[q];
        pa.src[q].nsrc = s->nsrc[q];
        pa.src[q].ijk = s->src_ijk[q];
        pa.src[q].stf = s->src_stf[q];
        pa.comp[q] = s->comp[q];
    }

    memset(&sa, 0, sizeof sa);
    sa.g = s->g; sa.ncomp = p->ncomp; sa.npts = s->npts; sa.ntiskp = p->ntiskp_sgt;
    sa.nsamp_written = s->nsamp_written; sa.nt_file = s->nt_file;
    sa.pt_idx = s->pt_idx; sa.sg = s->sg; sa.step = s->step;
    for (int q = 0; q < p->ncomp; q++) {
        sa.file[q] = s->sgt_file[q];
        sa.comp[q] = s->comp[q];
    }
}

static cudaError_t enqueue_steps(awp_solver *s, int nsteps)
{
    AwpStepArgs a; AwpPostArgs pa; AwpSgtArgs sa;
    fill_args(s, a, pa, sa);
    const bool any_sgt = s->npts > 0;
    for (int n = 0; n < nsteps; n++) {
        cudaError_t e = awp_launch_step(a, s->stream);
        if (e == cudaSuccess) e = awp_launch_post(pa, 0, s->stream);
        if (e == cudaSuccess && any_sgt && ((s->steps_done + n + 1) % s->p.ntiskp_sgt == 0))
            e = awp_launch_sgt(sa, s->stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

/* CUDA graph of NTISKP_SGT steps followed by the SGT gather; the kernels read
 * the device step counter, so the same graph replays for every chunk. */
static cudaError_t build_graph(awp_solver *s)
{
    if (s->graph) return cudaSuccess;
    const int gs = s->p.ntiskp_sgt;
    cudaGraph_t graph;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    AwpStepArgs a; AwpPostArgs pa; AwpSgtArgs sa;
    fill_args(s, a, pa, sa);
    cudaError_t le = cudaSuccess;
    for (int n = 0; n < gs && le == cudaSuccess; n++) {
        le = awp_launch_step(a, s->stream);
        if (le == cudaSuccess) le = awp_launch_post(pa, 0, s->stream);
    }
    if (le == cudaSuccess && s->npts > 0) le = awp_launch_sgt(sa, s->stream);
    e = cudaStreamEndCapture(s->stream, &graph);
    if (le != cudaSuccess) { if (e == cudaSuccess) cudaGraphDestroy(graph); return le; }
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&s->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { s->graph = NULL; return e; }
    s->graph_steps = gs;
    return cudaSuccess;
}

static awp_status start_if_needed(awp_solver *s)
{
    if (s->started) return AWP_OK;
    if (!s->media_loaded) return set_err(AWP_ERR_STATE, "media not loaded");
    AwpStepArgs a; AwpPostArgs pa; AwpSgtArgs sa;
    fill_args(s, a, pa, sa);
    CU(awp_launch_post(pa, 1, s->stream));     /* addsrc(1) */
    s->started = 1;
    return AWP_OK;
}

extern "C" awp_status awp_run(awp_solver *s, int nsteps, float *sgt_out)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    const awp_params *p = &s->p;
    CU(cudaSetDevice(p->device));
    awp_status st = start_if_needed(s);
    if (st != AWP_OK) return st;
    if (nsteps < 0) return set_err(AWP_ERR_PARAM, "nsteps < 0");
    int todo = nsteps;
    if (todo > p->nt - s->steps_done) todo = p->nt - s->steps_done;
    if (todo > 0) {
        CU(cudaEventRecord(s->ev0, s->stream));
        int left = todo;
        /* align to the graph period with single steps */
        const int gs = p->ntiskp_sgt;
        int head = (gs - (s->steps_done % gs)) % gs;
        if (head > left) head = left;
        if (head > 0) {
            CU(enqueue_steps(s, head));
            s->steps_done += head; left -= head;
        }
        if (left >= gs && gs >= 1 && gs <= 64) {
            CU(build_graph(s));
            while (left >= gs) {
                CU(cudaGraphLaunch(s->graph, s->stream));
                s->steps_done += gs; left -= gs;
            }
        }
        if (left > 0) {
            CU(enqueue_steps(s, left));
            s->steps_done += left;
        }
        CU(cudaEventRecord(s->ev1, s->stream));
        CU(cudaEventSynchronize(s->ev1));
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
        s->loop_seconds += ms * 1e-3;
        s->loop_steps += todo;
    }
    if (sgt_out) {
        for (int q = 0; q < p->ncomp; q++) {
            st = awp_get_sgt(s, q, sgt_out + (size_t)q * (size_t)s->sgt_file_floats);
            if (st != AWP_OK) return st;
        }
    }
    return AWP_OK;
}

extern "C" awp_status awp_get_sgt(awp_solver *s, int comp, float *out)
{
    if (!s || comp < 0 || comp >= s->p.ncomp) return set_err(AWP_ERR_PARAM, "bad solver/component");
    if (s->sgt_file_floats <= 0) return AWP_OK;
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    CU(cudaMemcpy(out, s->sgt_file[comp], sizeof(float) * (size_t)s->sgt_file_floats, cudaMemcpyDeviceToHost));
    return AWP_OK;
}

extern "C" awp_status awp_get_chkj(awp_solver *s, int comp, float *out)
{
    if (!s || comp < 0 || comp >= s->p.ncomp) return set_err(AWP_ERR_PARAM, "bad solver/component");
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    CU(cudaMemcpy(out, s->chkj[comp], sizeof(float) * 3 * (size_t)s->p.nt, cudaMemcpyDeviceToHost));
    return AWP_OK;
}

extern "C" awp_status awp_get_field(awp_solver *s, int comp, int field, float *out)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    const float *src = NULL;
    if (field >= 0 && field < AWP_NF_STATE) {
        if (comp < 0 || comp >= s->p.ncomp) return set_err(AWP_ERR_PARAM, "bad component");
        src = s->comp[comp].f[field];
    } else if (field >= AWP_NF_STATE && field < AWP_NF_STATE + AM_N) {
        src = s->md.m[field - AWP_NF_STATE];
    }
    if (!src) return set_err(AWP_ERR_PARAM, "field %d not held by this solver", field);
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    const AwpGeom &g = s->g;
    const size_t w = (size_t)(g.nx + 4);
    CU(cudaMemcpy2D(out, w * sizeof(float), src + (AWP_XO - 2), (size_t)g.px * sizeof(float),
                    w * sizeof(float), (size_t)(g.ny + 4) * (size_t)(g.nz + 4), cudaMemcpyDeviceToHost));
    return AWP_OK;
}

extern "C" awp_status awp_get_stats(awp_solver *s, awp_stats *o)
{
    if (!s || !o) return set_err(AWP_ERR_PARAM, "null argument");
    memset(o, 0, sizeof *o);
    o->steps_done = s->steps_done;
    o->seconds_loop = s->loop_seconds;
    const double cells = (double)s->p.nx * s->p.ny * s->p.nz * s->p.ncomp;
    o->gcell_updates_per_s = s->loop_seconds > 0 ? cells * (double)s->loop_steps / s->loop_seconds * 1e-9 : 0.0;
    o->bytes_per_cell_update = awp_bytes_per_cell_update(&s->p);
    o->device_bytes = s->device_bytes;
    o->vp_min = s->ext_host[0]; o->vp_max = s->ext_host[1];
    o->vs_min = s->ext_host[2]; o->vs_max = s->ext_host[3];
    o->rho_min = s->ext_host[4]; o->rho_max = s->ext_host[5];
    return AWP_OK;
}

extern "C" awp_status awp_reset(awp_solver *s)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    const awp_params *p = &s->p;
    CU(cudaSetDevice(p->device));
    CU(cudaStreamSynchronize(s->stream));
    const size_t vb = (size_t)s->g.vol * sizeof(float);
    for (int q = 0; q < p->ncomp; q++) {
        for (int f = 0; f < AWP_NF_STATE; f++)
            if (s->comp[q].f[f]) CU(cudaMemsetAsync(s->comp[q].f[f], 0, vb, s->stream));
        CU(cudaMemsetAsync(s->chkj[q], 0, sizeof(float) * 3 * (size_t)p->nt, s->stream));
        if (s->sgt_file[q]) CU(cudaMemsetAsync(s->sgt_file[q], 0, sizeof(float) * (size_t)s->sgt_file_floats, s->stream));
    }
    CU(cudaMemsetAsync(s->step, 0, sizeof(int), s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->steps_done = 0;
    s->started = 0;
    s->loop_seconds = 0;
    s->loop_steps = 0;
    return AWP_OK;
}
