/*
 * awp_solver.cu -- C ABI of libawpsgt: solver object, device memory, media
 * ingest, time loop orchestration (CUDA graphs), SGT output.
 *
 * Host-side set-up restates, for the device layout of awp_internal.h:
 *   relax.f:4-39 (tausub), viscoop.f:79-88 (tau1/tau2), cerjan.f:4-247 (1-D
 *   sponge factors), structure.f:461-468 (Q-band constants), source.f:834-835,
 *   station.f:31-80 (point location), pmcl3d.f:1589-1601 (file offsets).
 *
 * Steppers: the fused single-sweep kernel (default) reads one wavefield
 * buffer and writes the other, alternating every step; the two-sweep stepper
 * updates one buffer in place.  Memory variables r1..r6 are updated in place
 * by both.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "awp_internal.h"
#include "awp_kernels.h"
#include "../../include/awp_sgt.h"

/* NVTX range over a scope: solver phases show up by name on an Nsight
 * timeline (header-only NVTX 3; without a tool attached a push or pop is a
 * branch on a null pointer) */
struct NvtxScope {
    explicit NvtxScope(const char *name) { nvtxRangePushA(name); }
    ~NvtxScope() { nvtxRangePop(); }
};

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
    AwpComp comp[2][AWP_MAX_COMP];   /* [buffer][component]; r1..r6 shared  */
    int fused;
    int store;                       /* AWP_STORE_* of the media arrays     */
    int rstore;                      /* AWP_STORE_* of r1..r6               */
    AwpMedia md;                     /* FP32 media (ingest)                 */
    AwpMediaT mdt;                   /* media as the steppers read them     */
    float *cx, *cy, *cz;
    float *tau;
    int *step;
    int *ext;
    unsigned *rng;                   /* [2][AM_N] media |value| max / min   */
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
    int kchunk;                      /* z levels per fused work item        */
    int kchunk_sweep;                /* z levels per two-sweep work item    */
    int staged_on;                   /* TMA-staged velocity/stress sweeps   */
    float *kin[AWP_MAX_COMP];        /* kinematic subfault increments       */
    size_t stagger;                  /* base-address offset step of the field arrays */
    int nstag;
    struct { void *user, *raw; } stag[128];
    int kchunk_staged;               /* z levels per staged work item       */
    int staged_qslow;                /* staged items: component slowest     */
    int staged_rpt;                  /* staged stress sweep rows per thread */
    int staged_rpt_vel;              /* staged velocity sweep rows per thread */
    int staged_batch;                /* staged stress: components in one item */
    int staged_generic;              /* staged one-component sweeps: generic ring loads */
    int sm_limit;                    /* persistent grids for this many SMs (0 = all) */
    int fma;                         /* staged sweeps with multiply-add contraction */
    /* PML (npc = 1): split arrays per component, damping profiles, kernel arguments */
    float *pml_split[AWP_MAX_COMP];
    float *pml_prof;                 /* rf[nd + 1] then rh[nd + 1]         */
    int64_t pml_floats;              /* floats of one component's splits   */
    AwpPmlArgs pml_args;
    AwpStaged *staged;               /* their tensor maps (first step)      */
    int ty;                          /* thread-block rows of the steppers   */
    int unroll;                      /* two-sweep z-loop unroll             */
    float vtst, vtst1, dth, dh1;
    float ext_host[6];
    cudaEvent_t ev0, ev1;
    double loop_seconds;
    int64_t loop_steps;
    cudaGraphExec_t graph[2];        /* by the parity of the first step    */
    double device_bytes;
    /* stability monitor */
    double *en_partial;              /* scratch: AWP_EN_GRID * ncomp       */
    double *en_out;                  /* last energy per component          */
    int *flag;                       /* set by the monitor on NaN/Inf      */
    int next_check;
    int pending;                     /* asynchronous steps not yet synced  */
    int pending_steps;
    /* failure injection for tests (environment, read by awp_create) */
    unsigned long long wait_ns;      /* bound of a staged barrier wait (AWP_TEST_WAIT_US) */
    int withhold;                    /* AWP_TEST_TMA_WITHHOLD: ring use block 0 withholds, -1 off */
    int fail_alloc;                  /* AWP_TEST_FAIL_ALLOC: that device allocation fails, 0 off */
    int nalloc;                      /* device allocations so far          */
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
    p->npc = 0; p->pht = 0.1f;
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

/* storage of the media arrays */
static int store_of(const awp_params *p)
{
    return p->precision == AWP_PREC_BF16 ? AWP_STORE_BF16 : p->precision == AWP_PREC_F16 ? AWP_STORE_F16 : AWP_STORE_F32;
}
/* storage of r1..r6 */
static int rstore_of(const awp_params *p)
{
    return p->precision == AWP_PREC_F32 ? AWP_STORE_F32 : (p->precision == AWP_PREC_BFP ? AWP_STORE_BFP : AWP_STORE_BF16);
}
static int fused_of(const awp_params *p) { return p->kernel == AWP_KERNEL_FUSED; }
static double media_word(int store) { return store == AWP_STORE_F32 ? 4.0 : 2.0; }

extern "C" double awp_bytes_per_cell_update(const awp_params *p)
{
    const int nc = p->ncomp < 1 ? 1 : p->ncomp;
    const int st = store_of(p);
    const double mb = media_word(st);
    const double rcell = (p->nve == 1) ? 2.0 * awp_r_bytes(rstore_of(p)) : 0.0;   /* r1..r6 read+write */
    const int nmedia = (p->nve == 1) ? 5 : 3;
    double state;
    if (fused_of(p))
        state = 18 * 4.0 + rcell;                      /* u v w + 6 stresses R+W */
    else
        state = 12 * 4.0 + 15 * 4.0 + rcell;           /* vel R9 W3; stress R9 W6 */
    return (nc * state + nmedia * mb) / nc;
}

/* tuning overrides from the environment (AWP_TUNE_TY, AWP_TUNE_KCHUNK) */
static int env_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return (v && *v) ? atoi(v) : dflt;
}

/* z levels per work item of the persistent steppers: enough items to keep
 * every SM busy (about eight per SM), but chunks no shorter than kmin -- the
 * fused stepper recomputes four velocity levels per chunk -- nor longer than
 * kmax; a top chunk always holds at least the three levels fstr reads. */
static int choose_kchunk(const AwpGeom &g, int fused, int ty)
{
    const int over = env_int(fused ? "AWP_TUNE_KCHUNK" : "AWP_TUNE_KSWEEP", 0);
    if (over > 0) return over < 8 ? 8 : (over > g.nz ? g.nz : over);
    const int tiles = ((g.nx + 31) / 32) * ((g.ny + ty - 1) / ty);
    const int want = 148 * 8;
    int nzc = (want + tiles - 1) / tiles;
    if (nzc < 1) nzc = 1;
    int kc = (g.nz + nzc - 1) / nzc;
    const int kmin = fused ? 16 : 8, kmax = fused ? 64 : 8;
    if (kc < kmin) kc = kmin;
    if (kc > kmax) kc = kmax;
    if (kc > g.nz) kc = g.nz;
    return kc;
}

extern "C" int64_t awp_footprint_bytes(const awp_params *p, int npts)
{
    AwpGeom g = make_geom(p);
    const int nc = p->ncomp < 1 ? 1 : p->ncomp;
    const int st = store_of(p);
    const double mb = media_word(st);
    const int nbuf = fused_of(p) ? 2 : 1;
    const double rcell = p->nve == 1 ? awp_r_bytes(rstore_of(p)) : 0;
    int64_t b = (int64_t)g.vol * (int64_t)(nc * (9 * 4 * nbuf + rcell));
    b += (int64_t)g.vol * (int64_t)(AM_N * 4);                        /* FP32 media during ingest */
    if (st != AWP_STORE_F32) b += (int64_t)g.vol * (int64_t)(AM_N * mb);
    b += file_floats_of(p, npts) * 4 * nc;
    b += (int64_t)p->nt * 12 * nc;
    b += (int64_t)npts * 16;
    if (p->npc == 1)   /* PML split arrays */
        b += (int64_t)nc * 18 * 4 *
             (2 * (int64_t)p->nx * p->nd * p->nz + 2 * (int64_t)p->nd * p->ny * p->nz + (int64_t)p->nx * p->ny * p->nd);
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

static void dfree_field(awp_solver *s, void *p);
static void dfree(awp_solver *s, void *p);

static void free_media32(awp_solver *s)
{
    for (int m = 0; m < AM_N; m++) {
        if (s->md.m[m] && (void *)s->md.m[m] != s->mdt.m[m]) {
            dfree_field(s, s->md.m[m]);
            s->device_bytes -= (double)s->g.vol * 4;
        }
        s->md.m[m] = NULL;
    }
}

static void free_all(awp_solver *s)
{
    if (!s) return;
    for (int b = 0; b < 2; b++)
        if (s->graph[b]) cudaGraphExecDestroy(s->graph[b]);
    for (int q = 0; q < AWP_MAX_COMP; q++) {
        for (int f = 0; f < AWP_NF_ARRAYS; f++) {
            dfree_field(s, s->comp[0][q].f[f]);
            if (f < AF_R1 && s->comp[1][q].f[f] != s->comp[0][q].f[f]) dfree_field(s, s->comp[1][q].f[f]);
        }
        dfree(s, s->chkj[q]);
        dfree(s, s->src_ijk[q]);
        dfree(s, s->src_stf[q]);
        dfree(s, s->kin[q]);
        dfree(s, s->sgt_file[q]);
    }
    free_media32(s);
    awp_staged_destroy(s->staged);
    for (int m = 0; m < AM_N; m++) dfree_field(s, s->mdt.m[m]);
    dfree(s, s->cx); dfree(s, s->cy); dfree(s, s->cz);
    dfree(s, s->tau); dfree(s, s->step); dfree(s, s->ext); dfree(s, s->rng);
    dfree(s, s->pt_idx); dfree(s, s->sg);
    dfree(s, s->en_partial); dfree(s, s->en_out); dfree(s, s->flag);
    for (int q = 0; q < AWP_MAX_COMP; q++) dfree(s, s->pml_split[q]);
    dfree(s, s->pml_prof);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
}

/* ------------------------------------------------------------------ */
/* device block cache                                                  */
/* ------------------------------------------------------------------ */

/* Blocks a solver frees stay on the device for the next solver of the
 * process: the next job on the same grid asks for the same sizes, so its
 * create skips cudaMalloc and its destroy skips cudaFree, whose device-wide
 * synchronisation would also stall the other solvers of a server.  An idle
 * block is reused for a request of its size or up to 1/8 smaller (the
 * smallest such block).  A failed cudaMalloc returns the device's idle blocks
 * and tries again.  AWP_DEVICE_CACHE_MB bounds the idle bytes per device
 * (default: half the device memory; 0 turns the cache off).  Callers hand a
 * block back only when no queued work uses it. */
namespace {
struct BlkInfo {
    int dev;
    size_t bytes;
};
std::mutex g_blk_mu;
std::unordered_map<void *, BlkInfo> g_blk_live;
std::multimap<std::pair<int, size_t>, void *> g_blk_idle;
std::map<int, size_t> g_blk_idle_bytes, g_blk_limit;
}

static size_t blk_limit_locked(int dev)
{
    auto it = g_blk_limit.find(dev);
    if (it != g_blk_limit.end()) return it->second;
    size_t lim = 0;
    if (const char *e = getenv("AWP_DEVICE_CACHE_MB")) {
        lim = (size_t)strtoull(e, NULL, 10) << 20;
    } else {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) lim = prop.totalGlobalMem / 2;
    }
    g_blk_limit[dev] = lim;
    return lim;
}

/* frees idle blocks of `dev` (all of them when dev < 0) */
static void blk_trim(int dev)
{
    std::vector<void *> out;
    {
        std::lock_guard<std::mutex> lk(g_blk_mu);
        for (auto it = g_blk_idle.begin(); it != g_blk_idle.end();) {
            if (dev < 0 || it->first.first == dev) {
                g_blk_idle_bytes[it->first.first] -= it->first.second;
                out.push_back(it->second);
                it = g_blk_idle.erase(it);
            } else {
                ++it;
            }
        }
    }
    for (void *p : out) cudaFree(p);
}

static cudaError_t blk_alloc(int dev, void **ptr, size_t bytes)
{
    {
        std::lock_guard<std::mutex> lk(g_blk_mu);
        auto it = g_blk_idle.lower_bound(std::make_pair(dev, bytes));
        if (it != g_blk_idle.end() && it->first.first == dev && it->first.second - bytes <= bytes / 8) {
            const size_t have = it->first.second;
            *ptr = it->second;
            g_blk_idle.erase(it);
            g_blk_idle_bytes[dev] -= have;
            g_blk_live[*ptr] = BlkInfo{dev, have};
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        blk_trim(dev);
        e = cudaMalloc(ptr, bytes);
    }
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_blk_mu);
    g_blk_live[*ptr] = BlkInfo{dev, bytes};
    return cudaSuccess;
}

static void blk_free(void *p)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_blk_mu);
        auto it = g_blk_live.find(p);
        if (it != g_blk_live.end()) {
            const BlkInfo b = it->second;
            g_blk_live.erase(it);
            if (g_blk_idle_bytes[b.dev] + b.bytes <= blk_limit_locked(b.dev)) {
                g_blk_idle.emplace(std::make_pair(b.dev, b.bytes), p);
                g_blk_idle_bytes[b.dev] += b.bytes;
                return;
            }
        }
    }
    cudaFree(p);
}

/* a solver's block back to the cache, once the solver's queued work is done */
static void dfree(awp_solver *s, void *p)
{
    if (!p) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    blk_free(p);
}

extern "C" void awp_release_cached_memory(void) { blk_trim(-1); }

extern "C" awp_status awp_device_memory(int device, int64_t *live_bytes, int64_t *idle_bytes)
{
    if (!live_bytes || !idle_bytes) return set_err(AWP_ERR_PARAM, "null argument");
    std::lock_guard<std::mutex> lk(g_blk_mu);
    int64_t live = 0;
    for (const auto &kv : g_blk_live)
        if (kv.second.dev == device) live += (int64_t)kv.second.bytes;
    *live_bytes = live;
    auto it = g_blk_idle_bytes.find(device);
    *idle_bytes = it == g_blk_idle_bytes.end() ? 0 : (int64_t)it->second;
    return AWP_OK;
}

static awp_status dalloc(awp_solver *s, void **ptr, size_t bytes)
{
    if (s->fail_alloc > 0 && ++s->nalloc == s->fail_alloc) {
        *ptr = NULL;
        return set_err(AWP_ERR_OOM, "device allocation %d of %zu bytes failed (injected by AWP_TEST_FAIL_ALLOC)",
                       s->fail_alloc, bytes);
    }
    cudaError_t e = blk_alloc(s->p.device, ptr, bytes);
    if (e != cudaSuccess) {
        *ptr = NULL;
        return set_err(AWP_ERR_OOM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    s->device_bytes += (double)bytes;
    return AWP_OK;
}

/* field arrays with staggered base addresses (AWP_TUNE_STAGGER bytes times the
 * array's ordinal, modulo 32 ordinals), so that the same cell of different
 * arrays does not always fall on the same DRAM channel */
static awp_status dalloc_field(awp_solver *s, void **ptr, size_t bytes)
{
    const size_t off = s->stagger * (size_t)(s->nstag % 32);
    void *raw = NULL;
    awp_status st = dalloc(s, &raw, bytes + off);
    if (st != AWP_OK) return st;
    *ptr = (char *)raw + off;
    if (off && s->nstag < 128) {
        s->stag[s->nstag].user = *ptr;
        s->stag[s->nstag].raw = raw;
    }
    s->nstag++;
    return AWP_OK;
}

static void dfree_field(awp_solver *s, void *p)
{
    if (!p) return;
    for (int n = 0; n < s->nstag && n < 128; n++)
        if (s->stag[n].user == p && s->stag[n].raw) {
            dfree(s, s->stag[n].raw);
            s->stag[n].raw = NULL;
            return;
        }
    dfree(s, p);
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
    if (p->kinematic != 0 && p->kinematic != 1) return set_err(AWP_ERR_PARAM, "kinematic must be 0 or 1");
    if (p->kinematic && p->nst != 2)
        return set_err(AWP_ERR_PARAM, "a kinematic source (IFAULT=5) needs NST = 2 (two rows per subfault)");
    if (p->precision < AWP_PREC_F32 || p->precision > AWP_PREC_BFP) return set_err(AWP_ERR_PARAM, "unknown precision %d", p->precision);
    if (p->kernel < AWP_KERNEL_AUTO || p->kernel > AWP_KERNEL_STAGED_FMA)
        return set_err(AWP_ERR_PARAM, "unknown kernel %d", p->kernel);
    if ((p->kernel == AWP_KERNEL_STAGED || p->kernel == AWP_KERNEL_STAGED_FMA) && store_of(p) != AWP_STORE_F32)
        return set_err(AWP_ERR_PARAM, "the staged stepper reads FP32 media (precision f32, mixed or bfp)");
    if (p->nve == 1 && !(p->fl > 0 && p->fh > p->fl && p->fp > 0)) return set_err(AWP_ERR_PARAM, "Q band needs 0 < FL < FH and FP > 0");
    if (p->npc != 0 && p->npc != 1) return set_err(AWP_ERR_PARAM, "NPC must be 0 (Cerjan) or 1 (PML)");
    if (p->npc == 1) {
        if (p->kernel == AWP_KERNEL_FUSED)
            return set_err(AWP_ERR_PARAM, "the PML (NPC = 1) runs with the two-sweep or staged stepper, not the fused one");
        if (store_of(p) != AWP_STORE_F32) return set_err(AWP_ERR_PARAM, "the PML (NPC = 1) reads FP32 media");
        if (2 * p->nd >= p->nx || 2 * p->nd >= p->ny || p->nd >= p->nz || p->nd < 2)
            return set_err(AWP_ERR_PARAM, "PML width ND = %d does not fit the grid (2 ND < NX, NY; ND < NZ; ND >= 2)", p->nd);
    }
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

static awp_status alloc_media32(awp_solver *s)
{
    const size_t vb = (size_t)s->g.vol * sizeof(float);
    for (int m = 0; m < AM_N; m++) {
        if (s->md.m[m]) continue;
        awp_status st = dalloc_field(s, (void **)&s->md.m[m], vb);
        if (st != AWP_OK) return st;
        CU(cudaMemsetAsync(s->md.m[m], 0, vb, s->stream));
        if (s->store == AWP_STORE_F32) s->mdt.m[m] = s->md.m[m];
    }
    return AWP_OK;
}

extern "C" awp_status awp_create(const awp_params *pin, awp_solver **out)
{
    NvtxScope nvtx_("awp_create");
    *out = NULL;
    awp_status st = check_params(pin);
    if (st != AWP_OK) return st;
    CU(cudaSetDevice(pin->device));
    awp_solver *s = new (std::nothrow) awp_solver();
    if (!s) return set_err(AWP_ERR_OOM, "host allocation failed");
    memset(s, 0, sizeof *s);
    s->p = *pin;
    s->g = make_geom(pin);
    s->withhold = env_int("AWP_TEST_TMA_WITHHOLD", -1);
    {
        const int us = env_int("AWP_TEST_WAIT_US", 0);
        s->wait_ns = us > 0 ? (unsigned long long)us * 1000ull : 2000000000ull;
    }
    s->fail_alloc = env_int("AWP_TEST_FAIL_ALLOC", 0);
    s->fused = fused_of(pin);
    s->store = store_of(pin);
    s->rstore = rstore_of(pin);
    {
        const int sg = env_int("AWP_TUNE_STAGGER", 0);
        s->stagger = sg > 0 ? ((size_t)sg + 255) / 256 * 256 : 0;
    }
    const awp_params *p = &s->p;
    const size_t vb = (size_t)s->g.vol * sizeof(float);
    const size_t rb = (size_t)s->g.vol * (s->rstore == AWP_STORE_F32 ? 4 : 2);
#define TRY(x) do { awp_status t_ = (x); if (t_ != AWP_OK) { free_all(s); delete s; return t_; } } while (0)
#define TRYCU(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { free_all(s); delete s; \
    return set_err(AWP_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); } } while (0)
    TRYCU(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    TRYCU(cudaEventCreate(&s->ev0));
    TRYCU(cudaEventCreate(&s->ev1));
    for (int q = 0; q < p->ncomp; q++) {
        for (int f = 0; f < AWP_NF_ARRAYS; f++) {
            if (f >= AF_R1) {
                if (p->nve == 0 || (f == AF_RX && s->rstore != AWP_STORE_BFP)) continue;
                TRY(dalloc_field(s, (void **)&s->comp[0][q].f[f], rb));
                TRYCU(cudaMemsetAsync(s->comp[0][q].f[f], 0, rb, s->stream));
                s->comp[1][q].f[f] = s->comp[0][q].f[f];
                continue;
            }
            TRY(dalloc_field(s, (void **)&s->comp[0][q].f[f], vb));
            TRYCU(cudaMemsetAsync(s->comp[0][q].f[f], 0, vb, s->stream));
            if (s->fused) {
                TRY(dalloc_field(s, (void **)&s->comp[1][q].f[f], vb));
                TRYCU(cudaMemsetAsync(s->comp[1][q].f[f], 0, vb, s->stream));
            } else {
                s->comp[1][q].f[f] = s->comp[0][q].f[f];
            }
        }
    }
    s->mdt.type = s->store;
    for (int m = 0; m < AM_N; m++) { s->mdt.sc.scale[m] = 1.0f; s->mdt.sc.inv[m] = 1.0f; }
    if (s->store != AWP_STORE_F32)
        for (int m = 0; m < AM_N; m++) {
            TRY(dalloc(s, &s->mdt.m[m], (size_t)s->g.vol * 2));
            TRYCU(cudaMemsetAsync(s->mdt.m[m], 0, (size_t)s->g.vol * 2, s->stream));
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
                if (p->npc == 0 && i <= p->nd) f = f * crj_low(alpha, p->nd, i);
                if (p->npc == 0 && a < 2 && i >= n3[a] - p->nd + 1) f = f * crj_high(alpha, p->nd, n3[a], i);
                h[i] = f;   /* with the PML (NPC = 1) no sponge: every factor 1 (pmcl3d.f:928-932) */
            }
            TRY(dalloc(s, (void **)&dst[a], sizeof(float) * ((size_t)n3[a] + 2)));
            cudaError_t e = cudaMemcpy(dst[a], h, sizeof(float) * ((size_t)n3[a] + 2), cudaMemcpyHostToDevice);
            free(h);
            if (a == 0) s->cx = dst[a]; else if (a == 1) s->cy = dst[a]; else s->cz = dst[a];
            TRYCU(e);
        }
    }
    if (p->npc == 1) {
        /* split arrays of the five planes (memory.f:217-300), one buffer per
         * component: plane after plane S N W E B, each [T/H][field][cells] */
        AwpPmlArgs &pa = s->pml_args;
        const long long ns = (long long)p->nx * p->nd * p->nz, nw = (long long)p->nd * p->ny * p->nz,
                        nb = (long long)p->nx * p->ny * p->nd;
        const long long n[5] = {ns, ns, nw, nw, nb};
        long long off = 0;
        for (int a = 0; a < 5; a++) { pa.n[a] = n[a]; pa.off[a] = off; off += 18 * n[a]; }
        s->pml_floats = off;
        for (int q = 0; q < p->ncomp; q++) {
            TRY(dalloc(s, (void **)&s->pml_split[q], sizeof(float) * (size_t)off));
            TRYCU(cudaMemsetAsync(s->pml_split[q], 0, sizeof(float) * (size_t)off, s->stream));
            pa.split[q] = s->pml_split[q];
            pa.comp[q] = s->comp[0][q];
        }
        TRY(dalloc(s, (void **)&s->pml_prof, sizeof(float) * 2 * ((size_t)p->nd + 1)));
        pa.g = s->g; pa.ncomp = p->ncomp; pa.nd = p->nd;
        pa.dt = p->dt; pa.dth = p->dt / p->dh; pa.pht = p->pht;
        pa.rf = s->pml_prof; pa.rh = s->pml_prof + p->nd + 1;
        awp_pml_boxes(pa);                             /* from g and nd */
    }
    TRY(dalloc(s, (void **)&s->tau, 16 * sizeof(float)));
    TRY(dalloc(s, (void **)&s->step, sizeof(int)));
    TRYCU(cudaMemsetAsync(s->step, 0, sizeof(int), s->stream));
    TRY(dalloc(s, (void **)&s->ext, 8 * sizeof(int)));
    TRY(dalloc(s, (void **)&s->rng, 2 * AM_N * sizeof(unsigned)));
    TRY(dalloc(s, (void **)&s->en_partial, sizeof(double) * AWP_EN_GRID * AWP_MAX_COMP));
    TRY(dalloc(s, (void **)&s->en_out, sizeof(double) * AWP_MAX_COMP));
    TRY(dalloc(s, (void **)&s->flag, 2 * sizeof(int)));   /* [0] monitor, [1] AWP_KERR_* */
    TRYCU(cudaMemsetAsync(s->en_out, 0, sizeof(double) * AWP_MAX_COMP, s->stream));
    TRYCU(cudaMemsetAsync(s->flag, 0, 2 * sizeof(int), s->stream));
    s->next_check = p->monitor_every > 0 ? p->monitor_every : 0;
    for (int q = 0; q < p->ncomp; q++) {
        TRY(dalloc(s, (void **)&s->chkj[q], sizeof(float) * 3 * (size_t)p->nt));
        TRYCU(cudaMemsetAsync(s->chkj[q], 0, sizeof(float) * 3 * (size_t)p->nt, s->stream));
    }
    s->dth = p->dt / p->dh;
    s->dh1 = 1.0f / p->dh;
    s->vtst = p->dt / (p->dh * p->dh * p->dh);     /* source.f:834-835 */
    s->vtst1 = 1.0f / (p->dh * p->dh);
    s->ty = env_int("AWP_TUNE_TY", 8);
    if (s->ty != 4 && s->ty != 16) s->ty = 8;
    s->staged_on = p->kernel == AWP_KERNEL_STAGED || p->kernel == AWP_KERNEL_STAGED_FMA ||
                   (p->kernel == AWP_KERNEL_AUTO && s->store == AWP_STORE_F32);
    s->fma = p->kernel == AWP_KERNEL_STAGED_FMA;
    /* z-loop unroll: 1 or 2 (default 1 for the two-sweep kernels, 2 for the staged ones) */
    s->unroll = env_int("AWP_TUNE_UNROLL", 0);
    if (s->unroll != 1 && s->unroll != 2) s->unroll = s->staged_on ? 2 : 1;
    s->kchunk = choose_kchunk(s->g, 1, s->ty);
    s->kchunk_sweep = choose_kchunk(s->g, 0, s->ty == 4 ? 4 : 8);
    {
        /* z chunks of about 40 levels, split evenly: every chunk costs one
         * prologue level, and a short last chunk leaves blocks idle */
        int kc = env_int("AWP_TUNE_KSTAGE", 0);
        if (kc <= 0) {
            const int nch = (s->g.nz + 39) / 40;
            kc = (s->g.nz + nch - 1) / nch;
        }
        s->kchunk_staged = kc < 8 ? 8 : (kc > s->g.nz ? s->g.nz : kc);
        s->staged_qslow = env_int("AWP_TUNE_QSLOW", 1) != 0;
        /* stress sweep rows per consumer thread: two pay off once three
         * components share the sweep with FP32 memory variables */
        const int rpt = env_int("AWP_TUNE_RPT", 0);
        s->staged_rpt = rpt == 1 || rpt == 2 ? rpt : (p->ncomp == 3 && s->rstore == AWP_STORE_F32 ? 2 : 1);
        s->staged_rpt_vel = env_int("AWP_TUNE_RPTV", 1) == 2 ? 2 : 1;
        /* two or three components share one stress work item (media tiles
         * and cell coefficients once per level): 14 % faster for fx+fy on
         * 640 x 640 x 256 (14.7 GB), 3-4 % for fx+fy+fz on 400 x 400 x 200
         * (6.4 GB), but 10 % slower for fx+fy on 1400 x 1000 x 400 (78 GB),
         * where one component at a time touches half as many pages at once;
         * so by default up to 32 GiB of solver state */
        const int batch_default = (double)awp_footprint_bytes(p, 0) <= 32.0 * (double)(1ull << 30) ? 1 : 0;
        s->staged_batch = env_int("AWP_TUNE_BATCH", batch_default) & 3;
        /* the one-component sweeps read their rings with generic loads above
         * 32 GiB of state, where that measured faster (awp_staged.cu) */
        s->staged_generic = env_int("AWP_TUNE_GENERIC", batch_default ? 0 : 1) != 0;
    }
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

/* FP32 media -> the storage the steppers read.  binary16 arrays are scaled
 * by a power of two chosen from the array's largest magnitude; media whose
 * nonzero magnitudes span more than binary16's normal range are rejected. */
static awp_status convert_media(awp_solver *s)
{
    if (s->store == AWP_STORE_F32) return AWP_OK;
    if (s->store == AWP_STORE_F16) {
        unsigned init[2 * AM_N];
        for (int a = 0; a < AM_N; a++) { init[a] = 0u; init[AM_N + a] = 0x7f800000u; }
        CU(cudaMemcpyAsync(s->rng, init, sizeof init, cudaMemcpyHostToDevice, s->stream));
        CU(awp_launch_media_range(s->g, s->md, s->rng, s->rng + AM_N, s->stream));
        unsigned r[2 * AM_N];
        CU(cudaMemcpyAsync(r, s->rng, sizeof r, cudaMemcpyDeviceToHost, s->stream));
        CU(cudaStreamSynchronize(s->stream));
        for (int a = 0; a < AM_N; a++) {
            float mx, mn;
            memcpy(&mx, &r[a], 4);
            memcpy(&mn, &r[AM_N + a], 4);
            int e = 0;
            if (mx > 0) {
                frexpf(mx, &e);                         /* mx = f * 2^e, f in [0.5,1) */
                e = 14 - e;                             /* scaled max in [2^13, 2^14) */
                if (mn * ldexpf(1.0f, e) < ldexpf(1.0f, -14))
                    return set_err(AWP_ERR_PARAM, "media array %d spans %g..%g, beyond binary16 range; use BF16 or F32",
                                   a, (double)mn, (double)mx);
            }
            s->mdt.sc.scale[a] = ldexpf(1.0f, e);
            s->mdt.sc.inv[a] = ldexpf(1.0f, -e);
        }
    }
    CU(awp_launch_media_convert(s->md, s->mdt, s->g.vol, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    free_media32(s);
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
    awp_status st = convert_media(s);
    if (st != AWP_OK) return st;
    s->media_loaded = 1;
    if (s->npts > 0) {
        CU(awp_launch_sg_coeffs(s->mdt, s->npts, s->pt_idx, s->sg, s->stream));
        CU(cudaStreamSynchronize(s->stream));
    }
    return AWP_OK;
}

typedef int (*slab_reader)(void *ctx, float *dst, int zf0, int nzs, size_t floats_per_level);

/* rwg_nx > 0: the reader delivers z-slabs of RWG p/s/d volumes ([3][ny][n][nx],
 * rwg_nx x rwg_ny = ny x nx of the AWP grid), turned into AWP media order on
 * the device before the transform */
/* Two pinned staging slabs kept for the process (the read of slab n+1
 * overlaps the copy and transform of slab n); a second loader running at the
 * same time takes slabs of its own. */
namespace {
std::mutex g_stage_mu;
float *g_stage[2] = {NULL, NULL};
size_t g_stage_bytes = 0;
}

struct StageLease {
    float *h[2] = {NULL, NULL};
    bool shared = false;
    ~StageLease()
    {
        if (shared) {
            g_stage_mu.unlock();
        } else {
            if (h[0]) cudaFreeHost(h[0]);
            if (h[1]) cudaFreeHost(h[1]);
        }
    }
    cudaError_t take(size_t bytes)
    {
        if (g_stage_mu.try_lock()) {
            shared = true;
            if (g_stage_bytes < bytes) {
                for (int b = 0; b < 2; b++) {
                    if (g_stage[b]) cudaFreeHost(g_stage[b]);
                    g_stage[b] = NULL;
                }
                g_stage_bytes = 0;
                for (int b = 0; b < 2; b++) {
                    const cudaError_t e = cudaMallocHost((void **)&g_stage[b], bytes);
                    if (e != cudaSuccess) return e;
                }
                g_stage_bytes = bytes;
            }
            h[0] = g_stage[0], h[1] = g_stage[1];
            return cudaSuccess;
        }
        cudaError_t e = cudaMallocHost((void **)&h[0], bytes);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&h[1], bytes);
        return e;
    }
};

/* direct != NULL: the media are already in page-locked host memory and are
 * copied from there slab by slab, without staging */
static awp_status load_media_common(awp_solver *s, slab_reader rd, void *ctx, int rwg_nx = 0, int rwg_ny = 0,
                                    const float *direct = NULL)
{
    NvtxScope nvtx_("awp_load_media");
    const awp_params *p = &s->p;
    CU(cudaSetDevice(p->device));
    if (s->started) return set_err(AWP_ERR_STATE, "media must be loaded before the first step (or after awp_reset)");
    awp_status ast = alloc_media32(s);
    if (ast != AWP_OK) return ast;
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
    /* two pinned staging slabs: the read of slab n+1 overlaps the copy and
     * transform of slab n */
    float *hbuf[2] = {NULL, NULL}, *dbuf = NULL;
    cudaEvent_t done[2];
    StageLease lease;
    if (!direct) {
        CU(lease.take(per_level * nzs * sizeof(float)));
        hbuf[0] = lease.h[0], hbuf[1] = lease.h[1];
    }
    CU(cudaEventCreate(&done[0]));
    CU(cudaEventCreate(&done[1]));
    cudaError_t e = blk_alloc(p->device, (void **)&dbuf, per_level * nzs * sizeof(float) * (rwg_nx > 0 ? 3 : 2));
    awp_status st = AWP_OK;
    if (e != cudaSuccess) st = set_err(AWP_ERR_OOM, "media staging: %s", cudaGetErrorString(e));
    float *draw = rwg_nx > 0 && dbuf ? dbuf + 2 * per_level * nzs : NULL;
    int slab = 0;
    for (int z0 = 0; z0 < p->nz && st == AWP_OK; z0 += nzs, slab ^= 1) {
        const int n = (z0 + nzs <= p->nz) ? nzs : p->nz - z0;
        if (z0 >= 2 * nzs && cudaEventSynchronize(done[slab]) != cudaSuccess) { st = set_err(AWP_ERR_CUDA, "media stream"); break; }
        const float *src = direct ? direct + per_level * (size_t)z0 : hbuf[slab];
        if (!direct && rd(ctx, hbuf[slab], z0, n, per_level) != 0) { st = set_err(AWP_ERR_IO, "media: short read at level %d", z0); break; }
        float *d = dbuf + (size_t)slab * per_level * nzs;
        if (draw) {
            e = cudaMemcpyAsync(draw, src, per_level * n * sizeof(float), cudaMemcpyHostToDevice, s->stream);
            if (e == cudaSuccess) e = awp_launch_rwg_slab(draw, d, rwg_nx, rwg_ny, n, s->stream);
        } else {
            e = cudaMemcpyAsync(d, src, per_level * n * sizeof(float), cudaMemcpyHostToDevice, s->stream);
        }
        if (e == cudaSuccess)
            e = awp_launch_media_interior(s->g, s->md, d, z0, n, p->nvar, var_offset, p->socalq, p->nve,
                                          pi, lw, tmp1, tmp2, s->ext, s->stream);
        if (e == cudaSuccess) e = cudaEventRecord(done[slab], s->stream);
        if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "media upload: %s", cudaGetErrorString(e));
    }
    if (st == AWP_OK) {
        e = awp_launch_media_ghosts(s->g, s->md, p->nve, s->stream);
        if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "media ghosts: %s", cudaGetErrorString(e));
    }
    cudaStreamSynchronize(s->stream);
    blk_free(dbuf);
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
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
    cudaPointerAttributes attr;
    const bool pinned = media && cudaPointerGetAttributes(&attr, media) == cudaSuccess && attr.type == cudaMemoryTypeHost;
    if (media && !pinned) cudaGetLastError();
    return load_media_common(s, mem_reader, &m, 0, 0, pinned ? media : NULL);
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

/* z-slabs of RWG velocity volumes prefix.p / .s / .d: float, x fastest, then
 * z (surface first), then y; a slab of AWP levels z0..z0+n-1 is, per file and
 * per y plane, one contiguous run of n * nx values */
struct rwg_ctx { FILE *f[3]; int nx, ny, nz; };
static int rwg_reader(void *ctx, float *dst, int zf0, int nzs, size_t per_level)
{
    rwg_ctx *r = (rwg_ctx *)ctx;
    (void)per_level;
    const size_t run = (size_t)nzs * r->nx;
    for (int v = 0; v < 3; v++)
        for (int j = 0; j < r->ny; j++) {
            const long long off = ((long long)j * r->nz + zf0) * r->nx * (long long)sizeof(float);
            if (fseeko(r->f[v], (off_t)off, SEEK_SET) != 0) return -1;
            if (fread(dst + ((size_t)v * r->ny + j) * run, sizeof(float), run, r->f[v]) != run) return -1;
        }
    return 0;
}

static awp_status open_rwg(rwg_ctx *r, const char *prefix)
{
    static const char sfx[3] = {'p', 's', 'd'};
    for (int v = 0; v < 3; v++) r->f[v] = NULL;
    for (int v = 0; v < 3; v++) {
        char name[1100];
        snprintf(name, sizeof name, "%s.%c", prefix, sfx[v]);
        r->f[v] = fopen(name, "rb");
        if (!r->f[v]) {
            for (int u = 0; u < v; u++) fclose(r->f[u]);
            return set_err(AWP_ERR_IO, "cannot open velocity volume %s", name);
        }
    }
    return AWP_OK;
}

extern "C" awp_status awp_load_media_rwg(awp_solver *s, const char *prefix)
{
    if (!s || !prefix) return set_err(AWP_ERR_PARAM, "null argument");
    if (s->p.mediastart == 0) return set_err(AWP_ERR_PARAM, "MEDIARESTART 0 reads no media");
    if (s->p.nvar != 3) return set_err(AWP_ERR_PARAM, "RWG volumes carry vp, vs, rho: NVAR must be 3");
    rwg_ctx r;
    awp_status st = open_rwg(&r, prefix);
    if (st != AWP_OK) return st;
    r.nx = s->p.ny;            /* RWG x is AWP y */
    r.ny = s->p.nx;
    r.nz = s->p.nz;
    st = load_media_common(s, rwg_reader, &r, r.nx, r.ny);
    for (int v = 0; v < 3; v++) fclose(r.f[v]);
    return st;
}

extern "C" awp_status awp_reformat_velocity(int nx, int ny, int nz, const char *prefix, const char *out)
{
    if (nx < 1 || ny < 1 || nz < 1 || !prefix || !out) return set_err(AWP_ERR_PARAM, "bad argument");
    rwg_ctx r;
    awp_status st = open_rwg(&r, prefix);
    if (st != AWP_OK) return st;
    r.nx = nx; r.ny = ny; r.nz = nz;
    FILE *fo = fopen(out, "wb");
    if (!fo) {
        for (int v = 0; v < 3; v++) fclose(r.f[v]);
        return set_err(AWP_ERR_IO, "cannot create %s", out);
    }
    const size_t per_level = (size_t)3 * nx * ny;
    int nzs = (int)((256ull << 20) / (per_level * sizeof(float)));
    if (nzs < 1) nzs = 1;
    if (nzs > nz) nzs = nz;
    const size_t bytes = per_level * nzs * sizeof(float);
    float *h = NULL, *d_in = NULL, *d_out = NULL;
    cudaError_t e = cudaMallocHost((void **)&h, bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_in, bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_out, bytes);
    if (e != cudaSuccess) st = set_err(AWP_ERR_OOM, "reformat_velocity buffers: %s", cudaGetErrorString(e));
    for (int z0 = 0; z0 < nz && st == AWP_OK; z0 += nzs) {
        const int n = z0 + nzs <= nz ? nzs : nz - z0;
        const size_t sz = per_level * n * sizeof(float);
        if (rwg_reader(&r, h, z0, n, per_level) != 0) { st = set_err(AWP_ERR_IO, "velocity volumes: short read at z %d", z0); break; }
        e = cudaMemcpy(d_in, h, sz, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = awp_launch_rwg_slab(d_in, d_out, nx, ny, n, 0);
        if (e == cudaSuccess) e = cudaMemcpy(h, d_out, sz, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { st = set_err(AWP_ERR_CUDA, "reformat_velocity: %s", cudaGetErrorString(e)); break; }
        if (fwrite(h, 1, sz, fo) != sz) { st = set_err(AWP_ERR_IO, "cannot write %s", out); break; }
    }
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFreeHost(h);
    for (int v = 0; v < 3; v++) fclose(r.f[v]);
    if (fclose(fo) != 0 && st == AWP_OK) st = set_err(AWP_ERR_IO, "cannot write %s", out);
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
    for (int b = 0; b < 2; b++)
        if (s->graph[b]) { cudaGraphExecDestroy(s->graph[b]); s->graph[b] = NULL; }
    dfree(s, s->src_ijk[comp]); s->src_ijk[comp] = NULL;
    dfree(s, s->src_stf[comp]); s->src_stf[comp] = NULL;
    dfree(s, s->kin[comp]); s->kin[comp] = NULL;
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
    if (st == AWP_OK && p->kinematic) st = dalloc(s, (void **)&s->kin[comp], sizeof(float) * 6 * (size_t)nsrc);
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
    NvtxScope nvtx_("awp_set_points");
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
    for (int b = 0; b < 2; b++)
        if (s->graph[b]) { cudaGraphExecDestroy(s->graph[b]); s->graph[b] = NULL; }
    dfree(s, s->pt_idx); s->pt_idx = NULL;
    dfree(s, s->sg); s->sg = NULL;
    for (int q = 0; q < AWP_MAX_COMP; q++) { dfree(s, s->sgt_file[q]); s->sgt_file[q] = NULL; }
    s->npts = npts;
    s->sgt_file_floats = file_floats_of(p, npts);
    if (npts == 0) return AWP_OK;
    int *idx = (int *)malloc(sizeof(int) * (size_t)npts);
    for (int n = 0; n < npts; n++)   /* station.f:42-52: k = nz - z + 1 */
        idx[n] = s->g.idx(xyz[3 * n], xyz[3 * n + 1], p->nz - xyz[3 * n + 2] + 1);
    awp_status st = dalloc(s, (void **)&s->pt_idx, sizeof(int) * (size_t)npts);
    if (st == AWP_OK) st = dalloc(s, (void **)&s->sg, sizeof(float) * 3 * (size_t)npts);
    const size_t fb = sizeof(float) * (size_t)(s->sgt_file_floats > 0 ? s->sgt_file_floats : 1);
    for (int q = 0; q < p->ncomp && st == AWP_OK; q++) {
        st = dalloc(s, (void **)&s->sgt_file[q], fb);
        if (st == AWP_OK && cudaMemset(s->sgt_file[q], 0, fb) != cudaSuccess)
            st = set_err(AWP_ERR_CUDA, "memset SGT file image");
    }
    if (st == AWP_OK && cudaMemcpy(s->pt_idx, idx, sizeof(int) * (size_t)npts, cudaMemcpyHostToDevice) != cudaSuccess)
        st = set_err(AWP_ERR_CUDA, "point upload");
    free(idx);
    if (st == AWP_OK && s->media_loaded) {
        cudaError_t e = awp_launch_sg_coeffs(s->mdt, s->npts, s->pt_idx, s->sg, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "sg coefficients: %s", cudaGetErrorString(e));
    }
    return st;
}

extern "C" int64_t awp_sgt_file_floats(const awp_solver *s) { return s ? s->sgt_file_floats : 0; }

extern "C" int64_t awp_sgt_floats_for(const awp_params *p, int npts) { return p ? file_floats_of(p, npts) : 0; }

/* ------------------------------------------------------------------ */
/* time loop                                                           */
/* ------------------------------------------------------------------ */

/* buffer holding the wavefields after `steps` steps */
static int cur_buf(const awp_solver *s, int steps) { return s->fused ? (steps & 1) : 0; }

/* arguments of the step that follows `steps` completed steps */
static void fill_args(awp_solver *s, int steps, AwpStepArgs &a, AwpPostArgs &pa, AwpSgtArgs &sa)
{
    const awp_params *p = &s->p;
    const int rd = cur_buf(s, steps), wr = cur_buf(s, steps + 1);
    memset(&a, 0, sizeof a);
    a.g = s->g; a.md = s->mdt; a.ncomp = p->ncomp; a.fused = s->fused;
    for (int q = 0; q < p->ncomp; q++) { a.comp[q] = s->comp[rd][q]; a.comp_new[q] = s->comp[wr][q]; }
    a.cx = s->cx; a.cy = s->cy; a.cz = s->cz; a.tau = s->tau;
    a.dth = s->dth; a.dt = p->dt; a.dh1 = s->dh1; a.kchunk = s->kchunk; a.nve = p->nve;
    a.kchunk_sweep = s->kchunk_sweep;
    a.rtype = s->rstore;
    a.ty = s->ty;
    a.unroll = s->unroll;
    a.staged = s->staged_on ? s->staged : NULL;
    a.kchunk_staged = s->kchunk_staged;
    a.staged_qslow = s->staged_qslow;
    a.staged_rpt = s->staged_rpt;
    a.staged_rpt_vel = s->staged_rpt_vel;
    a.staged_batch = s->staged_batch;
    a.staged_generic = s->staged_generic;
    a.sm_limit = s->sm_limit;
    a.fma = s->fma;
    a.pml = s->p.npc == 1 ? &s->pml_args : NULL;
    a.kerr = s->flag + 1;
    a.wait_ns = s->wait_ns;
    a.withhold = s->withhold;

    memset(&pa, 0, sizeof pa);
    pa.g = s->g; pa.ncomp = p->ncomp; pa.nst = p->nst; pa.nt = p->nt;
    pa.vtst = s->vtst; pa.vtst1 = s->vtst1;
    const int q0 = p->nd + 2;
    pa.probe = (q0 <= p->nx && q0 <= p->ny && q0 <= p->nz) ? q0 : 0;
    pa.step = s->step;
    pa.d1 = s->mdt.m[AM_D1];
    pa.kinematic = p->kinematic;
    pa.dt = p->dt;
    pa.mu = s->mdt.m[AM_MU];
    pa.mu_inv = s->mdt.sc.inv[AM_MU];
    pa.media_type = s->mdt.type;
    pa.d1_inv = s->mdt.sc.inv[AM_D1];
    for (int q = 0; q < p->ncomp; q++) {
        pa.chkj[q] = s->chkj[q];
        pa.src[q].igreen = p->igreen[q];
        pa.src[q].nsrc = s->nsrc[q];
        pa.src[q].ijk = s->src_ijk[q];
        pa.src[q].stf = s->src_stf[q];
        pa.kin[q] = s->kin[q];
        pa.comp[q] = s->comp[wr][q];
    }

    memset(&sa, 0, sizeof sa);
    sa.g = s->g; sa.ncomp = p->ncomp; sa.npts = s->npts; sa.ntiskp = p->ntiskp_sgt;
    sa.nsamp_written = s->nsamp_written; sa.nt_file = s->nt_file;
    sa.pt_idx = s->pt_idx; sa.sg = s->sg; sa.step = s->step;
    for (int q = 0; q < p->ncomp; q++) {
        sa.file[q] = s->sgt_file[q];
        sa.comp[q] = s->comp[wr][q];
        sa.active[q] = p->igreen[q] != -1;
    }
}

/* one time step after `steps` completed steps: stepper, post, SGT gather */
static cudaError_t enqueue_one(awp_solver *s, int steps)
{
    AwpStepArgs a; AwpPostArgs pa; AwpSgtArgs sa;
    fill_args(s, steps, a, pa, sa);
    cudaError_t e = awp_launch_step(a, s->stream);
    if (e == cudaSuccess) e = awp_launch_post(pa, 0, s->stream);
    if (e == cudaSuccess && s->npts > 0 && ((steps + 1) % s->p.ntiskp_sgt == 0))
        e = awp_launch_sgt(sa, s->stream);
    return e;
}

/* CUDA graph of NTISKP_SGT steps ending with the SGT gather; kernels read the
 * device step counter, so a graph replays for every period that starts on
 * the same buffer parity. */
static cudaError_t build_graph(awp_solver *s, int par)
{
    if (s->graph[par]) return cudaSuccess;
    const int gs = s->p.ntiskp_sgt;
    cudaGraph_t graph;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    /* graphs start on a period boundary; a base of gs (odd periods only)
     * gives the steps the odd buffer parity while keeping the gather last */
    const int base = par ? gs : 0;
    cudaError_t le = cudaSuccess;
    for (int n = 0; n < gs && le == cudaSuccess; n++) le = enqueue_one(s, base + n);
    e = cudaStreamEndCapture(s->stream, &graph);
    if (le != cudaSuccess) { if (e == cudaSuccess) cudaGraphDestroy(graph); return le; }
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&s->graph[par], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { s->graph[par] = NULL; return e; }
    return cudaSuccess;
}

static awp_status start_if_needed(awp_solver *s)
{
    if (s->started) return AWP_OK;
    if (!s->media_loaded) return set_err(AWP_ERR_STATE, "media not loaded");
    if (s->staged_on && !s->staged) {
        /* the arrays are fixed from here on: u v w, the stresses, FP32 media */
        const cudaError_t e = awp_staged_create(&s->staged, s->g, s->p.ncomp, s->comp[0], s->mdt, s->rstore);
        if (e != cudaSuccess) return set_err(AWP_ERR_CUDA, "staged stepper: tensor maps: %s", cudaGetErrorString(e));
    }
    if (s->p.npc == 1) {
        /* inipml (pml.f:4-44) from the media's S velocity range (pmcl3d.f:928-929) */
        const int nd = s->p.nd;
        std::vector<float> prof(2 * ((size_t)nd + 1), 0.0f);
        awp_pml_profiles(nd, s->p.arbc, s->p.dh, s->ext_host[2], s->ext_host[3], &prof[0], &prof[nd + 1]);
        CU(cudaMemcpy(s->pml_prof, prof.data(), sizeof(float) * prof.size(), cudaMemcpyHostToDevice));
        s->pml_args.d1 = (const float *)s->mdt.m[AM_D1];
        s->pml_args.lam = (const float *)s->mdt.m[AM_LAM];
        s->pml_args.mu = (const float *)s->mdt.m[AM_MU];
    }
    AwpStepArgs a; AwpPostArgs pa; AwpSgtArgs sa;
    fill_args(s, -1, a, pa, sa);       /* addsrc(1) into the buffer step 1 reads */
    CU(awp_launch_post(pa, 1, s->stream));
    s->started = 1;
    return AWP_OK;
}

static void energy_args(awp_solver *s, AwpEnergyArgs &a)
{
    memset(&a, 0, sizeof a);
    a.g = s->g;
    a.ncomp = s->p.ncomp;
    const int b = cur_buf(s, s->steps_done);
    for (int q = 0; q < s->p.ncomp; q++)
        for (int f = 0; f < 3; f++) a.f[3 * q + f] = s->comp[b][q].f[AF_U + f];
}

/* stability monitor after the steps enqueued so far, when a check is due */
static cudaError_t maybe_monitor(awp_solver *s)
{
    if (s->p.monitor_every <= 0 || s->steps_done < s->next_check) return cudaSuccess;
    while (s->next_check <= s->steps_done) s->next_check += s->p.monitor_every;
    AwpEnergyArgs a;
    energy_args(s, a);
    return awp_launch_energy(a, s->en_partial, AWP_EN_GRID, s->en_out, s->flag, s->stream);
}

extern "C" awp_status awp_run_async(awp_solver *s, int nsteps)
{
    NvtxScope nvtx_("awp_run_async");
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    const awp_params *p = &s->p;
    CU(cudaSetDevice(p->device));
    awp_status st = start_if_needed(s);
    if (st != AWP_OK) return st;
    if (nsteps < 0) return set_err(AWP_ERR_PARAM, "nsteps < 0");
    int todo = nsteps;
    if (todo > p->nt - s->steps_done) todo = p->nt - s->steps_done;
    if (todo <= 0) return AWP_OK;
    if (!s->pending) CU(cudaEventRecord(s->ev0, s->stream));
    int left = todo;
    const int gs = p->ntiskp_sgt;
    int head = (gs - (s->steps_done % gs)) % gs;
    if (head > left) head = left;
    for (; head > 0; head--, left--) { CU(enqueue_one(s, s->steps_done++)); CU(maybe_monitor(s)); }
    if (left >= gs && gs <= 64) {
        while (left >= gs) {
            const int par = cur_buf(s, s->steps_done);
            CU(build_graph(s, par));
            CU(cudaGraphLaunch(s->graph[par], s->stream));
            s->steps_done += gs;
            left -= gs;
            CU(maybe_monitor(s));
        }
    }
    for (; left > 0; left--) { CU(enqueue_one(s, s->steps_done++)); CU(maybe_monitor(s)); }
    CU(cudaEventRecord(s->ev1, s->stream));
    s->pending = 1;
    s->pending_steps += todo;
    return AWP_OK;
}

extern "C" int awp_query(awp_solver *s)
{
    if (!s) return -1;
    if (!s->pending) return 1;
    cudaError_t e = cudaEventQuery(s->ev1);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    set_err(AWP_ERR_CUDA, "awp_query: %s", cudaGetErrorString(e));
    return -1;
}

extern "C" awp_status awp_sync(awp_solver *s)
{
    NvtxScope nvtx_("awp_sync");
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    CU(cudaSetDevice(s->p.device));
    if (s->pending) {
        CU(cudaEventSynchronize(s->ev1));
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
        s->loop_seconds += ms * 1e-3;
        s->loop_steps += s->pending_steps;
        s->pending = 0;
        s->pending_steps = 0;
    }
    if (s->p.monitor_every > 0 || s->staged_on) {
        int flag[2] = {0, 0};
        CU(cudaMemcpyAsync(flag, s->flag, sizeof flag, cudaMemcpyDeviceToHost, s->stream));
        CU(cudaStreamSynchronize(s->stream));
        if (flag[1]) return set_err(AWP_ERR_TIMEOUT, "staged stepper: a tile barrier wait ran out after %.3f s "
                                    "(error word %d); the solve's state is not valid", s->wait_ns * 1e-9, flag[1]);
        if (flag[0]) return set_err(AWP_ERR_UNSTABLE, "stability monitor: non-finite wavefield energy by step %d",
                                    s->steps_done);
    }
    return AWP_OK;
}

extern "C" awp_status awp_run(awp_solver *s, int nsteps, float *sgt_out)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    const awp_params *p = &s->p;
    awp_status st = awp_run_async(s, nsteps);
    if (st != AWP_OK) return st;
    st = awp_sync(s);
    if (st != AWP_OK) return st;
    if (sgt_out) {
        for (int q = 0; q < p->ncomp; q++) {
            st = awp_get_sgt(s, q, sgt_out + (size_t)q * (size_t)s->sgt_file_floats);
            if (st != AWP_OK) return st;
        }
    }
    return AWP_OK;
}

/* algorithmic bytes of one launch of each step kernel (compulsory traffic:
 * every array element the kernel reads or writes counted once) */
static double part_bytes(const awp_solver *s, int part)
{
    const awp_params *p = &s->p;
    const double cells = (double)p->nx * p->ny * p->nz;
    const double nc = p->ncomp;
    const double mb = media_word(s->store);
    const double rcell = p->nve == 1 ? 2.0 * awp_r_bytes(s->rstore) : 0.0;   /* r1..r6 read+write */
    const int nmed = p->nve == 1 ? 5 : 3;
    switch (part) {
    case AWP_PART_VEL: return cells * (nc * 12 * 4.0 + mb);                          /* R 9 W 3 + d1 */
    case AWP_PART_FSVEL: return (double)p->nx * p->ny * (nc * (8 * 4.0) + 2 * mb);
    case AWP_PART_STR: return cells * (nc * (15 * 4.0 + rcell) + (nmed - 1) * mb);
    case AWP_PART_FUSED: return cells * (nc * (18 * 4.0 + rcell) + nmed * mb);
    case AWP_PART_PML_VEL:
    case AWP_PART_PML_STR: {
        /* per boundary cell: the stresses (velocities) read, two splits of
         * each updated field read and written, the updated fields written,
         * the cell's media */
        const double nb = cells - (double)(p->nx - 2 * p->nd) * (p->ny - 2 * p->nd) * (p->nz - p->nd);
        return part == AWP_PART_PML_VEL ? nb * (nc * (6 + 12 + 3) * 4.0 + 4.0)
                                        : nb * (nc * (3 + 24 + 6) * 4.0 + 8.0);
    }
    }
    return 0.0;
}

extern "C" awp_status awp_profile_steps(awp_solver *s, int nsteps, awp_kernel_times *o)
{
    if (!s || !o) return set_err(AWP_ERR_PARAM, "null argument");
    const awp_params *p = &s->p;
    CU(cudaSetDevice(p->device));
    memset(o, 0, sizeof *o);
    awp_status st = start_if_needed(s);
    if (st != AWP_OK) return st;
    int todo = nsteps;
    if (todo > p->nt - s->steps_done) todo = p->nt - s->steps_done;
    /* kernel classes: the stepper kernels, then k_post, then k_sgt */
    int parts[6], np = 0;
    if (s->fused) parts[np++] = AWP_PART_FUSED;
    else {
        parts[np++] = AWP_PART_VEL;
        if (p->npc == 1) parts[np++] = AWP_PART_PML_VEL;
        parts[np++] = AWP_PART_FSVEL;
        parts[np++] = AWP_PART_STR;
        if (p->npc == 1) parts[np++] = AWP_PART_PML_STR;
    }
    static const char *pname[] = {"k_vel", "k_fsvel", "k_str", "k_fused", "k_pml_vel", "k_pml_str"};
    static const char *pname_staged[] = {"k_vel_tma", "k_fsvel", "k_str_tma", "k_fused", "k_pml_vel", "k_pml_str"};
    const int nk = np + 2;
    o->nkernels = nk;
    for (int k = 0; k < np; k++) {
        const bool bstr = s->staged_on && parts[k] == AWP_PART_STR && (s->staged_batch & 1) && p->ncomp >= 2;
        const bool bvel = s->staged_on && parts[k] == AWP_PART_VEL && (s->staged_batch & 2) && p->ncomp >= 2;
        snprintf(o->name[k], sizeof o->name[k], "%s",
                 bstr ? "k_str_tmab" : (bvel ? "k_vel_tmab" : (s->staged_on ? pname_staged : pname)[parts[k]]));
        o->bytes_per_launch[k] = part_bytes(s, parts[k]);
    }
    snprintf(o->name[np], sizeof o->name[np], "k_post");
    snprintf(o->name[np + 1], sizeof o->name[np + 1], "k_sgt");
    cudaEvent_t ev[16];
    for (int k = 0; k < 16; k++) CU(cudaEventCreate(&ev[k]));
    double tot[8] = {0};
    awp_status rs = AWP_OK;
    for (int n = 0; n < todo && rs == AWP_OK; n++) {
        AwpStepArgs a; AwpPostArgs pa; AwpSgtArgs sa;
        fill_args(s, s->steps_done, a, pa, sa);
        for (int k = 0; k < nk; k++) {
            const bool sgt_now = s->npts > 0 && ((s->steps_done + 1) % p->ntiskp_sgt == 0);
            if (k == np + 1 && !sgt_now) continue;
            cudaError_t e = cudaEventRecord(ev[2 * k], s->stream);
            if (e == cudaSuccess) {
                if (k < np && parts[k] == AWP_PART_PML_VEL) e = awp_launch_pml(*a.pml, 0, s->stream);
                else if (k < np && parts[k] == AWP_PART_PML_STR) e = awp_launch_pml(*a.pml, 1, s->stream);
                else if (k < np) e = awp_launch_part(a, parts[k], s->stream);
                else if (k == np) e = awp_launch_post(pa, 0, s->stream);
                else e = awp_launch_sgt(sa, s->stream);
            }
            if (e == cudaSuccess) e = cudaEventRecord(ev[2 * k + 1], s->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(ev[2 * k + 1]);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]);
            if (e != cudaSuccess) { rs = set_err(AWP_ERR_CUDA, "profile: %s", cudaGetErrorString(e)); break; }
            tot[k] += ms;
            o->launches[k]++;
        }
        s->steps_done++;
    }
    for (int k = 0; k < 16; k++) cudaEventDestroy(ev[k]);
    for (int k = 0; k < nk; k++) o->ms_per_launch[k] = o->launches[k] ? tot[k] / o->launches[k] : 0.0;
    return rs;
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

extern "C" awp_status awp_get_sgt_rwg(awp_solver *s, int comp, int z_source, float *out)
{
    if (!s || !out || comp < 0 || comp >= s->p.ncomp) return set_err(AWP_ERR_PARAM, "bad solver/component/output");
    if (s->sgt_file_floats <= 0) return AWP_OK;
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    float *tmp = NULL;
    CU(cudaMalloc((void **)&tmp, sizeof(float) * (size_t)s->sgt_file_floats));
    cudaError_t e = awp_launch_sgt_rwg(s->sgt_file[comp], tmp, s->npts, s->nt_file, z_source != 0, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, tmp, sizeof(float) * (size_t)s->sgt_file_floats, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return set_err(AWP_ERR_CUDA, "awp_get_sgt_rwg: %s", cudaGetErrorString(e));
    return AWP_OK;
}

extern "C" awp_status awp_sgt_reorder_rwg(const float *in, int64_t npts, int nt, int z_source, float *out)
{
    if (!in || !out || npts < 0 || nt < 0) return set_err(AWP_ERR_PARAM, "awp_sgt_reorder_rwg: bad argument");
    const size_t bytes = sizeof(float) * 6 * (size_t)npts * (size_t)nt;
    if (bytes == 0) return AWP_OK;
    float *d_in = NULL, *d_out = NULL;
    cudaError_t e = cudaMalloc((void **)&d_in, bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_out, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(d_in, in, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = awp_launch_sgt_rwg(d_in, d_out, npts, nt, z_source != 0, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    if (e != cudaSuccess) return set_err(AWP_ERR_CUDA, "awp_sgt_reorder_rwg: %s", cudaGetErrorString(e));
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

/* 16-bit block floating point of r1..r6 on the host (the rule of
 * awp_internal.h, as the device kernels apply it) */
static float f_of_bits(uint32_t b) { float v; memcpy(&v, &b, 4); return v; }
static uint32_t bits_of_f(float v) { uint32_t b; memcpy(&b, &v, 4); return b; }

static float bfp_down(uint32_t e) { return f_of_bits(((e < AWP_BFP_EMIN ? AWP_BFP_EMIN : e) - 14u) << 23); }

static uint32_t bfp_enc3_host(const float v[3], int16_t m[3])
{
    const float mx = fmaxf(fabsf(v[0]), fmaxf(fabsf(v[1]), fabsf(v[2])));
    const uint32_t e = bits_of_f(mx) >> 23;
    if (e < AWP_BFP_EMIN) {
        m[0] = m[1] = m[2] = 0;
        return 0u;
    }
    const float up = f_of_bits((268u - e) << 23);
    for (int a = 0; a < 3; a++) m[a] = (int16_t)lrintf(fminf(fmaxf(v[a] * up, -32767.f), 32767.f));
    return e;
}

/* the three mantissa arrays of r group g (0: r1..r3, 1: r4..r6) and the
 * exponent words of component q, in the padded host layout */
static awp_status bfp_fetch(awp_solver *s, int q, int grp, int16_t *m[3], uint16_t *x)
{
    const AwpGeom &g = s->g;
    const size_t w = (size_t)(g.nx + 4), rows = (size_t)(g.ny + 4) * (size_t)(g.nz + 4);
    const AwpComp &c = s->comp[0][q];
    for (int a = 0; a < 3; a++)
        CU(cudaMemcpy2D(m[a], w * 2, (const int16_t *)c.f[AF_R1 + 3 * grp + a] + (AWP_XO - 2), (size_t)g.px * 2,
                        w * 2, rows, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy2D(x, w * 2, (const uint16_t *)c.f[AF_RX] + (AWP_XO - 2), (size_t)g.px * 2, w * 2, rows,
                    cudaMemcpyDeviceToHost));
    return AWP_OK;
}

static awp_status bfp_get(awp_solver *s, int q, int field, float *out)
{
    const AwpGeom &g = s->g;
    const size_t n = (size_t)(g.nx + 4) * (g.ny + 4) * (g.nz + 4);
    const int a = field - AF_R1, grp = a / 3;
    std::vector<int16_t> mm(3 * n);
    std::vector<uint16_t> xx(n);
    int16_t *m[3] = {&mm[0], &mm[n], &mm[2 * n]};
    awp_status st = bfp_fetch(s, q, grp, m, xx.data());
    if (st != AWP_OK) return st;
    for (size_t c = 0; c < n; c++) {
        const uint32_t e = grp ? (uint32_t)(xx[c] >> 8) : (uint32_t)(xx[c] & 0xffu);
        out[c] = (float)m[a % 3][c] * bfp_down(e);
    }
    return AWP_OK;
}

/* stores one group of memory variables (grp 0: r1..r3, 1: r4..r6) of
 * component q: v[b] is the new value of member b, or NULL to keep the group's
 * current (decoded) value; the group is encoded once from the three values
 * (the other group's exponent byte is kept).  Setting all three members at
 * once restores decoded values exactly; setting them one at a time need not,
 * since each encode flushes to zero what lies below its exponent's range. */
static awp_status bfp_set_group(awp_solver *s, int q, int grp, const float *const v[3])
{
    const AwpGeom &g = s->g;
    const size_t w = (size_t)(g.nx + 4), rows = (size_t)(g.ny + 4) * (size_t)(g.nz + 4), n = w * rows;
    std::vector<int16_t> mm(3 * n);
    std::vector<uint16_t> xx(n);
    int16_t *m[3] = {&mm[0], &mm[n], &mm[2 * n]};
    awp_status st = bfp_fetch(s, q, grp, m, xx.data());
    if (st != AWP_OK) return st;
    for (size_t c = 0; c < n; c++) {
        const uint32_t e = grp ? (uint32_t)(xx[c] >> 8) : (uint32_t)(xx[c] & 0xffu);
        const float down = bfp_down(e);
        float val[3];
        for (int b = 0; b < 3; b++) val[b] = v[b] ? v[b][c] : (float)m[b][c] * down;
        int16_t nm[3];
        const uint32_t ne = bfp_enc3_host(val, nm);
        for (int b = 0; b < 3; b++) m[b][c] = nm[b];
        xx[c] = grp ? (uint16_t)((xx[c] & 0x00ffu) | (ne << 8)) : (uint16_t)((xx[c] & 0xff00u) | ne);
    }
    const AwpComp &cp = s->comp[0][q];
    for (int b = 0; b < 3; b++)
        CU(cudaMemcpy2D((int16_t *)cp.f[AF_R1 + 3 * grp + b] + (AWP_XO - 2), (size_t)g.px * 2, m[b], w * 2, w * 2,
                        rows, cudaMemcpyHostToDevice));
    CU(cudaMemcpy2D((uint16_t *)cp.f[AF_RX] + (AWP_XO - 2), (size_t)g.px * 2, xx.data(), w * 2, w * 2, rows,
                    cudaMemcpyHostToDevice));
    return AWP_OK;
}

static awp_status bfp_set(awp_solver *s, int q, int field, const float *in)
{
    const int a = field - AF_R1;
    const float *v[3] = {NULL, NULL, NULL};
    v[a % 3] = in;
    return bfp_set_group(s, q, a / 3, v);
}

extern "C" awp_status awp_get_plane(awp_solver *s, int comp, int field, int k, float *out)
{
    if (!s || !out) return set_err(AWP_ERR_PARAM, "null argument");
    if (comp < 0 || comp >= s->p.ncomp) return set_err(AWP_ERR_PARAM, "bad component");
    if (field < 0 || field >= AF_R1) return set_err(AWP_ERR_PARAM, "field %d is not a wavefield or stress", field);
    const AwpGeom &g = s->g;
    if (k < 1 || k > g.nz) return set_err(AWP_ERR_PARAM, "level %d outside 1..%d", k, g.nz);
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    const float *src = s->comp[cur_buf(s, s->steps_done)][comp].f[field];
    CU(cudaMemcpy2D(out, (size_t)g.nx * sizeof(float), src + g.idx(1, 1, k), (size_t)g.px * sizeof(float),
                    (size_t)g.nx * sizeof(float), (size_t)g.ny, cudaMemcpyDeviceToHost));
    return AWP_OK;
}

extern "C" awp_status awp_get_field(awp_solver *s, int comp, int field, float *out)
{
    if (!s) return set_err(AWP_ERR_PARAM, "null solver");
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    const AwpGeom &g = s->g;
    const size_t w = (size_t)(g.nx + 4), rows = (size_t)(g.ny + 4) * (size_t)(g.nz + 4);
    const void *src = NULL;
    int type = AWP_STORE_F32;
    float inv = 1.0f;
    if (field >= 0 && field < AWP_NF_STATE) {
        if (comp < 0 || comp >= s->p.ncomp) return set_err(AWP_ERR_PARAM, "bad component");
        src = s->comp[cur_buf(s, s->steps_done)][comp].f[field];
        if (field >= AF_R1) type = s->rstore;
        if (src && type == AWP_STORE_BFP) return bfp_get(s, comp, field, out);
    } else if (field >= AWP_NF_STATE && field < AWP_NF_STATE + AM_N) {
        src = s->mdt.m[field - AWP_NF_STATE];
        type = s->mdt.type;
        inv = s->mdt.sc.inv[field - AWP_NF_STATE];
    }
    if (!src) return set_err(AWP_ERR_PARAM, "field %d not held by this solver", field);
    if (type == AWP_STORE_F32) {
        CU(cudaMemcpy2D(out, w * sizeof(float), (const float *)src + (AWP_XO - 2), (size_t)g.px * sizeof(float),
                        w * sizeof(float), rows, cudaMemcpyDeviceToHost));
        return AWP_OK;
    }
    /* 16-bit storage: copy and widen on the host */
    unsigned short *tmp = (unsigned short *)malloc(w * rows * 2);
    if (!tmp) return set_err(AWP_ERR_OOM, "host buffer");
    cudaError_t e = cudaMemcpy2D(tmp, w * 2, (const unsigned short *)src + (AWP_XO - 2), (size_t)g.px * 2, w * 2, rows,
                                 cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { free(tmp); return set_err(AWP_ERR_CUDA, "get_field: %s", cudaGetErrorString(e)); }
    for (size_t n = 0; n < w * rows; n++) {
        uint32_t b = tmp[n];
        float v;
        if (type == AWP_STORE_BF16) {
            b <<= 16;
            memcpy(&v, &b, 4);
        } else {   /* IEEE binary16 -> float */
            uint32_t sgn = (b & 0x8000u) << 16, ex = (b >> 10) & 0x1f, man = b & 0x3ff;
            if (ex == 0) v = ldexpf((float)man, -24);
            else if (ex == 31) { uint32_t f = sgn | 0x7f800000u | (man << 13); memcpy(&v, &f, 4); out[n] = v; continue; }
            else v = ldexpf((float)(man | 0x400), (int)ex - 25);
            if (sgn) v = -v;
            v *= inv;
        }
        out[n] = v;
    }
    free(tmp);
    return AWP_OK;
}

/* float32 -> bfloat16, round to nearest even (the device's __float2bfloat16_rn;
 * NaN stays a quiet NaN) */
static uint16_t bf16_rn(float v)
{
    uint32_t b;
    memcpy(&b, &v, 4);
    if ((b & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((b >> 16) | 0x40);
    b += 0x7fffu + ((b >> 16) & 1u);
    return (uint16_t)(b >> 16);
}

extern "C" awp_status awp_set_field(awp_solver *s, int comp, int field, const float *in)
{
    if (!s || !in) return set_err(AWP_ERR_PARAM, "null argument");
    if (field < 0 || field >= AWP_NF_STATE)
        return set_err(AWP_ERR_PARAM, "awp_set_field: field %d is not a state field (0..%d)", field, AWP_NF_STATE - 1);
    if (comp < 0 || comp >= s->p.ncomp) return set_err(AWP_ERR_PARAM, "bad component");
    if (!s->comp[0][comp].f[field]) return set_err(AWP_ERR_PARAM, "field %d not held by this solver", field);
    if (s->pending) {
        awp_status st = awp_sync(s);
        if (st != AWP_OK) return st;
    }
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    const AwpGeom &g = s->g;
    const size_t w = (size_t)(g.nx + 4), rows = (size_t)(g.ny + 4) * (size_t)(g.nz + 4);
    const int type = field >= AF_R1 ? s->rstore : AWP_STORE_F32;
    if (type == AWP_STORE_BFP) return bfp_set(s, comp, field, in);
    uint16_t *tmp = NULL;
    if (type != AWP_STORE_F32) {
        tmp = (uint16_t *)malloc(w * rows * 2);
        if (!tmp) return set_err(AWP_ERR_OOM, "host buffer");
        for (size_t n = 0; n < w * rows; n++) tmp[n] = bf16_rn(in[n]);
    }
    /* both wavefield buffers of the fused stepper get the values, so the next
     * step reads them whatever its buffer parity */
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; b++) {
        void *dst = s->comp[b][comp].f[field];
        if (!dst || (b == 1 && dst == s->comp[0][comp].f[field])) continue;
        if (type == AWP_STORE_F32)
            e = cudaMemcpy2D((float *)dst + (AWP_XO - 2), (size_t)g.px * sizeof(float), in, w * sizeof(float),
                             w * sizeof(float), rows, cudaMemcpyHostToDevice);
        else
            e = cudaMemcpy2D((uint16_t *)dst + (AWP_XO - 2), (size_t)g.px * 2, tmp, w * 2, w * 2, rows,
                             cudaMemcpyHostToDevice);
    }
    free(tmp);
    if (e != cudaSuccess) return set_err(AWP_ERR_CUDA, "awp_set_field: %s", cudaGetErrorString(e));
    return AWP_OK;
}

/* ------------------------------------------------------------------ */
/* checkpoint / restart (pmcl3d.f:1018-1097 read, 1967-2045 write)     */
/* ------------------------------------------------------------------ */

#define AWP_CKP_MAGIC "AWPSGTCK"
#define AWP_CKP_VERSION 1

/* header of the ckpsgt file: what the reference's checkpoint does not hold
 * (it writes SGT chunks as it goes), so that a resumed solve ends with the
 * same SGT file image and CHKJ series as an uninterrupted one */
struct CkpSgtHeader {
    char magic[8];
    int32_t version, step, nt, npts;
    int64_t nt_file, sgt_floats;
};

static awp_status write_all(FILE *f, const void *p, size_t bytes, const char *path)
{
    if (bytes && fwrite(p, 1, bytes, f) != bytes) return set_err(AWP_ERR_IO, "cannot write %s", path);
    return AWP_OK;
}

static awp_status read_all(FILE *f, void *p, size_t bytes, const char *path)
{
    if (bytes && fread(p, 1, bytes, f) != bytes) return set_err(AWP_ERR_IO, "%s is short", path);
    return AWP_OK;
}

/* The PML split arrays of one component in the reference's checkpoint files
 * (pmcl3d.f:1995-2040): ckpew = the east plane then the west, ckpns = north
 * then south, ckpb = bottom; per plane three records of six arrays, fields u
 * v w | xx yy zz | xz yz xy, each as its T then its H split, in the plane's
 * own addressing (the device layout is the same per array). */
static awp_status pml_ckp_io(awp_solver *s, int q, const char *dir, int step, bool write)
{
    static const char *name[3] = {"ckpew", "ckpns", "ckpb"};
    static const int planes[3][2] = {{3, 2}, {1, 0}, {4, -1}};        /* E W | N S | B */
    static const int fields[9] = {0, 1, 2, 3, 4, 5, 7, 8, 6};        /* u v w xx yy zz xz yz xy */
    const AwpPmlArgs &pa = s->pml_args;
    char path[1200];
    awp_status st = AWP_OK;
    for (int fl = 0; fl < 3 && st == AWP_OK; fl++) {
        snprintf(path, sizeof path, "%s/%s%07d%07d.bin", dir, name[fl], q, step);
        FILE *f = fopen(path, write ? "wb" : "rb");
        if (!f) return set_err(AWP_ERR_IO, write ? "cannot create %s" : "checkpoint %s missing", path);
        for (int pp = 0; pp < 2 && st == AWP_OK; pp++) {
            const int pl = planes[fl][pp];
            if (pl < 0) continue;
            std::vector<float> buf((size_t)pa.n[pl]);
            for (int fd = 0; fd < 9 && st == AWP_OK; fd++)
                for (int sp = 0; sp < 2 && st == AWP_OK; sp++) {
                    float *dev = s->pml_split[q] + pa.off[pl] + (sp * 9 + fields[fd]) * pa.n[pl];
                    const size_t bytes = sizeof(float) * buf.size();
                    if (write) {
                        CU(cudaMemcpy(buf.data(), dev, bytes, cudaMemcpyDeviceToHost));
                        st = write_all(f, buf.data(), bytes, path);
                    } else {
                        st = read_all(f, buf.data(), bytes, path);
                        if (st == AWP_OK) CU(cudaMemcpy(dev, buf.data(), bytes, cudaMemcpyHostToDevice));
                    }
                }
        }
        if (fclose(f) != 0 && write && st == AWP_OK) st = set_err(AWP_ERR_IO, "cannot write %s", path);
    }
    return st;
}

extern "C" awp_status awp_checkpoint_write(awp_solver *s, const char *dir)
{
    NvtxScope nvtx_("awp_checkpoint_write");
    if (!s || !dir) return set_err(AWP_ERR_PARAM, "null argument");
    awp_status st = awp_sync(s);
    if (st != AWP_OK) return st;
    const awp_params *p = &s->p;
    const size_t nvol = (size_t)(p->nx + 4) * (p->ny + 4) * (p->nz + 4);
    float *buf = (float *)malloc(nvol * sizeof(float));
    float *aux = (float *)malloc(sizeof(float) * ((size_t)3 * p->nt + (size_t)s->sgt_file_floats + 1));
    if (!buf || !aux) { free(buf); free(aux); return set_err(AWP_ERR_OOM, "host buffer"); }
    char path[1200], tmpp[1300];
    const int step = s->steps_done;
    for (int q = 0; q < p->ncomp && st == AWP_OK; q++) {
        /* ckp<rank><step>.bin: five records [u1 v1 w1] [xx yy zz] [xy xz yz] [r1 r2 r3] [r4 r5 r6],
         * each array (nx+4)(ny+4)(nz+4) float32 with its ghost cells, x fastest */
        snprintf(path, sizeof path, "%s/ckp%07d%07d.bin", dir, q, step);
        FILE *f = fopen(path, "wb");
        if (!f) { st = set_err(AWP_ERR_IO, "cannot create %s", path); break; }
        for (int fld = 0; fld < AWP_NF_STATE && st == AWP_OK; fld++) {
            if (s->comp[0][q].f[fld]) st = awp_get_field(s, q, fld, buf);
            else memset(buf, 0, nvol * sizeof(float));      /* elastic scheme: no memory variables */
            if (st == AWP_OK) st = write_all(f, buf, nvol * sizeof(float), path);
        }
        if (fclose(f) != 0 && st == AWP_OK) st = set_err(AWP_ERR_IO, "cannot write %s", path);
        if (st != AWP_OK) break;
        /* ckpdy<rank><step>.bin: u2, broken (dynamic-rupture arrays, zero here), mu */
        snprintf(path, sizeof path, "%s/ckpdy%07d%07d.bin", dir, q, step);
        f = fopen(path, "wb");
        if (!f) { st = set_err(AWP_ERR_IO, "cannot create %s", path); break; }
        memset(buf, 0, nvol * sizeof(float));
        st = write_all(f, buf, nvol * sizeof(float), path);
        if (st == AWP_OK) st = write_all(f, buf, nvol * sizeof(float), path);
        if (st == AWP_OK) st = awp_get_field(s, q, AWP_NF_STATE + AM_MU, buf);
        if (st == AWP_OK) st = write_all(f, buf, nvol * sizeof(float), path);
        if (fclose(f) != 0 && st == AWP_OK) st = set_err(AWP_ERR_IO, "cannot write %s", path);
        if (st != AWP_OK) break;
        if (p->npc == 1 && (st = pml_ckp_io(s, q, dir, step, true)) != AWP_OK) break;
        /* ckpsgt<rank><step>.bin: the SGT file image and CHKJ series so far */
        snprintf(path, sizeof path, "%s/ckpsgt%07d%07d.bin", dir, q, step);
        f = fopen(path, "wb");
        if (!f) { st = set_err(AWP_ERR_IO, "cannot create %s", path); break; }
        CkpSgtHeader h;
        memset(&h, 0, sizeof h);
        memcpy(h.magic, AWP_CKP_MAGIC, 8);
        h.version = AWP_CKP_VERSION; h.step = step; h.nt = p->nt; h.npts = s->npts;
        h.nt_file = s->nt_file; h.sgt_floats = s->sgt_file_floats;
        st = write_all(f, &h, sizeof h, path);
        if (st == AWP_OK) st = awp_get_chkj(s, q, aux);
        if (st == AWP_OK && s->sgt_file_floats > 0) st = awp_get_sgt(s, q, aux + (size_t)3 * p->nt);
        if (st == AWP_OK)
            st = write_all(f, aux, sizeof(float) * ((size_t)3 * p->nt + (size_t)s->sgt_file_floats), path);
        if (fclose(f) != 0 && st == AWP_OK) st = set_err(AWP_ERR_IO, "cannot write %s", path);
        if (st != AWP_OK) break;
        /* ckp<rank>.hdr names the step last, once the data files are complete
         * (written to a temporary name and renamed into place) */
        snprintf(path, sizeof path, "%s/ckp%07d.hdr", dir, q);
        snprintf(tmpp, sizeof tmpp, "%s.tmp", path);
        f = fopen(tmpp, "w");
        if (!f) { st = set_err(AWP_ERR_IO, "cannot create %s", tmpp); break; }
        fprintf(f, "%12d\n", step);
        if (fclose(f) != 0 || rename(tmpp, path) != 0) st = set_err(AWP_ERR_IO, "cannot write %s", path);
    }
    free(buf);
    free(aux);
    return st;
}

extern "C" awp_status awp_checkpoint_read(awp_solver *s, const char *dir, int *step_out)
{
    NvtxScope nvtx_("awp_checkpoint_read");
    if (!s || !dir) return set_err(AWP_ERR_PARAM, "null argument");
    if (step_out) *step_out = 0;
    const awp_params *p = &s->p;
    /* the step to resume from: the smallest over the components' headers; a
     * missing header counts as 0 (pmcl3d.f:1019-1036, MPI_MIN over ranks) */
    char path[1200];
    int t0 = INT32_MAX;
    for (int q = 0; q < p->ncomp; q++) {
        snprintf(path, sizeof path, "%s/ckp%07d.hdr", dir, q);
        FILE *f = fopen(path, "r");
        int t = 0;
        if (f) {
            if (fscanf(f, "%d", &t) != 1) t = 0;
            fclose(f);
        }
        if (t < t0) t0 = t;
    }
    if (t0 <= 0) return AWP_OK;
    if (t0 > p->nt) return set_err(AWP_ERR_PARAM, "checkpoint step %d beyond the %d steps of the solve", t0, p->nt);
    if (!s->media_loaded) return set_err(AWP_ERR_STATE, "media must be loaded before restoring a checkpoint");
    awp_status st = awp_sync(s);
    if (st != AWP_OK) return st;
    const size_t nvol = (size_t)(p->nx + 4) * (p->ny + 4) * (p->nz + 4);
    float *buf = (float *)malloc(nvol * sizeof(float));
    float *aux = (float *)malloc(sizeof(float) * ((size_t)3 * p->nt + (size_t)s->sgt_file_floats + 1));
    if (!buf || !aux) { free(buf); free(aux); return set_err(AWP_ERR_OOM, "host buffer"); }
    /* the first step of the restored solve must not insert addsrc(1) again */
    if (!s->started) st = start_if_needed(s);
    for (int q = 0; q < p->ncomp && st == AWP_OK; q++) {
        snprintf(path, sizeof path, "%s/ckp%07d%07d.bin", dir, q, t0);
        FILE *f = fopen(path, "rb");
        if (!f) { st = set_err(AWP_ERR_IO, "checkpoint %s missing", path); break; }
        for (int fld = 0; fld < AWP_NF_STATE && st == AWP_OK; fld++) {
            if (fld >= AF_R1 && s->rstore == AWP_STORE_BFP && s->comp[0][q].f[fld]) {
                /* block floating point: each group of three encoded at once */
                if ((fld - AF_R1) % 3 == 0) {
                    std::vector<float> grp(3 * nvol);
                    st = read_all(f, grp.data(), 3 * nvol * sizeof(float), path);
                    const float *v[3] = {&grp[0], &grp[nvol], &grp[2 * nvol]};
                    if (st == AWP_OK) st = bfp_set_group(s, q, (fld - AF_R1) / 3, v);
                }
                continue;
            }
            st = read_all(f, buf, nvol * sizeof(float), path);
            if (st == AWP_OK && s->comp[0][q].f[fld]) st = awp_set_field(s, q, fld, buf);
        }
        fclose(f);
        if (st != AWP_OK) break;
        if (p->npc == 1 && (st = pml_ckp_io(s, q, dir, t0, false)) != AWP_OK) break;
        CU(cudaSetDevice(p->device));
        snprintf(path, sizeof path, "%s/ckpsgt%07d%07d.bin", dir, q, t0);
        f = fopen(path, "rb");
        /* a checkpoint without it (written by the reference) restores the
         * wavefield only: SGT samples and CHKJ before the step stay zero */
        if (!f) continue;
        CkpSgtHeader h;
        st = read_all(f, &h, sizeof h, path);
        if (st == AWP_OK && (memcmp(h.magic, AWP_CKP_MAGIC, 8) != 0 || h.version != AWP_CKP_VERSION || h.step != t0 ||
                             h.nt != p->nt || h.npts != s->npts || h.nt_file != s->nt_file ||
                             h.sgt_floats != s->sgt_file_floats))
            st = set_err(AWP_ERR_IO, "%s does not match this solve (step, nt, points or SGT size)", path);
        if (st == AWP_OK)
            st = read_all(f, aux, sizeof(float) * ((size_t)3 * p->nt + (size_t)s->sgt_file_floats), path);
        fclose(f);
        if (st != AWP_OK) break;
        CU(cudaMemcpy(s->chkj[q], aux, sizeof(float) * 3 * (size_t)p->nt, cudaMemcpyHostToDevice));
        if (s->sgt_file_floats > 0)
            CU(cudaMemcpy(s->sgt_file[q], aux + (size_t)3 * p->nt, sizeof(float) * (size_t)s->sgt_file_floats,
                          cudaMemcpyHostToDevice));
    }
    free(buf);
    free(aux);
    if (st != AWP_OK) return st;
    /* the device step counter drives the source, CHKJ and SGT kernels */
    CU(cudaMemcpy(s->step, &t0, sizeof(int), cudaMemcpyHostToDevice));
    s->steps_done = t0;
    if (p->monitor_every > 0) s->next_check = (t0 / p->monitor_every + 1) * p->monitor_every;
    if (step_out) *step_out = t0;
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
    const size_t rb = (size_t)s->g.vol * (s->rstore == AWP_STORE_F32 ? 4 : 2);
    for (int q = 0; q < p->ncomp; q++) {
        for (int b = 0; b < 2; b++)
            for (int f = 0; f < AWP_NF_ARRAYS; f++) {
                if (!s->comp[b][q].f[f] || (b == 1 && s->comp[1][q].f[f] == s->comp[0][q].f[f])) continue;
                CU(cudaMemsetAsync(s->comp[b][q].f[f], 0, f >= AF_R1 ? rb : vb, s->stream));
            }
        CU(cudaMemsetAsync(s->chkj[q], 0, sizeof(float) * 3 * (size_t)p->nt, s->stream));
        if (s->sgt_file[q]) CU(cudaMemsetAsync(s->sgt_file[q], 0, sizeof(float) * (size_t)s->sgt_file_floats, s->stream));
    }
    for (int q = 0; q < p->ncomp; q++)
        if (s->pml_split[q]) CU(cudaMemsetAsync(s->pml_split[q], 0, sizeof(float) * (size_t)s->pml_floats, s->stream));
    CU(cudaMemsetAsync(s->step, 0, sizeof(int), s->stream));
    CU(cudaMemsetAsync(s->flag, 0, 2 * sizeof(int), s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->steps_done = 0;
    s->started = 0;
    s->loop_seconds = 0;
    s->loop_steps = 0;
    s->pending = 0;
    s->pending_steps = 0;
    s->next_check = p->monitor_every > 0 ? p->monitor_every : 0;
    return AWP_OK;
}

/* ------------------------------------------------------------------ */
/* device views and the FP64 energy                                    */
/* ------------------------------------------------------------------ */

static awp_layout layout_of(const AwpGeom &g)
{
    awp_layout L;
    L.nx = g.nx; L.ny = g.ny; L.nz = g.nz; L.pitch = g.px; L.plane = g.plane; L.vol = g.vol;
    return L;
}

extern "C" awp_status awp_device_field(awp_solver *s, int comp, int field, float **ptr, awp_layout *layout)
{
    if (!s || !ptr) return set_err(AWP_ERR_PARAM, "null argument");
    if (comp < 0 || comp >= s->p.ncomp || field < 0 || field >= AWP_NF_STATE + AM_N)
        return set_err(AWP_ERR_PARAM, "bad component/field");
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));
    *ptr = field < AWP_NF_STATE ? s->comp[cur_buf(s, s->steps_done)][comp].f[field]
                                : (float *)s->mdt.m[field - AWP_NF_STATE];
    if (layout) *layout = layout_of(s->g);
    return AWP_OK;
}

static awp_status check_layout(const float *const *fields, int ncomp, const awp_layout *L)
{
    if (!fields || !L) return set_err(AWP_ERR_PARAM, "null argument");
    if (ncomp < 1 || ncomp > AWP_MAX_COMP) return set_err(AWP_ERR_PARAM, "ncomp must be 1..3");
    if (L->nx < 1 || L->ny < 1 || L->nz < 1 || L->pitch < L->nx + AWP_XO + 2 || L->plane < L->pitch * (L->ny + 4) ||
        L->vol < (int64_t)L->plane * (L->nz + 4) || L->vol >= ((int64_t)1 << 31))
        return set_err(AWP_ERR_PARAM, "inconsistent layout");
    for (int n = 0; n < 3 * ncomp; n++)
        if (!fields[n]) return set_err(AWP_ERR_PARAM, "null field pointer %d", n);
    return AWP_OK;
}

static void energy_args_from(const float *const *fields, int ncomp, const awp_layout *L, AwpEnergyArgs &a)
{
    memset(&a, 0, sizeof a);
    a.g.nx = L->nx; a.g.ny = L->ny; a.g.nz = L->nz;
    a.g.px = L->pitch; a.g.py = L->ny + 4; a.g.plane = L->plane; a.g.vol = L->vol;
    a.ncomp = ncomp;
    for (int n = 0; n < 3 * ncomp; n++) a.f[n] = fields[n];
}

extern "C" awp_status awp_field_energy(const float *const *fields, int ncomp, const awp_layout *L, double *out)
{
    awp_status st = check_layout(fields, ncomp, L);
    if (st != AWP_OK) return st;
    if (!out) return set_err(AWP_ERR_PARAM, "null output");
    AwpEnergyArgs a;
    energy_args_from(fields, ncomp, L, a);
    double *partial = NULL;
    CU(cudaMalloc((void **)&partial, sizeof(double) * AWP_EN_GRID * ncomp));
    cudaError_t e = awp_launch_energy(a, partial, AWP_EN_GRID, out, NULL, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    cudaFree(partial);
    if (e != cudaSuccess) return set_err(AWP_ERR_CUDA, "awp_field_energy: %s", cudaGetErrorString(e));
    return AWP_OK;
}

/* Scratch of awp_field_energy_noalloc: the pass-1 partial sums, one FP64
 * value per block and component (592 x 3 doubles, 14,208 bytes), in static
 * device memory of this module so that the call itself allocates nothing.
 * Every slot pass 2 reads is written by pass 1 of the same call, so nothing
 * has to start at zero.  Calls on one device share it: two of them that
 * overlap in time (other streams or threads) race on it. */
#define AWP_NOALLOC_PARTIALS (AWP_EN_GRID * AWP_MAX_COMP)
#define AWP_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) double g_energy_scratch[AWP_NOALLOC_PARTIALS];
static double *g_energy_scratch_addr[AWP_NOALLOC_MAX_DEVICES];
static std::mutex g_energy_scratch_mu;

/* Device address of the scratch on the current device: looked up once per
 * device (cudaGetSymbolAddress, which may load this module onto the device --
 * the reason the first call on a device is the set-up call), then cached for
 * the life of the process.  A device reset (cudaDeviceReset) between calls
 * would leave the cached address stale; the header rules that out. */
static awp_status energy_scratch(double **addr)
{
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= AWP_NOALLOC_MAX_DEVICES)
        return set_err(AWP_ERR_PARAM, "awp_field_energy_noalloc: device %d beyond the %d it keeps scratch for", dev,
                       AWP_NOALLOC_MAX_DEVICES);
    std::lock_guard<std::mutex> lock(g_energy_scratch_mu);
    if (!g_energy_scratch_addr[dev]) {
        void *a = NULL;
        const cudaError_t e = cudaGetSymbolAddress(&a, g_energy_scratch);
        if (e != cudaSuccess || !a)
            return set_err(AWP_ERR_CUDA, "awp_field_energy_noalloc: scratch address on device %d: %s", dev,
                           cudaGetErrorString(e));
        g_energy_scratch_addr[dev] = (double *)a;
    }
    *addr = g_energy_scratch_addr[dev];
    return AWP_OK;
}

extern "C" awp_status awp_field_energy_noalloc(const float *const *fields, int ncomp, const awp_layout *L,
                                               double *out, void *stream)
{
    if (ncomp > AWP_MAX_COMP || (int64_t)ncomp * AWP_EN_GRID > AWP_NOALLOC_PARTIALS)
        return set_err(AWP_ERR_PARAM, "awp_field_energy_noalloc: %d components exceed the static scratch "
                       "(%d partial sums: at most %d components)", ncomp, AWP_NOALLOC_PARTIALS, AWP_MAX_COMP);
    awp_status st = check_layout(fields, ncomp, L);
    if (st != AWP_OK) return st;
    if (!out) return set_err(AWP_ERR_PARAM, "null output");
    /* an error left pending by earlier work of this thread is not this call's
     * failure: report it without clearing it, and launch nothing */
    const cudaError_t pend = cudaPeekAtLastError();
    if (pend != cudaSuccess)
        return set_err(AWP_ERR_CUDA, "awp_field_energy_noalloc: a CUDA error from earlier work is pending: %s",
                       cudaGetErrorString(pend));
    double *partial = NULL;
    st = energy_scratch(&partial);
    if (st != AWP_OK) return st;
    AwpEnergyArgs a;
    energy_args_from(fields, ncomp, L, a);
    const cudaError_t e = awp_launch_energy(a, partial, AWP_EN_GRID, out, NULL, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_err(AWP_ERR_CUDA, "awp_field_energy_noalloc: %s", cudaGetErrorString(e));
    return AWP_OK;
}

extern "C" awp_status awp_energy(awp_solver *s, double *out)
{
    if (!s || !out) return set_err(AWP_ERR_PARAM, "null argument");
    CU(cudaSetDevice(s->p.device));
    AwpEnergyArgs a;
    energy_args(s, a);
    CU(awp_launch_energy(a, s->en_partial, AWP_EN_GRID, s->en_out, NULL, s->stream));
    CU(cudaMemcpyAsync(out, s->en_out, sizeof(double) * s->p.ncomp, cudaMemcpyDeviceToHost, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    return AWP_OK;
}

/* ------------------------------------------------------------------ */
/* launch shapes and the autotuner                                     */
/* ------------------------------------------------------------------ */

static void drop_graphs(awp_solver *s)
{
    for (int b = 0; b < 2; b++)
        if (s->graph[b]) {
            cudaGraphExecDestroy(s->graph[b]);
            s->graph[b] = NULL;
        }
}

extern "C" awp_status awp_get_tuning(awp_solver *s, awp_tuning *t)
{
    if (!s || !t) return set_err(AWP_ERR_PARAM, "awp_get_tuning: null argument");
    t->kchunk_staged = s->kchunk_staged;
    t->staged_qslow = s->staged_qslow;
    t->staged_rpt = s->staged_rpt;
    t->staged_rpt_vel = s->staged_rpt_vel;
    t->unroll = s->unroll;
    t->ty = s->ty;
    t->kchunk = s->kchunk;
    t->kchunk_sweep = s->kchunk_sweep;
    t->staged_batch = s->staged_batch;
    t->sm_limit = s->sm_limit;
    return AWP_OK;
}

extern "C" awp_status awp_set_tuning(awp_solver *s, const awp_tuning *t)
{
    if (!s || !t) return set_err(AWP_ERR_PARAM, "awp_set_tuning: null argument");
    const int nz = s->g.nz, kmax = nz > 8 ? nz : 8;
    if (t->kchunk_staged < 8 || t->kchunk_staged > kmax || t->kchunk < 8 || t->kchunk > kmax ||
        t->kchunk_sweep < 8 || t->kchunk_sweep > kmax)
        return set_err(AWP_ERR_PARAM, "awp_set_tuning: z levels per work item must be 8..%d", kmax);
    if ((t->staged_qslow != 0 && t->staged_qslow != 1) || (t->staged_rpt != 1 && t->staged_rpt != 2) ||
        (t->staged_rpt_vel != 1 && t->staged_rpt_vel != 2) || (t->unroll != 1 && t->unroll != 2) ||
        (t->ty != 4 && t->ty != 8 && t->ty != 16) || t->staged_batch < 0 || t->staged_batch > 3 || t->sm_limit < 0)
        return set_err(AWP_ERR_PARAM, "awp_set_tuning: qslow 0/1, rows per thread 1/2, unroll 1/2, ty 4/8/16, batch "
                       "0-3, sm_limit >= 0");
    CU(cudaSetDevice(s->p.device));
    CU(cudaStreamSynchronize(s->stream));   /* no captured step in flight when its graph goes */
    s->kchunk_staged = t->kchunk_staged;
    s->staged_qslow = t->staged_qslow;
    s->staged_rpt = t->staged_rpt;
    s->staged_rpt_vel = t->staged_rpt_vel;
    s->unroll = t->unroll;
    s->ty = t->ty;
    s->kchunk = t->kchunk;
    s->kchunk_sweep = t->kchunk_sweep;
    s->staged_batch = t->staged_batch;
    s->sm_limit = t->sm_limit;
    drop_graphs(s);
    return AWP_OK;
}

/* "nx ny nz ncomp precision nve stepper gpu-model" */
static void tune_key(const awp_params *p, int stepper, char *key, size_t n)
{
    cudaDeviceProp prop;
    char model[256] = "unknown";
    if (cudaGetDeviceProperties(&prop, p->device) == cudaSuccess) {
        snprintf(model, sizeof model, "%s", prop.name);
        for (char *c = model; *c; ++c)
            if (*c == ' ') *c = '_';
    }
    snprintf(key, n, "%d %d %d %d %d %d %d %s", p->nx, p->ny, p->nz, p->ncomp, (int)p->precision, p->nve, stepper,
             model);
}

static int tune_cache_get(const char *path, const char *key, awp_tuning *t, double *rate)
{
    FILE *f = path ? fopen(path, "r") : NULL;
    if (!f) return 0;
    char line[512];
    int found = 0;
    const size_t kl = strlen(key);
    while (fgets(line, sizeof line, f)) {
        if (strncmp(line, key, kl) != 0 || line[kl] != ' ') continue;
        awp_tuning u;
        double r = 0.0;
        if (sscanf(line + kl, "%d %d %d %d %d %d %d %d %d %lf", &u.kchunk_staged, &u.staged_qslow, &u.staged_rpt,
                   &u.staged_rpt_vel, &u.unroll, &u.ty, &u.kchunk, &u.kchunk_sweep, &u.staged_batch, &r) == 10) {
            *t = u;
            *rate = r;
            found = 1;                        /* the last entry for a key wins */
        }
    }
    fclose(f);
    return found;
}

static void tune_cache_put(const char *path, const char *key, const awp_tuning *t, double rate)
{
    FILE *f = path ? fopen(path, "a") : NULL;
    if (!f) return;
    fprintf(f, "%s %d %d %d %d %d %d %d %d %d %.6g\n", key, t->kchunk_staged, t->staged_qslow, t->staged_rpt,
            t->staged_rpt_vel, t->unroll, t->ty, t->kchunk, t->kchunk_sweep, t->staged_batch, rate);
    fclose(f);
}

/* Gcell-updates/s of trial_steps steps with tuning t (after one warm-up
 * step that rebuilds the captured graph) */
static awp_status tune_trial(awp_solver *s, const awp_tuning *t, int trial_steps, double *rate)
{
    awp_status st = awp_set_tuning(s, t);
    if (st != AWP_OK) return st;
    if ((st = awp_run(s, s->p.ntiskp_sgt, NULL)) != AWP_OK) return st;
    awp_stats a, b;
    if ((st = awp_get_stats(s, &a)) != AWP_OK) return st;
    if ((st = awp_run(s, trial_steps, NULL)) != AWP_OK) return st;
    if ((st = awp_get_stats(s, &b)) != AWP_OK) return st;
    const double sec = b.seconds_loop - a.seconds_loop;
    const double upd = (double)s->g.nx * s->g.ny * s->g.nz * s->p.ncomp * (double)(b.steps_done - a.steps_done);
    *rate = sec > 0 ? upd / sec * 1e-9 : 0.0;
    return AWP_OK;
}

extern "C" awp_status awp_autotune(const awp_params *pin, const float *media, int trial_steps, const char *cache_path,
                                   awp_tuning *best, double *gcell_updates_per_s)
{
    if (!pin || !best) return set_err(AWP_ERR_PARAM, "awp_autotune: null argument");
    if (trial_steps < 1 || trial_steps > 100000)
        return set_err(AWP_ERR_PARAM, "awp_autotune: trial_steps must be 1..100000");
    awp_params p = *pin;
    const int max_trials = 24;
    p.nt = max_trials * (trial_steps + p.ntiskp_sgt) + p.ntiskp_sgt + 1;
    p.nst = 1;
    p.monitor_every = 0;
    if (!media) p.mediastart = 0;
    awp_solver *s = NULL;
    awp_status st = awp_create(&p, &s);
    if (st != AWP_OK) return st;
    const int stepper = s->staged_on ? (s->fma ? AWP_KERNEL_STAGED_FMA : AWP_KERNEL_STAGED)
                                     : (fused_of(&s->p) ? AWP_KERNEL_FUSED : AWP_KERNEL_TWO_SWEEP);
    char key[320];
    tune_key(&p, stepper, key, sizeof key);
    double rate = 0.0;
    awp_tuning t;
    if (tune_cache_get(cache_path, key, &t, &rate)) {
        awp_destroy(s);
        *best = t;
        if (gcell_updates_per_s) *gcell_updates_per_s = rate;
        return AWP_OK;
    }
    /* without media the trial solve uses the homogeneous medium (inihomo):
     * the speed of a step does not depend on the values */
    st = awp_load_media(s, media);
    /* a developed wavefield: under the power cap a zero wavefield runs at
     * higher clocks than a real solve, so the trials start from bounded noise
     * in u v w and the stresses (the memory variables follow within a step) */
    for (int q = 0; q < p.ncomp && st == AWP_OK; q++)
        for (int b = 0; b < 2 && st == AWP_OK; b++)
            for (int f = 0; f < 9 && st == AWP_OK; f++) {
                if (b == 1 && s->comp[1][q].f[f] == s->comp[0][q].f[f]) continue;
                const cudaError_t e = awp_launch_fill_noise(s->comp[b][q].f[f], s->g.vol,
                                                            0x5EED0000u + 64u * q + 16u * b + f, 1e-3f, s->stream);
                if (e != cudaSuccess) st = set_err(AWP_ERR_CUDA, "awp_autotune: %s", cudaGetErrorString(e));
            }
    awp_tuning cur;
    if (st == AWP_OK) st = awp_get_tuning(s, &cur);
    double cur_rate = 0.0;
    if (st == AWP_OK) st = tune_trial(s, &cur, trial_steps, &cur_rate);
    /* coordinate descent over the fields the stepper uses */
    enum { F_KSTAGE, F_RPT, F_UNROLL, F_QSLOW, F_RPTV, F_TY, F_KFUSED, F_KSWEEP, F_BATCH };
    int fields[9], nf = 0;
    if (stepper == AWP_KERNEL_STAGED || stepper == AWP_KERNEL_STAGED_FMA) {
        if (p.ncomp >= 2) fields[nf++] = F_BATCH;
        fields[nf++] = F_KSTAGE, fields[nf++] = F_RPT, fields[nf++] = F_UNROLL, fields[nf++] = F_QSLOW;
        fields[nf++] = F_RPTV;
    } else if (stepper == AWP_KERNEL_FUSED) {
        fields[nf++] = F_TY, fields[nf++] = F_KFUSED;
    } else {
        fields[nf++] = F_TY, fields[nf++] = F_UNROLL, fields[nf++] = F_KSWEEP;
    }
    int trials = 1;
    for (int fi = 0; fi < nf && st == AWP_OK; fi++) {
        int vals[6], nv = 0;
        switch (fields[fi]) {
        case F_KSTAGE:
            for (int target : {24, 32, 40, 48, 64}) {
                const int nch = (p.nz + target - 1) / target;
                int kc = (p.nz + nch - 1) / nch;
                kc = kc < 8 ? 8 : kc;
                bool dup = kc == cur.kchunk_staged;
                for (int i = 0; i < nv; i++) dup = dup || vals[i] == kc;
                if (!dup) vals[nv++] = kc;
            }
            break;
        /* the side-by-side sweeps ignore rows per thread and component order */
        case F_RPT:
            if (!((cur.staged_batch & 1) && p.ncomp >= 2)) vals[nv++] = 3 - cur.staged_rpt;
            break;
        case F_RPTV:
            if (!((cur.staged_batch & 2) && p.ncomp >= 2)) vals[nv++] = 3 - cur.staged_rpt_vel;
            break;
        case F_UNROLL: vals[nv++] = 3 - cur.unroll; break;
        case F_QSLOW:
            if (!(cur.staged_batch == 3 && p.ncomp >= 2)) vals[nv++] = 1 - cur.staged_qslow;
            break;
        case F_BATCH:
            for (int b = 0; b < 4; b++)
                if (b != cur.staged_batch) vals[nv++] = b;
            break;
        case F_TY:
            for (int ty : {4, 8, 16})
                if (ty != cur.ty && (stepper == AWP_KERNEL_FUSED || ty != 16)) vals[nv++] = ty;
            break;
        case F_KFUSED:
            for (int kc : {16, 32, 64})
                if (kc != cur.kchunk && kc <= (p.nz > 8 ? p.nz : 8)) vals[nv++] = kc;
            break;
        case F_KSWEEP:
            for (int kc : {16, 32})
                if (kc != cur.kchunk_sweep && kc <= (p.nz > 8 ? p.nz : 8)) vals[nv++] = kc;
            break;
        }
        for (int vi = 0; vi < nv && st == AWP_OK && trials < max_trials; vi++, trials++) {
            awp_tuning cand = cur;
            switch (fields[fi]) {
            case F_KSTAGE: cand.kchunk_staged = vals[vi]; break;
            case F_RPT: cand.staged_rpt = vals[vi]; break;
            case F_RPTV: cand.staged_rpt_vel = vals[vi]; break;
            case F_UNROLL: cand.unroll = vals[vi]; break;
            case F_QSLOW: cand.staged_qslow = vals[vi]; break;
            case F_BATCH: cand.staged_batch = vals[vi]; break;
            case F_TY: cand.ty = vals[vi]; break;
            case F_KFUSED: cand.kchunk = vals[vi]; break;
            case F_KSWEEP: cand.kchunk_sweep = vals[vi]; break;
            }
            double r = 0.0;
            st = tune_trial(s, &cand, trial_steps, &r);
            if (st == AWP_OK && r > cur_rate) cur = cand, cur_rate = r;
        }
    }
    awp_destroy(s);
    if (st != AWP_OK) return st;
    *best = cur;
    if (gcell_updates_per_s) *gcell_updates_per_s = cur_rate;
    tune_cache_put(cache_path, key, &cur, cur_rate);
    return AWP_OK;
}
