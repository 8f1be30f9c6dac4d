/*
 * awp_oracle.c -- CPU restatement of the AWP-ODC-SGT Fortran time stepper.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this code, and only as
 * the oracle the device results are compared with or as the timed CPU
 * baseline.  The product path (the CUDA library under cybershake-core_b200/)
 * never links, loads or calls it.
 *
 * PINNING.  The reference ships no solver tests, no golden SGT output and no
 * fixtures for this path, and its Fortran cannot be built in this image (no
 * Fortran compiler, no MPI).  This file restates the Fortran semantics
 * statement by statement, with the same evaluation order, and is pinned to
 * code the reference ships, built from its sources (tests/test_oracle_pin.py):
 *   - the set-up stage (media transform, relaxation times, Cerjan factors) to
 *     the reference CUDA variant's host code (mesh.c, cerjan.c);
 *   - the time loop (velocity, stress and memory-variable updates with the
 *     sponge) to that variant's own dvelcx and dstrqc kernels run on the host
 *     CPU, within 2e-6 relative L2 per field after several steps (their
 *     arithmetic is an algebraic regrouping of the Fortran's), in the cells
 *     the free surface does not reach -- the CUDA variant's free-surface
 *     image differs from the Fortran's by design;
 * and checked by known-answer tests (analytic travel times, linearity,
 * symmetry).  The free-surface, source and SGT-gather statements follow the
 * Fortran lines cited below and are covered by those known-answer tests.
 *
 * Compiled twice: -DORC_REAL=float (FP32, operation order of the Fortran) and
 * -DORC_REAL=double (FP64 reference for rounding error).  Inputs are always
 * FP32 (the reference reads FP32 files); the FP64 build promotes them.
 *
 * Index convention (Fortran): i = 1..nx (x), j = 1..ny (y), k = 1..nz (z) with
 * k = nz the free surface; every array carries two ghost cells per side
 * (Fortran bounds -1:n+2, memory.f:147-156).
 *
 * Reference files followed (paths inside the reference project):
 *   AWP-ODC-SGT/src/operator.f:92-306, 575-612   velocity, free surface
 *   AWP-ODC-SGT/src/viscoop.f:49-191             stress + memory variables
 *   AWP-ODC-SGT/src/relax.f:4-39                 relaxation times
 *   AWP-ODC-SGT/src/structure.f:449-558, 563-707, 709-765  media
 *   AWP-ODC-SGT/src/cerjan.f:4-330               sponge
 *   AWP-ODC-SGT/src/source.f:812-913             source insertion
 *   AWP-ODC-SGT/src/station.f:31-80              SGT point location
 *   AWP-ODC-SGT/src/pmcl3d.f:966-988, 1158-1173, 1183-1611  main loop, SGT
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORC_REAL
#define ORC_REAL float
#endif
typedef ORC_REAL real;

#define ORC_IS_F64 (sizeof(real) == 8)

static inline real r_exp(real x) { return ORC_IS_F64 ? (real)exp((double)x) : (real)expf((float)x); }
static inline real r_log(real x) { return ORC_IS_F64 ? (real)log((double)x) : (real)logf((float)x); }
static inline real r_sqrt(real x) { return ORC_IS_F64 ? (real)sqrt((double)x) : (real)sqrtf((float)x); }
static inline real r_atan(real x) { return ORC_IS_F64 ? (real)atan((double)x) : (real)atanf((float)x); }

/* Parameters: the subset of IN3D (io.f:327-417) that the stepper uses. */
typedef struct {
    int nx, ny, nz;
    float dh, dt;
    int nd;
    float arbc;
    float fl, fh, fp;
    int socalq;
    int nve;         /* 1 = viscoelastic (the CyberShake setting) */
    int mediastart;  /* 0 = homogeneous (inihomo), >0 = read from media array */
    int nvar;        /* 3, 5 or 8 */
    int idyna;       /* only selects the homogeneous medium values */
    int nst;         /* source time-function length */
    int nt;          /* number of time steps */
    int ntiskp_sgt;
    int write_step;
    int igreen;
    int kinematic;   /* 1: IFAULT=5 subfault sources (NST = 2) */
    int rstore;      /* storage of r1..r6 (FP32 build only): ORC_RS_* */
    int npc;         /* 1: PML absorbing boundary (pml.f), 0: Cerjan sponge */
    float pht;       /* PHT: PML damping ratio of the splits tangential to a face */
} orc_params;

/* Storage formats of the memory variables r1..r6 emulated by the FP32 build:
 * the new value of a memory variable feeds the stress update as computed and
 * is stored rounded to the format (the device steppers' order).  Stochastic
 * rounding takes its bits from orc_sr_bits, a counter-based hash of the cell,
 * the step and the variable, which the device kernels compute the same way. */
enum { ORC_RS_F32 = 0, ORC_RS_BF16_RN = 1, ORC_RS_BF16_SR = 2, ORC_RS_F16M_RN = 3, ORC_RS_F16M_SR = 4,
       ORC_RS_BFP6 = 5, ORC_RS_BFP33 = 6 };

enum { F_U1, F_V1, F_W1, F_XX, F_YY, F_ZZ, F_XY, F_XZ, F_YZ,
       F_R1, F_R2, F_R3, F_R4, F_R5, F_R6,
       F_LAM, F_MU, F_D1, F_QP, F_QS, F_NFIELDS };

typedef struct {
    orc_params p;
    int sx, sy, sz;      /* padded extents n+4 */
    size_t nvol;
    real *f[F_NFIELDS];
    real tau1[2][2][2], tau2[2][2][2];   /* [itz][ity][itx], 0-based parity */
    real tau[2][2][2];                   /* relaxation times before viscoop.f:80-88 */
    real *cx, *cy, *cz;                  /* 1-D sponge factors, index 1..n */
    float vpe[2], vse[2], dde[2];
    /* source */
    int nsrc;
    int *src;            /* local (i,j,k) per source */
    float *stf;          /* [nsrc][nst][6] : axx ayy azz axz ayz axy */
    /* SGT points */
    int npts;
    int *pts;            /* local (i,j,k) */
    real *sg;            /* [npts][3] : sg1 sg2 sg3 */
    float *sgt_buf;      /* [npts][6][write_step] */
    int sgt_count;
    float *sgt_file;     /* raw SGT file image */
    int64_t sgt_file_floats;
    int nt_file;
    float *chkj;         /* [nt][3] */
    int cur;             /* completed steps */
    int started;
    /* PML (npc = 1): T and H splits of the nine fields per plane S N W E B */
    real *pml[5][2][9];
    real *rf, *rh;       /* damping profiles, index 1..nd */
    int box[6];          /* x0 x1 y0 y1 z0 z1 of the 4th-order interior zone */
} orc_t;

#define IDX(h, i, j, k) ((((size_t)((k) + 1)) * (size_t)(h)->sy + (size_t)((j) + 1)) * (size_t)(h)->sx + (size_t)((i) + 1))

/* ------------------------------------------------------------------ */
/* creation                                                            */
/* ------------------------------------------------------------------ */

static void orc_tausub(orc_t *h, real taumin, real taumax)
{
    /* relax.f:15-36 ; tautem(idx,idy,idz) */
    static const int tautem[2][2][2] = {   /* [idz][idy][idx] */
        {{1, 6}, {7, 4}},
        {{8, 3}, {2, 5}},
    };
    real dt1 = (real)1 / (real)h->p.dt;   /* viscoop.f:79 */
    for (int z = 0; z < 2; z++)
        for (int y = 0; y < 2; y++)
            for (int x = 0; x < 2; x++) {
                real tmp = (real)tautem[z][y][x];
                tmp = (tmp - (real)0.5) / (real)8;
                tmp = (real)2.0 * tmp - (real)1.0;
                real tau = r_exp((real)0.5 * (r_log(taumax * taumin) + r_log(taumax / taumin) * tmp));
                h->tau[z][y][x] = tau;
                /* viscoop.f:80-88 */
                h->tau1[z][y][x] = (real)1 / ((tau * dt1) + ((real)1. / (real)2.));
                h->tau2[z][y][x] = (tau * dt1) - ((real)1. / (real)2.);
            }
}

static real crj_low(real alpha, int nd, int g)   /* cerjan.f:52 */
{
    real a = alpha * (real)(nd - g + 1);
    return r_exp(-(a * a));
}
static real crj_high(real alpha, int nd, int n, int g)   /* cerjan.f:76 */
{
    real a = alpha * (real)(nd - (n - g));
    return r_exp(-(a * a));
}

static void orc_inicrj(orc_t *h)
{
    /* cerjan.f:19 ; both lateral faces damped (multi-rank behaviour), bottom
     * face damped, free surface undamped.  The 3-D zone arrays of the
     * Fortran hold the separable product ((1*fx)*fy)*fz of these factors. */
    const orc_params *p = &h->p;
    real alpha = r_sqrt(-r_log((real)p->arbc)) / (real)p->nd;
    h->cx = calloc((size_t)p->nx + 2, sizeof(real));
    h->cy = calloc((size_t)p->ny + 2, sizeof(real));
    h->cz = calloc((size_t)p->nz + 2, sizeof(real));
    for (int i = 1; i <= p->nx; i++) {
        real f = 1;
        if (i <= p->nd) f = f * crj_low(alpha, p->nd, i);
        if (i >= p->nx - p->nd + 1) f = f * crj_high(alpha, p->nd, p->nx, i);
        h->cx[i] = f;
    }
    for (int j = 1; j <= p->ny; j++) {
        real f = 1;
        if (j <= p->nd) f = f * crj_low(alpha, p->nd, j);
        if (j >= p->ny - p->nd + 1) f = f * crj_high(alpha, p->nd, p->ny, j);
        h->cy[j] = f;
    }
    for (int k = 1; k <= p->nz; k++) {
        real f = 1;
        if (k <= p->nd) f = f * crj_low(alpha, p->nd, k);
        h->cz[k] = f;
    }
}

void orc_destroy(orc_t *h)
{
    if (!h) return;
    for (int q = 0; q < F_NFIELDS; q++) free(h->f[q]);
    free(h->cx); free(h->cy); free(h->cz);
    free(h->src); free(h->stf); free(h->pts); free(h->sg);
    free(h->sgt_buf); free(h->sgt_file); free(h->chkj);
    for (int a = 0; a < 5; a++)
        for (int b = 0; b < 2; b++)
            for (int f = 0; f < 9; f++) free(h->pml[a][b][f]);
    free(h->rf); free(h->rh);
    free(h);
}

/* nt_file = int(int(nt/write_step)*write_step/ntiskp_sgt)  (pmcl3d.f:1590-1594) */
static int orc_nt_file(const orc_params *p)
{
    return ((p->nt / p->write_step) * p->write_step) / p->ntiskp_sgt;
}

orc_t *orc_create(const orc_params *p)
{
    if (p->nx < 4 || p->ny < 4 || p->nz < 4 || p->nd < 1 || p->dt <= 0 || p->dh <= 0) return NULL;
    if (p->ntiskp_sgt < 1 || p->write_step < 1 || p->nt < 1) return NULL;
    if (p->kinematic && p->nst != 2) return NULL;   /* two rows per subfault */
    orc_t *h = calloc(1, sizeof(orc_t));
    h->p = *p;
    h->sx = p->nx + 4; h->sy = p->ny + 4; h->sz = p->nz + 4;
    h->nvol = (size_t)h->sx * h->sy * h->sz;
    for (int q = 0; q < F_NFIELDS; q++) {
        h->f[q] = calloc(h->nvol, sizeof(real));
        if (!h->f[q]) { orc_destroy(h); return NULL; }
    }
    orc_inicrj(h);
    h->chkj = calloc((size_t)p->nt * 3, sizeof(float));
    h->nt_file = orc_nt_file(p);
    h->box[0] = 1; h->box[1] = p->nx; h->box[2] = 1; h->box[3] = p->ny; h->box[4] = 1; h->box[5] = p->nz;
    if (p->npc == 1) {
        /* plane extents (memory.f:217-300): S, N nx x nd x nz; W, E nd x ny x nz; B nx x ny x nd */
        if (2 * p->nd >= p->nx || 2 * p->nd >= p->ny || p->nd >= p->nz) { orc_destroy(h); return NULL; }
        const size_t n[5] = {(size_t)p->nx * p->nd * p->nz, (size_t)p->nx * p->nd * p->nz,
                             (size_t)p->nd * p->ny * p->nz, (size_t)p->nd * p->ny * p->nz,
                             (size_t)p->nx * p->ny * p->nd};
        for (int a = 0; a < 5; a++)
            for (int b = 0; b < 2; b++)
                for (int f = 0; f < 9; f++)
                    if (!(h->pml[a][b][f] = calloc(n[a], sizeof(real)))) { orc_destroy(h); return NULL; }
        h->rf = calloc((size_t)p->nd + 2, sizeof(real));
        h->rh = calloc((size_t)p->nd + 2, sizeof(real));
        /* the interior zone 18 (bound.f:890-892) */
        h->box[0] = p->nd + 1; h->box[1] = p->nx - p->nd; h->box[2] = p->nd + 1; h->box[3] = p->ny - p->nd;
        h->box[4] = p->nd + 1;
    }
    return h;
}

int orc_nt_file_of(const orc_t *h) { return h->nt_file; }

/* ------------------------------------------------------------------ */
/* media: inimesh cases 0-2 (structure.f:88-93, 449-558), padmedia,    */
/* afsmedia (structure.f:563-707), inihomo (structure.f:709-765)       */
/* ------------------------------------------------------------------ */

static void orc_padmedia(orc_t *h)
{
    const int nxt = h->p.nx, nyt = h->p.ny, nzt = h->p.nz;
    real *lam = h->f[F_LAM], *mu = h->f[F_MU], *d1 = h->f[F_D1];
#define M(a, i, j, k) a[IDX(h, i, j, k)]
    for (int k = 1; k <= nzt; k++)
        for (int j = 1; j <= nyt; j++) {
            M(lam, 0, j, k) = M(lam, 1, j, k); M(lam, nxt + 1, j, k) = M(lam, nxt, j, k);
            M(mu, 0, j, k) = M(mu, 1, j, k);   M(mu, nxt + 1, j, k) = M(mu, nxt, j, k);
            M(d1, 0, j, k) = M(d1, 1, j, k);   M(d1, nxt + 1, j, k) = M(d1, nxt, j, k);
        }
    for (int k = 1; k <= nzt; k++)
        for (int i = 1; i <= nxt; i++) {
            M(lam, i, 0, k) = M(lam, i, 1, k); M(lam, i, nyt + 1, k) = M(lam, i, nyt, k);
            M(mu, i, 0, k) = M(mu, i, 1, k);   M(mu, i, nyt + 1, k) = M(mu, i, nyt, k);
            M(d1, i, 0, k) = M(d1, i, 1, k);   M(d1, i, nyt + 1, k) = M(d1, i, nyt, k);
        }
    for (int j = 1; j <= nyt; j++)
        for (int i = 1; i <= nxt; i++) {
            M(lam, i, j, 0) = M(lam, i, j, 1);
            M(mu, i, j, 0) = M(mu, i, j, 1);
            M(d1, i, j, 0) = M(d1, i, j, 1);
        }
    for (int i = 1; i <= nxt; i++) {
        M(lam, i, 0, 0) = M(lam, i, 1, 1); M(mu, i, 0, 0) = M(mu, i, 1, 1); M(d1, i, 0, 0) = M(d1, i, 1, 1);
        M(lam, i, nyt + 1, 0) = M(lam, i, nyt, 1); M(mu, i, nyt + 1, 0) = M(mu, i, nyt, 1); M(d1, i, nyt + 1, 0) = M(d1, i, nyt, 1);
        M(lam, i, 0, nzt + 1) = M(lam, i, 1, nzt); M(mu, i, 0, nzt + 1) = M(mu, i, 1, nzt); M(d1, i, 0, nzt + 1) = M(d1, i, 1, nzt);
        M(lam, i, nyt + 1, nzt + 1) = M(lam, i, nyt, nzt); M(mu, i, nyt + 1, nzt + 1) = M(mu, i, nyt, nzt); M(d1, i, nyt + 1, nzt + 1) = M(d1, i, nyt, nzt);
    }
    for (int j = 1; j <= nyt; j++) {
        M(lam, 0, j, 0) = M(lam, 1, j, 1); M(mu, 0, j, 0) = M(mu, 1, j, 1); M(d1, 0, j, 0) = M(d1, 1, j, 1);
        M(lam, nxt + 1, j, 0) = M(lam, nxt, j, 1); M(mu, nxt + 1, j, 0) = M(mu, nxt, j, 1); M(d1, nxt + 1, j, 0) = M(d1, nxt, j, 1);
        M(lam, 0, j, nzt + 1) = M(lam, 1, j, nzt); M(mu, 0, j, nzt + 1) = M(mu, 1, j, nzt); M(d1, 0, j, nzt + 1) = M(d1, 1, j, nzt);
        M(lam, nxt + 1, j, nzt + 1) = M(lam, nxt, j, nzt); M(mu, nxt + 1, j, nzt + 1) = M(mu, nxt, j, nzt); M(d1, nxt + 1, j, nzt + 1) = M(d1, nxt, j, nzt);
    }
    for (int k = 1; k <= nzt; k++) {
        M(lam, 0, 0, k) = M(lam, 1, 1, k); M(mu, 0, 0, k) = M(mu, 1, 1, k); M(d1, 0, 0, k) = M(d1, 1, 1, k);
        M(lam, nxt + 1, 0, k) = M(lam, nxt, 1, k); M(mu, nxt + 1, 0, k) = M(mu, nxt, 1, k); M(d1, nxt + 1, 0, k) = M(d1, nxt, 1, k);
        M(lam, 0, nyt + 1, k) = M(lam, 1, nyt, k); M(mu, 0, nyt + 1, k) = M(mu, 1, nyt, k); M(d1, 0, nyt + 1, k) = M(d1, 1, nyt, k);
        M(lam, nxt + 1, nyt + 1, k) = M(lam, nxt, nyt, k); M(mu, nxt + 1, nyt + 1, k) = M(mu, nxt, nyt, k); M(d1, nxt + 1, nyt + 1, k) = M(d1, nxt, nyt, k);
    }
    /* 8 corners (structure.f:650-673), including the two assignments at
     * (nxt+1,0,0) that copy lam into mu and d1. */
    M(lam, 0, 0, 0) = M(lam, 1, 1, 1); M(mu, 0, 0, 0) = M(mu, 1, 1, 1); M(d1, 0, 0, 0) = M(d1, 1, 1, 1);
    M(lam, nxt + 1, 0, 0) = M(lam, nxt, 1, 1); M(mu, nxt + 1, 0, 0) = M(lam, nxt, 1, 1); M(d1, nxt + 1, 0, 0) = M(lam, nxt, 1, 1);
    M(lam, 0, nyt + 1, 0) = M(lam, 1, nyt, 1); M(mu, 0, nyt + 1, 0) = M(mu, 1, nyt, 1); M(d1, 0, nyt + 1, 0) = M(d1, 1, nyt, 1);
    M(lam, 0, 0, nzt + 1) = M(lam, 1, 1, nzt); M(mu, 0, 0, nzt + 1) = M(mu, 1, 1, nzt); M(d1, 0, 0, nzt + 1) = M(d1, 1, 1, nzt);
    M(lam, nxt + 1, 0, nzt + 1) = M(lam, nxt, 1, nzt); M(mu, nxt + 1, 0, nzt + 1) = M(mu, nxt, 1, nzt); M(d1, nxt + 1, 0, nzt + 1) = M(d1, nxt, 1, nzt);
    M(lam, nxt + 1, nyt + 1, 0) = M(lam, nxt, nyt, 1); M(mu, nxt + 1, nyt + 1, 0) = M(mu, nxt, nyt, 1); M(d1, nxt + 1, nyt + 1, 0) = M(d1, nxt, nyt, 1);
    M(lam, 0, nyt + 1, nzt + 1) = M(lam, 1, nyt, nzt); M(mu, 0, nyt + 1, nzt + 1) = M(mu, 1, nyt, nzt); M(d1, 0, nyt + 1, nzt + 1) = M(d1, 1, nyt, nzt);
    M(lam, nxt + 1, nyt + 1, nzt + 1) = M(lam, nxt, nyt, nzt); M(mu, nxt + 1, nyt + 1, nzt + 1) = M(mu, nxt, nyt, nzt); M(d1, nxt + 1, nyt + 1, nzt + 1) = M(d1, nxt, nyt, nzt);
    /* afsmedia (structure.f:690-704): plane above the free surface */
    for (int i = 1; i <= nxt; i++)
        for (int j = 1; j <= nyt; j++) {
            M(d1, i, j, nzt + 1) = M(d1, i, j, nzt);
            M(mu, i, j, nzt + 1) = M(mu, i, j, nzt);
            M(lam, i, j, nzt + 1) = M(lam, i, j, nzt);
            if (h->p.nve == 1) {
                M(h->f[F_QP], i, j, nzt + 1) = M(h->f[F_QP], i, j, nzt);
                M(h->f[F_QS], i, j, nzt + 1) = M(h->f[F_QS], i, j, nzt);
            }
        }
#undef M
}

/* media: float32 [z][y][x][nvar], z = 0 at the free surface (file layout of
 * structure.f:142-173).  Ignored when mediastart == 0. */
int orc_set_media(orc_t *h, const float *media)
{
    const orc_params *p = &h->p;
    real pi = (real)4. * r_atan((real)1.);
    real taumax, taumin;
    if (p->mediastart == 0) {
        /* inihomo (structure.f:709-765) */
        taumax = (real)1. / ((real)2 * pi * (real)p->fl);
        taumin = (real)1. / ((real)2 * pi * (real)p->fh);
        float vp, vs, dd;
        if (p->idyna == 1) { vp = 6000.f; vs = 3464.f; dd = 2670.f; }
        else { vp = 4800.f; vs = 2800.f; dd = 2500.f; }
        h->vpe[0] = h->vpe[1] = vp; h->vse[0] = h->vse[1] = vs; h->dde[0] = h->dde[1] = dd;
        for (int k = 0; k <= p->nz + 1; k++)
            for (int j = 0; j <= p->ny + 1; j++)
                for (int i = 0; i <= p->nx + 1; i++) {
                    size_t c = IDX(h, i, j, k);
                    real rvp = vp, rvs = vs, rdd = dd;
                    h->f[F_LAM][c] = (real)1. / (rdd * (rvp * rvp - (real)2. * rvs * rvs));
                    h->f[F_MU][c] = (real)1. / (rdd * rvs * rvs);
                    h->f[F_D1][c] = rdd;
                }
        if (p->nve == 1) orc_tausub(h, taumin, taumax);
        return 0;
    }
    int var_offset = 0, act_nvar = 3;
    if (p->nvar == 8) { var_offset = 3; act_nvar = 5; }
    else if (p->nvar == 5) { var_offset = 0; act_nvar = 5; }
    else if (p->nvar != 3) return -1;
    (void)act_nvar;
    real w0 = (real)2 * pi * (real)p->fp;
    real ww1 = (real)2 * pi * (real)p->fl;
    real w2 = (real)2 * pi * (real)p->fh;
    taumax = (real)1. / ww1;
    taumin = (real)1. / w2;
    real tmp1 = (real)2. / pi * (r_log(taumax / taumin));
    real tmp2 = (real)2. / pi * r_log(w0 * taumin);
    real lw = r_log(w2 / w0);
    float vpe0 = 99999.f, vpe1 = 0.f, vse0 = 99999.f, vse1 = 0.f, dde0 = 99999.f, dde1 = 0.f;
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    for (int kf = 1; kf <= nz; kf++)        /* Fortran tmp index k; file z = kf-1 */
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) {
                const float *rec = media + (((size_t)(kf - 1) * ny + (j - 1)) * nx + (i - 1)) * p->nvar + var_offset;
                real vp = (real)rec[0], vs = (real)rec[1], dd = (real)rec[2];
                real pq = 0, sq = 0;
                if (p->nvar > 3) { pq = (real)rec[3]; sq = (real)rec[4]; }
                if (p->nvar == 3) { sq = (real)0.05 * vs; pq = (real)2.0 * sq; }
                if (p->socalq == 1) {
                    vs = vs * ((real)1 + (lw) / (pi * sq));
                    vp = vp * ((real)1 + (lw) / (pi * pq));
                    real vpvs = vp / vs;
                    if (vpvs < (real)1.45) vs = vp / (real)1.45;
                }
                int k = nz + 1 - kf;
                size_t c = IDX(h, i, j, k);
                h->f[F_MU][c] = (real)1. / (dd * vs * vs);
                h->f[F_LAM][c] = (real)1. / (dd * (vp * vp - (real)2. * vs * vs));
                h->f[F_D1][c] = dd;
                if (p->nve == 1) {
                    real qpinv, qsinv;
                    if (pq <= (real)0.0) { qpinv = 0; qsinv = 0; }
                    else { qpinv = (real)1. / pq; qsinv = (real)1. / sq; }
                    h->f[F_QP][c] = tmp1 * qpinv / ((real)1.0 - tmp2 * qpinv);
                    h->f[F_QS][c] = tmp1 * qsinv / ((real)1.0 - tmp2 * qsinv);
                }
                float fvs = (float)vs, fvp = (float)vp, fdd = (float)dd;
                if (fvs < vse0) vse0 = fvs;
                if (fvs > vse1) vse1 = fvs;
                if (fvp < vpe0) vpe0 = fvp;
                if (fvp > vpe1) vpe1 = fvp;
                if (fdd < dde0) dde0 = fdd;
                if (fdd > dde1) dde1 = fdd;
            }
    h->vpe[0] = vpe0; h->vpe[1] = vpe1; h->vse[0] = vse0; h->vse[1] = vse1; h->dde[0] = dde0; h->dde[1] = dde1;
    orc_padmedia(h);
    if (p->nve == 1) orc_tausub(h, taumin, taumax);
    return 0;
}

void orc_get_extremes(const orc_t *h, float *out6)
{
    out6[0] = h->vpe[0]; out6[1] = h->vpe[1];
    out6[2] = h->vse[0]; out6[3] = h->vse[1];
    out6[4] = h->dde[0]; out6[5] = h->dde[1];
}

/* ------------------------------------------------------------------ */
/* source (source.f:170-198, 378-437) and SGT points (station.f:31-80) */
/* ------------------------------------------------------------------ */

/* xyz: [nsrc][3] 1-based x, y, z with z = 1 at the free surface.
 * stf: [nsrc][nst][6] columns axx ayy azz axz ayz axy. */
int orc_set_source(orc_t *h, int nsrc, const int *xyz, const float *stf)
{
    const orc_params *p = &h->p;
    for (int s = 0; s < nsrc; s++) {
        if (xyz[3 * s] < 1 || xyz[3 * s] > p->nx) return -1;
        if (xyz[3 * s + 1] < 1 || xyz[3 * s + 1] > p->ny) return -1;
        if (xyz[3 * s + 2] < 1 || xyz[3 * s + 2] > p->nz) return -1;
    }
    free(h->src); free(h->stf);
    h->nsrc = nsrc;
    h->src = malloc(sizeof(int) * 3 * (size_t)(nsrc > 0 ? nsrc : 1));
    h->stf = malloc(sizeof(float) * 6 * (size_t)p->nst * (size_t)(nsrc > 0 ? nsrc : 1));
    for (int s = 0; s < nsrc; s++) {
        h->src[3 * s] = xyz[3 * s];
        h->src[3 * s + 1] = xyz[3 * s + 1];
        h->src[3 * s + 2] = p->nz + 1 - xyz[3 * s + 2];
    }
    memcpy(h->stf, stf, sizeof(float) * 6 * (size_t)p->nst * (size_t)nsrc);
    return 0;
}

/* pts: [npts][3] cordfile x y z (1-based, z = 1 at the free surface). */
int orc_set_points(orc_t *h, int npts, const int *xyz)
{
    const orc_params *p = &h->p;
    for (int n = 0; n < npts; n++) {
        if (xyz[3 * n] < 1 || xyz[3 * n] > p->nx) return -1;
        if (xyz[3 * n + 1] < 1 || xyz[3 * n + 1] > p->ny) return -1;
        if (xyz[3 * n + 2] < 1 || xyz[3 * n + 2] > p->nz) return -1;
    }
    free(h->pts); free(h->sg); free(h->sgt_buf); free(h->sgt_file);
    h->npts = npts;
    h->pts = malloc(sizeof(int) * 3 * (size_t)(npts > 0 ? npts : 1));
    h->sg = malloc(sizeof(real) * 3 * (size_t)(npts > 0 ? npts : 1));
    for (int n = 0; n < npts; n++) {
        h->pts[3 * n] = xyz[3 * n];
        h->pts[3 * n + 1] = xyz[3 * n + 1];
        h->pts[3 * n + 2] = p->nz - xyz[3 * n + 2] + 1;
    }
    h->sgt_buf = calloc((size_t)(npts > 0 ? npts : 1) * 6 * (size_t)p->write_step, sizeof(float));
    h->sgt_count = 0;
    h->sgt_file_floats = (int64_t)npts * 6 * h->nt_file;
    int nsamp = p->nt / p->ntiskp_sgt;
    int nchunk = nsamp / p->write_step;
    if (npts > 0 && nchunk > 0) {
        int64_t last = (int64_t)(npts - 1) * 6 * h->nt_file + (int64_t)5 * h->nt_file
                     + (int64_t)(nchunk - 1) * p->write_step + p->write_step;
        if (last > h->sgt_file_floats) h->sgt_file_floats = last;
    }
    h->sgt_file = calloc((size_t)(h->sgt_file_floats > 0 ? h->sgt_file_floats : 1), sizeof(float));
    return 0;
}

int64_t orc_sgt_file_floats(const orc_t *h) { return h->sgt_file_floats; }

/* sg1, sg2, sg3 at each point (pmcl3d.f:1166-1168); compliances -> moduli */
static void orc_sgt_coeffs(orc_t *h)
{
    for (int n = 0; n < h->npts; n++) {
        size_t c = IDX(h, h->pts[3 * n], h->pts[3 * n + 1], h->pts[3 * n + 2]);
        real lam = h->f[F_LAM][c], mu = h->f[F_MU][c];
        h->sg[3 * n] = ((real)1. / lam + (real)1. / mu) / ((real)1. / mu * ((real)3.0 / lam + (real)2.0 / mu));
        h->sg[3 * n + 1] = -((real)1. / lam / ((real)2.0 / mu * ((real)3.0 / lam + (real)2.0 / mu)));
        h->sg[3 * n + 2] = mu;
    }
}

/* ------------------------------------------------------------------ */
/* time step                                                           */
/* ------------------------------------------------------------------ */

static void orc_dvelc(orc_t *h)
{
    /* operator.f:92-244 */
    const orc_params *p = &h->p;
    const real dth = (real)p->dt / (real)p->dh;
    const real c1 = (real)9. / (real)8.;
    const real c2 = -((real)1. / (real)24.);
    real *u1 = h->f[F_U1], *v1 = h->f[F_V1], *w1 = h->f[F_W1];
    const real *xx = h->f[F_XX], *yy = h->f[F_YY], *zz = h->f[F_ZZ];
    const real *xy = h->f[F_XY], *xz = h->f[F_XZ], *yz = h->f[F_YZ], *d1 = h->f[F_D1];
    const long sx = 1, sy = h->sx, sz = (long)h->sx * h->sy;
    #pragma omp parallel for schedule(static)
    for (int k = h->box[4]; k <= h->box[5]; k++)
        for (int j = h->box[2]; j <= h->box[3]; j++)
            for (int i = h->box[0]; i <= h->box[1]; i++) {
                const long c = (long)IDX(h, i, j, k);
                real d;
                d = (real)0.25 * ((d1[c] + d1[c - sy]) + (d1[c - sz] + d1[c - sy - sz]));
                u1[c] = u1[c] + (dth / d) * (
                    c1 * (xx[c] - xx[c - sx]) +
                    c2 * (xx[c + sx] - xx[c - 2 * sx]) +
                    c1 * (xy[c] - xy[c - sy]) +
                    c2 * (xy[c + sy] - xy[c - 2 * sy]) +
                    c1 * (xz[c] - xz[c - sz]) +
                    c2 * (xz[c + sz] - xz[c - 2 * sz]));
                d = (real)0.25 * ((d1[c] + d1[c + sx]) + (d1[c - sz] + d1[c + sx - sz]));
                v1[c] = v1[c] + (dth / d) * (
                    c1 * (xy[c + sx] - xy[c]) +
                    c2 * (xy[c + 2 * sx] - xy[c - sx]) +
                    c1 * (yy[c + sy] - yy[c]) +
                    c2 * (yy[c + 2 * sy] - yy[c - sy]) +
                    c1 * (yz[c] - yz[c - sz]) +
                    c2 * (yz[c + sz] - yz[c - 2 * sz]));
                d = (real)0.25 * ((d1[c] + d1[c + sx]) + (d1[c - sy] + d1[c + sx - sy]));
                w1[c] = w1[c] + (dth / d) * (
                    c1 * (xz[c + sx] - xz[c]) +
                    c2 * (xz[c + 2 * sx] - xz[c - sx]) +
                    c1 * (yz[c] - yz[c - sy]) +
                    c2 * (yz[c + sy] - yz[c - 2 * sy]) +
                    c1 * (zz[c + sz] - zz[c]) +
                    c2 * (zz[c + 2 * sz] - zz[c - sz]));
            }
    (void)sx;
}

static void orc_addcrj(orc_t *h, int first, int last)
{
    /* cerjan.f:249-330: fields first..last multiplied by the zone factor */
    const orc_params *p = &h->p;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= p->nz; k++)
        for (int j = 1; j <= p->ny; j++)
            for (int i = 1; i <= p->nx; i++) {
                int inzone = (i <= p->nd) || (i >= p->nx - p->nd + 1) || (j <= p->nd) ||
                             (j >= p->ny - p->nd + 1) || (k <= p->nd);
                if (!inzone) continue;
                real dcrj = (h->cx[i] * h->cy[j]) * h->cz[k];
                size_t c = IDX(h, i, j, k);
                for (int q = first; q <= last; q++) h->f[q][c] = h->f[q][c] * dcrj;
            }
}

static void orc_fvel(orc_t *h)
{
    /* fvelxy (operator.f:246-272) then fvelz (operator.f:274-306) */
    const orc_params *p = &h->p;
    const int nzt = p->nz;
    real *u1 = h->f[F_U1], *v1 = h->f[F_V1], *w1 = h->f[F_W1];
    const real *lam = h->f[F_LAM], *mu = h->f[F_MU];
    for (int j = 1; j <= p->ny; j++)
        for (int i = 1; i <= p->nx; i++)
            u1[IDX(h, i, j, nzt + 1)] = u1[IDX(h, i, j, nzt)] - (w1[IDX(h, i, j, nzt)] - w1[IDX(h, i - 1, j, nzt)]);
    for (int j = 1; j <= p->ny; j++)
        for (int i = 1; i <= p->nx; i++)
            v1[IDX(h, i, j, nzt + 1)] = v1[IDX(h, i, j, nzt)] - (w1[IDX(h, i, j + 1, nzt)] - w1[IDX(h, i, j, nzt)]);
    for (int j = 1; j <= p->ny; j++)
        for (int i = 1; i <= p->nx; i++) {
            real xl = (real)1. / lam[IDX(h, i, j, nzt)];
            real xl2m = (real)2. / mu[IDX(h, i, j, nzt)] + xl;
            w1[IDX(h, i, j, nzt + 1)] = w1[IDX(h, i, j, nzt - 1)] - (xl / xl2m) * (
                (u1[IDX(h, i + 1, j, nzt + 1)] - u1[IDX(h, i, j, nzt + 1)]) +
                (u1[IDX(h, i + 1, j, nzt)] - u1[IDX(h, i, j, nzt)]) +
                (v1[IDX(h, i, j, nzt + 1)] - v1[IDX(h, i, j - 1, nzt + 1)]) +
                (v1[IDX(h, i, j, nzt)] - v1[IDX(h, i, j - 1, nzt)]));
        }
}

/* 32 random bits for stochastic rounding of memory variable pair `pair`
 * (0: r1 r2, 1: r3 r4, 2: r5 r6; low half for the first) of cell (i,j,k) at
 * step `step`: an integer mix of the three counters (multiply-xorshift
 * rounds), the same on the host and the device. */
static inline uint32_t orc_sr_bits(int i, int j, int k, int nx, int ny, int step, int pair)
{
    uint32_t h = (((uint32_t)k * (uint32_t)ny + (uint32_t)j) * (uint32_t)nx + (uint32_t)i) * 0x9E3779B1u;
    h += (uint32_t)step * 0x85EBCA77u + (uint32_t)pair * 0xC2B2AE3Du;
    h ^= h >> 15; h *= 0x2C1B3C6Du;
    h ^= h >> 12; h *= 0x297A2D39u;
    h ^= h >> 15;
    return h;
}

static inline float orc_bits_f(uint32_t b) { float v; memcpy(&v, &b, 4); return v; }
static inline uint32_t orc_f_bits(float v) { uint32_t b; memcpy(&b, &v, 4); return b; }

/* float rounded to `keep` mantissa bits (bf16 keeps 7, binary16 10; the
 * exponent range of float is kept): nearest even, or stochastic with the
 * low bits of `rnd` (adding a uniform integer below one unit of the kept
 * last place to the magnitude, then truncating, rounds away from zero with
 * the probability of the dropped fraction) */
static inline float orc_round_mant(float v, int keep, int stochastic, uint32_t rnd)
{
    const int drop = 23 - keep;
    const uint32_t mask = (1u << drop) - 1u;
    uint32_t b = orc_f_bits(v);
    if ((b & 0x7fffffffu) >= 0x7f800000u) return v;
    if (stochastic) b += rnd & mask;
    else b += (mask >> 1) + ((b >> drop) & 1u);
    return orc_bits_f(b & ~mask);
}

/* Block floating point of n values sharing one exponent (the storage
 * AWP_PREC_BFP of the device steppers; ORC_RS_BFP33 is that mode, two groups
 * of three): E = the float exponent field of the largest magnitude; with
 * E >= 15 each value is stored as the integer nearest (ties to even) to
 * v * 2^(141 - E) clamped to [-32767, 32767] (the magnitude is below 2^15),
 * read back as m * 2^(E - 141); E < 15 stores zeros.  Both scalings are
 * exact; the integer conversion makes a value that rounds to 0 a +0. */
static inline void orc_bfp(float *v, int n)
{
    float mx = 0.f;
    for (int a = 0; a < n; a++) mx = fmaxf(fabsf(v[a]), mx);
    const uint32_t e = orc_f_bits(mx) >> 23;
    if (e < 15u) {
        for (int a = 0; a < n; a++) v[a] = 0.f;
        return;
    }
    const float up = orc_bits_f((268u - e) << 23), down = orc_bits_f((e - 14u) << 23);
    for (int a = 0; a < n; a++) {
        const long m = lrintf(fminf(fmaxf(v[a] * up, -32767.f), 32767.f));
        v[a] = (float)m * down;
    }
}

static inline real orc_rstore(int mode, real v, uint32_t rnd)
{
#if ORC_IS_DOUBLE
    (void)mode; (void)rnd;
    return v;
#else
    switch (mode) {
    case ORC_RS_BF16_RN: return orc_round_mant(v, 7, 0, 0);
    case ORC_RS_BF16_SR: return orc_round_mant(v, 7, 1, rnd);
    case ORC_RS_F16M_RN: return orc_round_mant(v, 10, 0, 0);
    case ORC_RS_F16M_SR: return orc_round_mant(v, 10, 1, rnd);
    default: return v;
    }
#endif
}

static void orc_dstrqc(orc_t *h)
{
    /* viscoop.f:49-191 (allq over the whole subdomain) */
    const orc_params *p = &h->p;
    const real dh1 = (real)1. / (real)p->dh;
    const real dth = (real)p->dt / (real)p->dh;
    const real dt = (real)p->dt;
    const real c1 = (real)9. / (real)8.;
    const real c2 = -((real)1. / (real)24.);
    const real *u1 = h->f[F_U1], *v1 = h->f[F_V1], *w1 = h->f[F_W1];
    real *xx = h->f[F_XX], *yy = h->f[F_YY], *zz = h->f[F_ZZ];
    real *xy = h->f[F_XY], *xz = h->f[F_XZ], *yz = h->f[F_YZ];
    real *r1 = h->f[F_R1], *r2 = h->f[F_R2], *r3 = h->f[F_R3];
    real *r4 = h->f[F_R4], *r5 = h->f[F_R5], *r6 = h->f[F_R6];
    const real *lam = h->f[F_LAM], *mu = h->f[F_MU], *qp = h->f[F_QP], *qs = h->f[F_QS];
    const long sx = 1, sy = h->sx, sz = (long)h->sx * h->sy;
    const int nz = p->nz;
    const int rs = p->rstore, step = h->cur;
    #pragma omp parallel for schedule(static)
    for (int k = h->box[4]; k <= h->box[5]; k++) {
        const int itz = ((nz + 1) - k) % 2;          /* mod(...,2)+1, 0-based */
        for (int j = h->box[2]; j <= h->box[3]; j++) {
            const int ity = j % 2;
            for (int i = h->box[0]; i <= h->box[1]; i++) {
                const int itx = i % 2;
                const real vx1 = h->tau1[itz][ity][itx];
                const real vx2 = h->tau2[itz][ity][itx];
                const long c = (long)IDX(h, i, j, k);
                real xl = (real)8. / (lam[c] + lam[c + sx] + lam[c - sy] + lam[c + sx - sy] +
                                      lam[c - sz] + lam[c + sx - sz] + lam[c - sy - sz] + lam[c + sx - sy - sz]);
                real xm = (real)8. / (mu[c] + mu[c + sx] + mu[c - sy] + mu[c + sx - sy] +
                                      mu[c - sz] + mu[c + sx - sz] + mu[c - sy - sz] + mu[c + sx - sy - sz]);
                xl = xl + (real)2. * xm;
                real qpa = (real)0.125 * (qp[c] + qp[c + sx] + qp[c - sy] + qp[c + sx - sy] +
                                          qp[c - sz] + qp[c + sx - sz] + qp[c - sy - sz] + qp[c + sx - sy - sz]);
                real qsa = (real)0.125 * (qs[c] + qs[c + sx] + qs[c - sy] + qs[c + sx - sy] +
                                          qs[c - sz] + qs[c + sx - sz] + qs[c - sy - sz] + qs[c + sx - sy - sz]);
                real vt1 = c1 * (u1[c + sx] - u1[c]) + c2 * (u1[c + 2 * sx] - u1[c - sx]);
                real vt2 = c1 * (v1[c] - v1[c - sy]) + c2 * (v1[c + sy] - v1[c - 2 * sy]);
                real vt3 = c1 * (w1[c] - w1[c - sz]) + c2 * (w1[c + sz] - w1[c - 2 * sz]);
                real vt4 = c1 * (u1[c + sy] - u1[c]) + c2 * (u1[c + 2 * sy] - u1[c - sy]) +
                           c1 * (v1[c] - v1[c - sx]) + c2 * (v1[c + sx] - v1[c - 2 * sx]);
                real vt5 = c1 * (u1[c + sz] - u1[c]) + c2 * (u1[c + 2 * sz] - u1[c - sz]) +
                           c1 * (w1[c] - w1[c - sx]) + c2 * (w1[c + sx] - w1[c - 2 * sx]);
                real vt6 = c1 * (v1[c + sz] - v1[c]) + c2 * (v1[c + 2 * sz] - v1[c - sz]);
                real vt7 = c1 * (w1[c + sy] - w1[c]) + c2 * (w1[c + 2 * sy] - w1[c - sy]);

                real vh1 = -(xm * qsa);
                real vtmp = xl * (vt1 + vt2 + vt3);
                real va1 = -(qpa * xl * dh1 * (vt1 + vt2 + vt3) / (real)2.);

                xx[c] = xx[c] + dth * (vtmp - (real)2. * xm * (vt2 + vt3)) + dt * r1[c];
                yy[c] = yy[c] + dth * (vtmp - (real)2. * xm * (vt1 + vt3)) + dt * r2[c];
                zz[c] = zz[c] + dth * (vtmp - (real)2. * xm * (vt1 + vt2)) + dt * r3[c];

                real vxmu, vaas;
                vxmu = (real)2. / (mu[c] + mu[c - sz]);
                vaas = (real)0.5 * (qs[c] + qs[c - sz]);
                real vh2_r4 = -(vaas * vxmu / (real)2.);
                xy[c] = xy[c] + vxmu * dth * vt4 + dt * r4[c];
                vxmu = (real)2. / (mu[c] + mu[c - sy]);
                vaas = (real)0.5 * (qs[c] + qs[c - sy]);
                real vh2_r5 = -(vaas * vxmu / (real)2.);
                xz[c] = xz[c] + vxmu * dth * vt5 + dt * r5[c];
                vxmu = (real)2. / (mu[c] + mu[c + sx]);
                vaas = (real)0.5 * (qs[c] + qs[c + sx]);
                real vh2_r6 = -(vaas * vxmu / (real)2.);
                yz[c] = yz[c] + vxmu * (dth * vt6 + dth * vt7) + dt * r6[c];

                const real n1 = (vx2 * r1[c] - vh1 * (vt2 + vt3) * dh1 + va1) * vx1;
                const real n2 = (vx2 * r2[c] - vh1 * (vt1 + vt3) * dh1 + va1) * vx1;
                const real n3 = (vx2 * r3[c] - vh1 * (vt1 + vt2) * dh1 + va1) * vx1;
                const real n4 = (vx2 * r4[c] + vh2_r4 * dh1 * vt4) * vx1;
                const real n5 = (vx2 * r5[c] + vh2_r5 * dh1 * vt5) * vx1;
                const real n6 = (vx2 * r6[c] + vh2_r6 * dh1 * (vt6 + vt7)) * vx1;

                xx[c] = xx[c] + dt * n1;
                yy[c] = yy[c] + dt * n2;
                zz[c] = zz[c] + dt * n3;
                xy[c] = xy[c] + dt * n4;
                xz[c] = xz[c] + dt * n5;
                yz[c] = yz[c] + dt * n6;
                if (rs == ORC_RS_F32) {
                    r1[c] = n1; r2[c] = n2; r3[c] = n3; r4[c] = n4; r5[c] = n5; r6[c] = n6;
                } else if (rs == ORC_RS_BFP6 || rs == ORC_RS_BFP33) {
#if ORC_IS_DOUBLE
                    r1[c] = n1; r2[c] = n2; r3[c] = n3; r4[c] = n4; r5[c] = n5; r6[c] = n6;
#else
                    float v[6] = {n1, n2, n3, n4, n5, n6};
                    if (rs == ORC_RS_BFP6) orc_bfp(v, 6);
                    else { orc_bfp(v, 3); orc_bfp(v + 3, 3); }
                    r1[c] = v[0]; r2[c] = v[1]; r3[c] = v[2]; r4[c] = v[3]; r5[c] = v[4]; r6[c] = v[5];
#endif
                } else {
                    const uint32_t b0 = orc_sr_bits(i, j, k, p->nx, p->ny, step, 0);
                    const uint32_t b1 = orc_sr_bits(i, j, k, p->nx, p->ny, step, 1);
                    const uint32_t b2 = orc_sr_bits(i, j, k, p->nx, p->ny, step, 2);
                    r1[c] = orc_rstore(rs, n1, b0); r2[c] = orc_rstore(rs, n2, b0 >> 16);
                    r3[c] = orc_rstore(rs, n3, b1); r4[c] = orc_rstore(rs, n4, b1 >> 16);
                    r5[c] = orc_rstore(rs, n5, b2); r6[c] = orc_rstore(rs, n6, b2 >> 16);
                }
            }
        }
    }
}

static void orc_dstrc(orc_t *h)
{
    /* elastic stress update, operator.f:348-571 (nve = 0) */
    const orc_params *p = &h->p;
    const real dth = (real)p->dt / (real)p->dh;
    const real c1 = (real)9. / (real)8.;
    const real c2 = -((real)1. / (real)24.);
    const real *u1 = h->f[F_U1], *v1 = h->f[F_V1], *w1 = h->f[F_W1];
    real *xx = h->f[F_XX], *yy = h->f[F_YY], *zz = h->f[F_ZZ];
    real *xy = h->f[F_XY], *xz = h->f[F_XZ], *yz = h->f[F_YZ];
    const real *lam = h->f[F_LAM], *mu = h->f[F_MU];
    const long sx = 1, sy = h->sx, sz = (long)h->sx * h->sy;
    #pragma omp parallel for schedule(static)
    for (int k = h->box[4]; k <= h->box[5]; k++)
        for (int j = h->box[2]; j <= h->box[3]; j++)
            for (int i = h->box[0]; i <= h->box[1]; i++) {
                const long c = (long)IDX(h, i, j, k);
                real xl = (real)8. / (lam[c] + lam[c + sx] + lam[c - sy] + lam[c + sx - sy] +
                                      lam[c - sz] + lam[c + sx - sz] + lam[c - sy - sz] + lam[c + sx - sy - sz]);
                real xm = (real)8. / (mu[c] + mu[c + sx] + mu[c - sy] + mu[c + sx - sy] +
                                      mu[c - sz] + mu[c + sx - sz] + mu[c - sy - sz] + mu[c + sx - sy - sz]);
                real a = xl + (real)2. * xm;
                real b = xl;
                /* individual difference terms; the sums keep the Fortran
                 * left-to-right grouping of operator.f:389-426 */
                real u_a = c1 * (u1[c + sx] - u1[c]), u_b = c2 * (u1[c + 2 * sx] - u1[c - sx]);
                real v_a = c1 * (v1[c] - v1[c - sy]), v_b = c2 * (v1[c + sy] - v1[c - 2 * sy]);
                real w_a = c1 * (w1[c] - w1[c - sz]), w_b = c2 * (w1[c + sz] - w1[c - 2 * sz]);
                xx[c] = xx[c] + dth * a * (u_a + u_b) + dth * b * (v_a + v_b + w_a + w_b);
                yy[c] = yy[c] + dth * a * (v_a + v_b) + dth * b * (u_a + u_b + w_a + w_b);
                zz[c] = zz[c] + dth * a * (w_a + w_b) + dth * b * (u_a + u_b + v_a + v_b);
                real xmu;
                xmu = (real)2. / (mu[c] + mu[c - sz]);
                xy[c] = xy[c] + dth * xmu * (c1 * (u1[c + sy] - u1[c]) + c2 * (u1[c + 2 * sy] - u1[c - sy]) +
                                             c1 * (v1[c] - v1[c - sx]) + c2 * (v1[c + sx] - v1[c - 2 * sx]));
                xmu = (real)2. / (mu[c] + mu[c - sy]);
                xz[c] = xz[c] + dth * xmu * (c1 * (u1[c + sz] - u1[c]) + c2 * (u1[c + 2 * sz] - u1[c - sz]) +
                                             c1 * (w1[c] - w1[c - sx]) + c2 * (w1[c + sx] - w1[c - 2 * sx]));
                xmu = (real)2. / (mu[c] + mu[c + sx]);
                yz[c] = yz[c] + dth * xmu * (c1 * (v1[c + sz] - v1[c]) + c2 * (v1[c + 2 * sz] - v1[c - sz]) +
                                             c1 * (w1[c + sy] - w1[c]) + c2 * (w1[c + 2 * sy] - w1[c - sy]));
            }
}

static void orc_fstr(orc_t *h)
{
    /* operator.f:575-612 */
    const int nzt = h->p.nz;
    real *zz = h->f[F_ZZ], *xz = h->f[F_XZ], *yz = h->f[F_YZ];
    for (int j = 1; j <= h->p.ny; j++)
        for (int i = 1; i <= h->p.nx; i++) {
            zz[IDX(h, i, j, nzt + 1)] = -zz[IDX(h, i, j, nzt)];
            zz[IDX(h, i, j, nzt + 2)] = -zz[IDX(h, i, j, nzt - 1)];
            xz[IDX(h, i, j, nzt + 1)] = -xz[IDX(h, i, j, nzt - 1)];
            xz[IDX(h, i, j, nzt + 2)] = -xz[IDX(h, i, j, nzt - 2)];
            yz[IDX(h, i, j, nzt + 1)] = -yz[IDX(h, i, j, nzt - 1)];
            yz[IDX(h, i, j, nzt + 2)] = -yz[IDX(h, i, j, nzt - 2)];
            xz[IDX(h, i, j, nzt)] = 0;
            yz[IDX(h, i, j, nzt)] = 0;
        }
}

static void orc_addsrc(orc_t *h, int it)
{
    /* source.f:812-913, sample it (1-based) */
    const orc_params *p = &h->p;
    if (it > p->nst) return;
    const int k = it;
    const real dx = (real)p->dh;
    const real vtst = (real)p->dt / (dx * dx * dx);
    const real vtst1 = (real)1. / (dx * dx);
    const int nzt = p->nz;
    for (int s = 0; s < h->nsrc; s++) {
        const int i = h->src[3 * s], j = h->src[3 * s + 1], kk = h->src[3 * s + 2];
        const float *a = h->stf + ((size_t)s * p->nst + (size_t)(k - 1)) * 6;
        const real axx = a[0], ayy = a[1], azz = a[2], axz = a[3], ayz = a[4], axy = a[5];
        const size_t c = IDX(h, i, j, kk);
        real *F = NULL;
        switch (p->igreen) {
        case -1:
            h->f[F_XX][c] = h->f[F_XX][c] - vtst * axx;
            h->f[F_YY][c] = h->f[F_YY][c] - vtst * ayy;
            h->f[F_ZZ][c] = h->f[F_ZZ][c] - vtst * azz;
            h->f[F_XZ][c] = h->f[F_XZ][c] - vtst * axz;
            h->f[F_YZ][c] = h->f[F_YZ][c] - vtst * ayz;
            h->f[F_XY][c] = h->f[F_XY][c] - vtst * axy;
            break;
        case 1:
            h->f[F_U1][c] = h->f[F_U1][c] + axx * vtst / h->f[F_D1][c];
            break;
        case 2:
            h->f[F_V1][c] = h->f[F_V1][c] + ayy * vtst / h->f[F_D1][c];
            break;
        case 3:
            h->f[F_W1][c] = h->f[F_W1][c] + azz * vtst / h->f[F_D1][c];
            break;
        case -2:
            h->f[F_U1][c] = h->f[F_U1][c] + axx * vtst / h->f[F_D1][c];
            h->f[F_V1][c] = h->f[F_V1][c] + ayy * vtst / h->f[F_D1][c];
            h->f[F_W1][c] = h->f[F_W1][c] + azz * vtst / h->f[F_D1][c];
            break;
        case 4:
            F = h->f[F_XZ];
            F[IDX(h, i, j, nzt)] = axx * vtst1;
            F[IDX(h, i, j, nzt + 1)] = (real)2. * axx * vtst1 - F[IDX(h, i, j, nzt - 1)];
            F[IDX(h, i, j, nzt + 2)] = (real)2. * axx * vtst1 - F[IDX(h, i, j, nzt - 2)];
            break;
        case 5:
            F = h->f[F_YZ];
            F[IDX(h, i, j, nzt)] = ayy * vtst1;
            F[IDX(h, i, j, nzt + 1)] = (real)2. * ayy * vtst1 - F[IDX(h, i, j, nzt - 1)];
            F[IDX(h, i, j, nzt + 2)] = (real)2. * ayy * vtst1 - F[IDX(h, i, j, nzt - 2)];
            break;
        case 6:
            F = h->f[F_ZZ];
            F[IDX(h, i, j, nzt + 1)] = (real)2. * azz * vtst1 - F[IDX(h, i, j, nzt)];
            F[IDX(h, i, j, nzt + 2)] = (real)2. * azz * vtst1 - F[IDX(h, i, j, nzt - 1)];
            break;
        default:
            break;
        }
    }
}

static void orc_sgt_sample(orc_t *h, int it)
{
    /* pmcl3d.f:1537-1608 */
    const orc_params *p = &h->p;
    if (p->igreen == -1 || h->npts <= 0) return;
    int itk = p->ntiskp_sgt * (it / p->ntiskp_sgt);
    if (it != itk) return;
    const int ws = p->write_step;
    const int cnt = h->sgt_count;   /* 0-based sample slot */
    for (int n = 0; n < h->npts; n++) {
        size_t c = IDX(h, h->pts[3 * n], h->pts[3 * n + 1], h->pts[3 * n + 2]);
        real sg1 = h->sg[3 * n], sg2 = h->sg[3 * n + 1], sg3 = h->sg[3 * n + 2];
        real xx = h->f[F_XX][c], yy = h->f[F_YY][c], zz = h->f[F_ZZ][c];
        real xy = h->f[F_XY][c], xz = h->f[F_XZ][c], yz = h->f[F_YZ][c];
        float *b = h->sgt_buf + (size_t)n * 6 * ws;
        b[0 * ws + cnt] = (float)(sg1 * xx + sg2 * yy + sg2 * zz);
        b[1 * ws + cnt] = (float)(sg2 * xx + sg1 * yy + sg2 * zz);
        b[2 * ws + cnt] = (float)(sg2 * xx + sg2 * yy + sg1 * zz);
        b[3 * ws + cnt] = (float)(sg3 * xy);
        b[4 * ws + cnt] = (float)(sg3 * xz);
        b[5 * ws + cnt] = (float)(sg3 * yz);
    }
    h->sgt_count++;
    if (h->sgt_count == ws) {
        int64_t chunk = (it / p->ntiskp_sgt / ws) - 1;
        for (int n = 0; n < h->npts; n++)
            for (int q = 0; q < 6; q++) {
                int64_t off = (int64_t)n * 6 * h->nt_file + (int64_t)q * h->nt_file + chunk * ws;
                if (off < 0 || off + ws > h->sgt_file_floats) continue;
                memcpy(h->sgt_file + off, h->sgt_buf + ((size_t)n * 6 + q) * ws, sizeof(float) * ws);
            }
        h->sgt_count = 0;
    }
}

/* IFAULT=5 kinematic source, AWP-GPU-SGT/src/kernel_kp1_fix_havg_ifault5.cu:
 * 210-376 (compmt, brune, liu, gp10, addkinsrc_cu): after the stress update of
 * step it, every subfault whose rupture time has passed adds its moment rate
 * (slip x area x mu x slip-rate function) times the double-couple tensor of
 * its strike, dip and rake, in subfault order.  The FP32 build follows the
 * float / double evaluation points of the CUDA code with the C library's
 * sinf / cosf / expf / powf; the FP64 build evaluates everything in double. */
#if ORC_IS_DOUBLE
#define KSIN sin
#define KCOS cos
#define KEXP exp
#define KPOW pow
#else
#define KSIN sinf
#define KCOS cosf
#define KEXP expf
#define KPOW powf
#endif
static void orc_kin_mt(real str, real dip, real rake, real m[6])
{
    m[1] = -(KSIN(dip) * KCOS(rake) * KSIN(2. * str) + KSIN(2. * dip) * KSIN(rake) * KSIN(str) * KSIN(str));
    m[5] = KSIN(dip) * KCOS(rake) * KCOS(2. * str) + 0.5 * (KSIN(2. * dip) * KSIN(rake) * KSIN(2. * str));
    m[4] = (KCOS(dip) * KCOS(rake) * KCOS(str) + KCOS(2. * dip) * KSIN(rake) * KSIN(str));
    m[0] = KSIN(dip) * KCOS(rake) * KSIN(2. * str) - KSIN(2. * dip) * KSIN(rake) * KCOS(str) * KCOS(str);
    m[3] = (KCOS(dip) * KCOS(rake) * KSIN(str) - KCOS(2. * dip) * KSIN(rake) * KCOS(str));
    m[2] = KSIN(2. * dip) * KSIN(rake);
}

static real orc_kin_stf(int type, real rise, real t)
{
    const double pi = 3.14159265358979323846;
    if (type == 1) {
        const real freq = 1. / rise;
        const real omega = freq * pi * 2.;
        return t > 0. ? KPOW(omega, (real)2.) * t * KEXP(-omega * t) : (real)0.;
    }
    if (type != 2 && type != 3) return 0;
    const int rev = type == 3;
    const real tau1 = 0.13 * rise, tau2 = rise - tau1;
    const real cn = rev ? pi / (1.5 * pi * tau1 + 1.2 * tau1 + 0.2 * pi * tau2)
                        : pi / (1.4 * pi * tau1 + 1.2 * tau1 + 0.3 * pi * tau2);
    if (rev && t < 0.) return 0;
    if (t < tau1) return cn * (0.7 - 0.7 * KCOS(pi * t / tau1) + 0.6 * KSIN(0.5 * pi * t / tau1));
    if (t < 2 * tau1)
        return rev ? cn * (1.0 - 0.8 * KCOS(pi * t / tau1) + 0.2 * KCOS(pi * (t - tau1) / tau2))
                   : cn * (1.0 - 0.7 * KCOS(pi * t / tau1) + 0.3 * KCOS(pi * (t - tau1) / tau2));
    if (t < rise)
        return rev ? cn * (0.2 + 0.2 * KCOS(pi * (t - tau1) / tau2)) : cn * (0.3 + 0.3 * KCOS(pi * (t - tau1) / tau2));
    return 0;
}

static void orc_addkinsrc(orc_t *h, int it)
{
    const orc_params *p = &h->p;
    const double pi = 3.14159265358979323846;
    const real dx = (real)p->dh;
    const real vtst = (real)p->dt / (dx * dx * dx);
    const real atime = it * (real)p->dt;
    for (int s = 0; s < h->nsrc; s++) {
        const float *r0 = h->stf + (size_t)s * 12, *r1 = r0 + 6;
        if (!(atime > r0[2])) continue;
        real m[6];
        orc_kin_mt(r1[0] / 180. * pi, r1[1] / 180. * pi, r1[2] / 180. * pi, m);
        real stf = orc_kin_stf((int)r0[0], r0[3], atime - r0[2]);
        const size_t c = IDX(h, h->src[3 * s], h->src[3 * s + 1], h->src[3 * s + 2]);
        stf *= (real)r0[1] * (real)r0[4] / h->f[F_MU][c];
        stf *= vtst;
        h->f[F_XX][c] = h->f[F_XX][c] - stf * m[0];
        h->f[F_YY][c] = h->f[F_YY][c] - stf * m[1];
        h->f[F_ZZ][c] = h->f[F_ZZ][c] - stf * m[2];
        h->f[F_XZ][c] = h->f[F_XZ][c] - stf * m[3];
        h->f[F_YZ][c] = h->f[F_YZ][c] - stf * m[4];
        h->f[F_XY][c] = h->f[F_XY][c] - stf * m[5];
    }
}

#include "awp_oracle_pml.h"

/* one step in the order of pmcl3d.f:1234-1388: with NPC = 1 the interior
 * operators cover zone 18 and the PML routines the other zones, and no
 * Cerjan sponge is applied */
static void orc_one_step(orc_t *h, int it)
{
    const orc_params *p = &h->p;
    orc_dvelc(h);
    if (p->npc == 1) orc_pmlvel(h);
    else orc_addcrj(h, F_U1, F_W1);
    orc_fvel(h);
    if (p->nve == 1) orc_dstrqc(h); else orc_dstrc(h);
    if (p->npc == 1) orc_pmlstr(h);
    else orc_addcrj(h, F_XX, F_YZ);
    if (p->kinematic) {
        orc_fstr(h);
        orc_addkinsrc(h, it);
    } else if (p->igreen >= 4 && p->igreen <= 6) {
        orc_fstr(h);
        orc_addsrc(h, it + 1);
    } else {
        orc_addsrc(h, it + 1);
        orc_fstr(h);
    }
    /* CHKJ (pmcl3d.f:1478-1479): u1,v1,w1 at (nd+2,nd+2,nd+2) */
    int q = p->nd + 2;
    if (q <= p->nx && q <= p->ny && q <= p->nz && it >= 1 && it <= p->nt) {
        size_t c = IDX(h, q, q, q);
        h->chkj[3 * (size_t)(it - 1)] = (float)h->f[F_U1][c];
        h->chkj[3 * (size_t)(it - 1) + 1] = (float)h->f[F_V1][c];
        h->chkj[3 * (size_t)(it - 1) + 2] = (float)h->f[F_W1][c];
    }
    orc_sgt_sample(h, it);
}

/* Runs steps cur+1 .. cur+nsteps (capped at nt).  The first call performs
 * addsrc(1) (pmcl3d.f:966-988) and builds the SGT coefficients. */
int orc_run(orc_t *h, int nsteps)
{
    if (!h->started) {
        if (h->p.npc == 1) orc_inipml(h);   /* pmcl3d.f:928-929, after the media (vse) */
        orc_sgt_coeffs(h);
        if (!h->p.kinematic) orc_addsrc(h, 1);
        h->started = 1;
    }
    for (int s = 0; s < nsteps && h->cur < h->p.nt; s++) {
        h->cur++;
        orc_one_step(h, h->cur);
    }
    return h->cur;
}

void orc_get_sgt_file(const orc_t *h, float *out)
{
    memcpy(out, h->sgt_file, sizeof(float) * (size_t)h->sgt_file_floats);
}

void orc_get_chkj(const orc_t *h, float *out)
{
    memcpy(out, h->chkj, sizeof(float) * 3 * (size_t)h->p.nt);
}

/* Copies a field with its ghosts: out[(k+1)][(j+1)][(i+1)], extents
 * (nz+4, ny+4, nx+4), in the oracle's own precision. */
int orc_get_field(const orc_t *h, int fid, real *out)
{
    if (fid < 0 || fid >= F_NFIELDS) return -1;
    memcpy(out, h->f[fid], sizeof(real) * h->nvol);
    return 0;
}

int orc_set_field(orc_t *h, int fid, const real *in)
{
    if (fid < 0 || fid >= F_NFIELDS) return -1;
    memcpy(h->f[fid], in, sizeof(real) * h->nvol);
    return 0;
}

int orc_real_bytes(void) { return (int)sizeof(real); }

/* relaxation times [itz][ity][itx] (relax.f:15-36), as float */
void orc_get_tau(const orc_t *h, float *out8)
{
    for (int z = 0; z < 2; z++)
        for (int y = 0; y < 2; y++)
            for (int x = 0; x < 2; x++) out8[(z * 2 + y) * 2 + x] = (float)h->tau[z][y][x];
}

/* relaxation coefficients tau1 then tau2 of viscoop.f:79-88, each [itz][ity][itx]
 * with the 0-based parities itx = i mod 2, ity = j mod 2, itz = (nz+1-k) mod 2 */
void orc_get_tau12(const orc_t *h, float *out16)
{
    for (int z = 0; z < 2; z++)
        for (int y = 0; y < 2; y++)
            for (int x = 0; x < 2; x++) {
                out16[(z * 2 + y) * 2 + x] = (float)h->tau1[z][y][x];
                out16[8 + (z * 2 + y) * 2 + x] = (float)h->tau2[z][y][x];
            }
}

/* Cerjan factors cx[1..nx], cy[1..ny], cz[1..nz] (cerjan.f), as float */
void orc_get_sponge(const orc_t *h, float *cx, float *cy, float *cz)
{
    for (int i = 0; i < h->p.nx; i++) cx[i] = (float)h->cx[i + 1];
    for (int j = 0; j < h->p.ny; j++) cy[j] = (float)h->cy[j + 1];
    for (int k = 0; k < h->p.nz; k++) cz[k] = (float)h->cz[k + 1];
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
