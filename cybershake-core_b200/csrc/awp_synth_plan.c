/*
 * awp_synth_plan.c -- host set-up of the reciprocity synthesis: SRF reading,
 * the site / rupture point lookup in the SGT grid, and per term the scalars
 * the kernels need (mechanism coefficients, time shifts, scaled slip rates).
 *
 * Everything here is O(1) per (variation, point) and stays on the host so
 * that the float / double evaluation points are exactly those of the C
 * reference (a float argument of cos() is widened to double, as C does).
 * The file is compiled without FMA contraction.  The per-sample work (the
 * SGT combination and the convolution) runs in awp_synth.cu.
 */
#define _FILE_OFFSET_BITS 64
#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "awp_synth_internal.h"

void awp_set_error_text(const char *msg);

static awp_status perr(const char *msg)
{
    awp_set_error_text(msg);
    return AWP_ERR_PARAM;
}

/* ---- geoproj 1 (DirectSynth/src/jbsim/geoproj_subs.c) -------------------- */

#define GEO_RPERD 0.017453292     /* geoproj_subs.c:6  */
#define GEO_ERAD 6378.139         /* geoproj_subs.c:7  */

/* rotation of the model frame: y-axis azimuth alpha, origin (lon, lat)
 * (geoproj_subs.c:79-125) */
static void geo_matrices(awp_synth_geo *g, float alpha, float lon, float lat)
{
    const double rperd = GEO_RPERD;
    double arg = (double)alpha * rperd;
    const double ca = cos(arg), sa = sin(arg);
    arg = (double)(90.0 - lat) * rperd;
    const double ct = cos(arg), st = sin(arg);
    arg = (double)lon * rperd;
    const double cp = cos(arg), sp = sin(arg);
    double *a = g->amat;
    a[0] = ca * ct * cp + sa * sp;
    a[1] = sa * ct * cp - ca * sp;
    a[2] = st * cp;
    a[3] = ca * ct * sp - sa * cp;
    a[4] = sa * ct * sp + ca * cp;
    a[5] = st * sp;
    a[6] = -ca * st;
    a[7] = -sa * st;
    a[8] = ct;
    double det = a[0] * (a[4] * a[8] - a[7] * a[5]) - a[1] * (a[3] * a[8] - a[6] * a[5]) +
                 a[2] * (a[3] * a[7] - a[6] * a[4]);
    det = 1.0 / det;
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) g->ainv[3 * r + c] = det * a[3 * c + r];
}

/* set_geoproj for geoproj 1 (geoproj_subs.c:157-197) */
awp_status awp_synth_geo_init(const awp_sgtmaster *m, awp_synth_geo *g)
{
    if (m->geoproj != 1) return perr("synthesis: only geoproj 1 (great-circle arcs) SGT headers are supported");
    memset(g, 0, sizeof *g);
    g->erad = (float)GEO_ERAD;
    const float xlen = (float)(-2.0 * m->xshift);
    const float ylen = (float)(-2.0 * m->yshift);
    geo_matrices(g, m->modelrot, m->modellon, m->modellat);
    g->g0 = (double)(0.5 * ylen) / (double)g->erad;
    g->b0 = (double)(0.5 * xlen) / (double)g->erad;
    return AWP_OK;
}

/* longitude / latitude to model-frame km (geoproj_subs.c:10-77, gflag 1) */
static void geo_lonlat_to_xy(const awp_synth_geo *g, float lon, float lat, float *xf, float *yf)
{
    const double rperd = GEO_RPERD;
    double arg = lon * rperd;
    double cg = cos(arg), sg = sin(arg);
    arg = (90.0 - lat) * rperd;
    double cb = cos(arg), sb = sin(arg);
    const double xg = sb * cg, yg = sb * sg, zg = cb;
    const double *v = g->ainv;
    const double xp = xg * v[0] + yg * v[1] + zg * v[2];
    const double yp = xg * v[3] + yg * v[4] + zg * v[5];
    sg = xp / sqrt(1.0 - yp * yp);
    sb = yp / sqrt(1.0 - xp * xp);
    *xf = (float)((double)g->erad * (asin(sb) + g->b0));
    *yf = (float)((double)g->erad * (asin(sg) + g->g0));
}

/* grid location and index of a point (misc_subs.c:151-173) */
void awp_synth_get_indx(const awp_synth_geo *g, float lon, float lat, float dep, float h, awp_sgtindex *o)
{
    const double invh = 1.0 / (double)h;
    float xr, yr;
    geo_lonlat_to_xy(g, lon, lat, &xr, &yr);
    o->h = h;
    o->xsgt = (int)((double)xr * invh + 0.5);
    o->ysgt = (int)((double)yr * invh + 0.5);
    o->zsgt = (int)((double)dep * invh + 1.5);
    o->indx = (long long)o->xsgt * 1000000000000LL + (long long)o->ysgt * 1000000LL + (long long)o->zsgt;
}

/* ---- SGT points bracketing a rupture point (sgt3d_subs.c:751-961) ------- */

void awp_synth_find_sgt(const awp_sgtindex *ix, int np, const awp_sgtindex *eq, const awp_sgtindex *st,
                        awp_synth_bracket *o)
{
    /* exact match by bisection over the sorted index (sgt3d_subs.c:763-791) */
    int lo = 0, hi = np - 1, mid = (lo + hi) / 2;
    while (hi >= lo) {
        mid = (lo + hi) / 2;
        if (eq->indx > ix[mid].indx) lo = mid + 1;
        else if (eq->indx < ix[mid].indx) hi = mid - 1;
        else break;
    }
    memset(o, 0, sizeof *o);
    if (np > 0 && eq->indx == ix[mid].indx) {
        o->nsgt = 1;
        o->indx[0] = ix[mid].indx;
        o->wt[0] = 1.0f;
        o->pos[0] = mid;
        return;
    }
    /* nearest SGT point in each of the four quadrants of (horizontal range,
     * depth) relative to the site, inverse-distance weights (:803-936) */
    float delta[4] = {1.0e+15f, 1.0e+15f, 1.0e+15f, 1.0e+15f};
    int slot[4] = {-1, -1, -1, -1};
    float xx = (float)(eq->xsgt - st->xsgt), yy = (float)(eq->ysgt - st->ysgt);
    const float rexact = xx * xx + yy * yy;
    const float zexact = (float)(eq->zsgt - st->zsgt);
    for (int ip = 0; ip < np; ip++) {
        xx = (float)(ix[ip].xsgt - st->xsgt);
        yy = (float)(ix[ip].ysgt - st->ysgt);
        const float rng = xx * xx + yy * yy;
        const float zdp = (float)(ix[ip].zsgt - st->zsgt);
        xx = (float)(ix[ip].xsgt - eq->xsgt);
        yy = (float)(ix[ip].ysgt - eq->ysgt);
        const float zz = (float)(ix[ip].zsgt - eq->zsgt);
        const float del = xx * xx + yy * yy + zz * zz;
        const int q = (rng <= rexact ? 0 : 1) + (zdp <= zexact ? 0 : 2);
        if (slot[q] < 0) slot[q] = o->nsgt++;
        const int s = slot[q];
        if (del < delta[s]) {
            delta[s] = del;
            o->indx[s] = ix[ip].indx;
            o->wt[s] = (float)sqrt(del);
            o->pos[s] = ip;
        }
    }
    int zflag = -1;
    for (int i = 0; i < o->nsgt; i++)
        if (o->wt[i] == 0.0f) zflag = i;
    if (zflag >= 0) {
        for (int i = 0; i < o->nsgt; i++) o->wt[i] = 0.0f;
        o->wt[zflag] = 1.0f;
    } else {
        float sum = 0.0f;
        for (int i = 0; i < o->nsgt; i++) sum = (float)(sum + 1.0 / o->wt[i]);
        sum = (float)(1.0 / sum);
        for (int i = 0; i < o->nsgt; i++) o->wt[i] = sum / o->wt[i];
    }
}

/* ---- per-term scalars ---------------------------------------------------- */

/* cosine taper over the last SY_TAPLEN samples (sgt3d_subs.c:1201-1212):
 * fac[d] multiplies sample tapst + d, d = 1 .. SY_TAPLEN - 1 */
void awp_synth_taper(int nt, float *fac)
{
    const float pi = 3.141592654f, half = 0.5f, one = 1.0f;
    const float arg = pi / (float)SY_TAPLEN;
    (void)nt;
    fac[0] = 1.0f;
    for (int d = 1; d < SY_TAPLEN; d++) fac[d] = (float)(half * (one + cos(arg * (float)d)));
}

long long awp_synth_count_terms(const awp_srf_point *pts, int np)
{
    long long n = 0;
    for (int i = 0; i < np; i++) n += (pts[i].nt1 > 0) + (pts[i].nt2 > 0) + (pts[i].nt3 > 0);
    return n;
}

/* One variation, points ip0 .. ip1 - 1 in order: get_srfpars (srf_rupm.c:7-53), the
 * scalars of mech_sgt (sgt3d_subs.c:1260-1422), the time shifts of sum_sgt /
 * timeshift_sgt (:1121-1258) and the dt-scaled slip rates of srf_stf
 * (srf_rupm.c:55-153). */
awp_status awp_synth_plan_variation(const awp_synth_plan_ctx *cx, const awp_srf_point *pts, const float *pool,
                                    long long npool, int ip0, int ip1, awp_synth_gterm *gt, awp_synth_cterm *ct,
                                    float *stf, long long stf_base, long long *nterms, long long *nstf_used,
                                    long long *macs)
{
    const float rperd = 0.017453293f, two = 2.0f;
    const float ratio_tol = 0.00001f;
    const float ptol = (float)(1.0 + ratio_tol), mtol = (float)(1.0 - ratio_tol);
    long long nt_ = 0, ns = 0, mac = 0;
    for (int ip = ip0; ip < ip1; ip++) {
        const awp_srf_point *a = &pts[ip];
        const awp_synth_bracket *b = &cx->br[ip];
        int flag[3], nmech = 0;
        if (a->nt1 > 0) flag[nmech++] = 1;
        if (a->nt2 > 0) flag[nmech++] = 2;
        if (a->nt3 > 0) flag[nmech++] = 3;
        if (nmech == 0) continue;
        const float dr = cx->dtout / a->dt;
        if (dr > ptol || dr < mtol)
            return perr("synthesis: SRF sample interval differs from dtout (resampling is not supported)");
        const float scl = 1.0f * a->area;           /* slip_conv * area (jbsim3d.c:502) */

        /* sum_sgt: shifts shared by the point's slip components */
        float pbar = 0.0f, gft[4], t0[4], maxgft = -1.0e+15f, backt0 = 0.0f;
        for (int ig = 0; ig < b->nsgt; ig++) {
            const awp_sgtheader *h = &cx->hd[b->pos[ig]];
            pbar = (float)(pbar + sqrt(h->rho / h->mu));
        }
        pbar = pbar / (float)b->nsgt;
        for (int ig = 0; ig < b->nsgt; ig++) {
            gft[ig] = pbar * cx->hd[b->pos[ig]].cdist;
            if (gft[ig] > maxgft) maxgft = gft[ig];
        }
        for (int ig = 0; ig < b->nsgt; ig++) {
            t0[ig] = maxgft - gft[ig];
            backt0 = backt0 - t0[ig] * b->wt[ig];
            t0[ig] = t0[ig] + cx->hd[b->pos[ig]].tst;
        }
        backt0 = backt0 + a->tinit - cx->tstart;

        /* mech_sgt: dip and rake terms */
        float arg = a->dip * rperd;
        const float cxD = (float)cos(arg), sxD = (float)sin(arg);
        arg = a->rake * rperd;
        const float cxL = (float)cos(arg), sxL = (float)sin(arg);

        for (int im = 0; im < nmech; im++) {
            awp_synth_gterm *g = &gt[nt_];
            awp_synth_cterm *c = &ct[nt_];
            const float u1 = flag[im] == 1 ? 1.0f : 0.0f, u2 = flag[im] == 2 ? 1.0f : 0.0f;
            const float u3 = flag[im] == 3 ? 1.0f : 0.0f;
            g->nsgt = b->nsgt;
            for (int ig = 0; ig < b->nsgt; ig++) {
                const awp_sgtheader *h = &cx->hd[b->pos[ig]];
                float *k = g->c[ig];
                arg = (a->stk - h->xazim) * rperd;
                const float cxT = (float)cos(arg), sxT = (float)sin(arg);
                const float vx = -sxD * sxT, vy = sxD * cxT, vz = -cxD;
                const float us = u1 * cxL - u2 * sxL, ud = u1 * sxL + u2 * cxL;
                const float ux = -(u3 * sxD - ud * cxD) * sxT + us * cxT;
                const float uy = (u3 * sxD - ud * cxD) * cxT + us * sxT;
                const float uz = -(u3 * cxD + ud * sxD);
                const float l2m = h->lam + two * h->mu;
                k[SY_MXX] = l2m * vx * ux + h->lam * vy * uy + h->lam * vz * uz;
                k[SY_MYY] = h->lam * vx * ux + l2m * vy * uy + h->lam * vz * uz;
                k[SY_MZZ] = h->lam * vx * ux + h->lam * vy * uy + l2m * vz * uz;
                k[SY_MXY] = h->mu * (vx * uy + vy * ux);
                k[SY_MXZ] = h->mu * (vx * uz + vz * ux);
                k[SY_MYZ] = h->mu * (vy * uz + vz * uy);
                arg = h->xazim * rperd;
                k[SY_COSA] = (float)cos(arg);
                k[SY_SINA] = (float)sin(arg);
                k[SY_XAMP] = h->xmom > 0.0f ? scl * b->wt[ig] / h->xmom : 0.0f;
                k[SY_YAMP] = h->ymom > 0.0f ? scl * b->wt[ig] / h->ymom : 0.0f;
                k[SY_ZAMP] = h->zmom > 0.0f ? scl * b->wt[ig] / h->zmom : 0.0f;

                /* timeshift_sgt (sgt3d_subs.c:1214-1255) */
                const float tsh = t0[ig] + backt0;
                const int sh = tsh >= 0.0f ? (int)(tsh / h->dt + 0.5) : (int)(tsh / h->dt - 0.5);
                int it0 = h->nt + sh;
                if (it0 > cx->ntsum) it0 = cx->ntsum;
                if (it0 > cx->ntout) it0 = cx->ntout;
                g->pt[ig] = b->pos[ig];
                g->shift[ig] = sh;
                g->lo[ig] = sh < 0 ? 0 : sh;
                g->hi[ig] = it0 > g->lo[ig] ? it0 : g->lo[ig];
            }
            for (int ig = b->nsgt; ig < 4; ig++) {
                g->pt[ig] = 0;
                g->shift[ig] = g->lo[ig] = g->hi[ig] = 0;
                memset(g->c[ig], 0, sizeof g->c[ig]);
            }

            /* srf_stf: stf[it] = dt * slip rate (srf_rupm.c:111-112) */
            const int nstf = flag[im] == 1 ? a->nt1 : flag[im] == 2 ? a->nt2 : a->nt3;
            const long long off = flag[im] == 1 ? a->stf1 : flag[im] == 2 ? a->stf2 : a->stf3;
            if (off < 0 || off + nstf > npool) return perr("synthesis: SRF slip-rate offset outside the sample pool");
            if (nstf > cx->ntout) return perr("synthesis: slip-rate function longer than ntout");
            for (int it = 0; it < nstf; it++) stf[ns + it] = cx->dtout * pool[off + it];
            c->stf = stf_base + ns;
            c->nstf = nstf;
            c->slot = 0;
            /* a single SGT point reaches [lo, hi) only; with several the
             * combination kernel writes every sample */
            c->lo = b->nsgt == 1 ? g->lo[0] : 0;
            c->hi = b->nsgt == 1 ? g->hi[0] : cx->ntout;
            ns += nstf;
            /* per component: sum over it < ntout of min(it + 1, nstf) */
            mac += (long long)nstf * (nstf + 1) / 2 + (long long)(cx->ntout - nstf) * nstf;
            nt_++;
        }
    }
    *nterms = nt_;
    *nstf_used = ns;
    *macs = mac;
    return AWP_OK;
}

/* ---- SRF files (DirectSynth/src/jbsim/srf_subs.c:521-690) --------------- */

typedef struct {
    awp_srf_point *p;
    int np;
    float *pool;
    long long npool, cap;
} srf_buf;

static int pool_reserve(srf_buf *b, long long extra)
{
    if (b->npool + extra <= b->cap) return 0;
    long long c = b->cap ? b->cap : 4096;
    while (c < b->npool + extra) c *= 2;
    float *q = (float *)realloc(b->pool, (size_t)c * sizeof(float));
    if (!q) return -1;
    b->pool = q;
    b->cap = c;
    return 0;
}

static awp_status srf_fail(srf_buf *b, const char *msg, const char *path)
{
    char t[1300];
    snprintf(t, sizeof t, "%s: %s", path, msg);
    awp_set_error_text(t);
    free(b->p);
    free(b->pool);
    return AWP_ERR_IO;
}

static awp_status read_srf_text(FILE *f, const char *path, srf_buf *b)
{
    char line[1024], word[64] = {0};
    if (!fgets(line, sizeof line, f) || !fgets(line, sizeof line, f)) return srf_fail(b, "SRF header missing", path);
    if (sscanf(line, "%63s", word) != 1) return srf_fail(b, "SRF header missing", path);
    if (strncmp(word, "PLANE", 5) == 0) {
        int nseg = 0;
        if (sscanf(line, "%*s %d", &nseg) != 1 || nseg < 0) return srf_fail(b, "bad PLANE line", path);
        for (int i = 0; i < 2 * nseg; i++)
            if (!fgets(line, sizeof line, f)) return srf_fail(b, "PLANE block cut short", path);
        while (strncmp(word, "POINTS", 6) != 0) {
            if (!fgets(line, sizeof line, f)) return srf_fail(b, "no POINTS block", path);
            word[0] = 0;
            sscanf(line, "%63s", word);
        }
    }
    if (strncmp(word, "POINTS", 6) != 0) return srf_fail(b, "no POINTS block", path);
    if (sscanf(line, "%*s %d", &b->np) != 1 || b->np < 0) return srf_fail(b, "bad POINTS count", path);
    b->p = (awp_srf_point *)calloc((size_t)(b->np ? b->np : 1), sizeof(awp_srf_point));
    if (!b->p) return srf_fail(b, "out of host memory", path);
    for (int i = 0; i < b->np; i++) {
        awp_srf_point *a = &b->p[i];
        if (fscanf(f, "%f %f %f %f %f %f %f %f", &a->lon, &a->lat, &a->dep, &a->stk, &a->dip, &a->area, &a->tinit,
                   &a->dt) != 8 ||
            fgets(line, sizeof line, f) == NULL)
            return srf_fail(b, "point record cut short", path);
        if (fscanf(f, "%f %f %d %f %d %f %d", &a->rake, &a->slip1, &a->nt1, &a->slip2, &a->nt2, &a->slip3,
                   &a->nt3) != 7)
            return srf_fail(b, "point slip line cut short", path);
        if (a->nt1 < 0 || a->nt2 < 0 || a->nt3 < 0) return srf_fail(b, "negative sample count", path);
        const int n[3] = {a->nt1, a->nt2, a->nt3};
        long long *off[3] = {&a->stf1, &a->stf2, &a->stf3};
        for (int q = 0; q < 3; q++) {
            if (pool_reserve(b, n[q])) return srf_fail(b, "out of host memory", path);
            *off[q] = b->npool;
            for (int it = 0; it < n[q]; it++)
                if (fscanf(f, "%f", &b->pool[b->npool + it]) != 1) return srf_fail(b, "slip-rate samples cut short", path);
            b->npool += n[q];
        }
    }
    return AWP_OK;
}

static int rd(int fd, void *dst, size_t n)
{
    char *p = (char *)dst;
    while (n) {
        ssize_t r = read(fd, p, n);
        if (r <= 0) return -1;
        p += r;
        n -= (size_t)r;
    }
    return 0;
}

/* binary SRF: version[32], a 32-byte word, optional PLANE segments, POINTS
 * np, then per point 15 words and the three sample lists (srf_subs.c:534-598).
 * The segment record of srf_structure.h is 2 floats, 2 ints, 9 floats. */
static awp_status read_srf_binary(int fd, const char *path, srf_buf *b)
{
    char version[32], word[32];
    if (rd(fd, version, sizeof version) || rd(fd, word, sizeof word)) return srf_fail(b, "SRF header missing", path);
    if (strncmp(word, "PLANE", 6) == 0) {
        int nseg;
        if (rd(fd, &nseg, sizeof nseg) || nseg < 0) return srf_fail(b, "bad PLANE block", path);
        char seg[52];
        for (int i = 0; i < nseg; i++)
            if (rd(fd, seg, sizeof seg)) return srf_fail(b, "PLANE block cut short", path);
        while (strncmp(word, "POINTS", 6) != 0)
            if (rd(fd, word, sizeof word)) return srf_fail(b, "no POINTS block", path);
    }
    if (strncmp(word, "POINTS", 6) != 0) return srf_fail(b, "no POINTS block", path);
    if (rd(fd, &b->np, sizeof b->np) || b->np < 0) return srf_fail(b, "bad POINTS count", path);
    b->p = (awp_srf_point *)calloc((size_t)(b->np ? b->np : 1), sizeof(awp_srf_point));
    if (!b->p) return srf_fail(b, "out of host memory", path);
    for (int i = 0; i < b->np; i++) {
        awp_srf_point *a = &b->p[i];
        float f9[9];
        if (rd(fd, f9, sizeof f9)) return srf_fail(b, "point record cut short", path);
        a->lon = f9[0], a->lat = f9[1], a->dep = f9[2], a->stk = f9[3], a->dip = f9[4], a->area = f9[5];
        a->tinit = f9[6], a->dt = f9[7], a->rake = f9[8];
        if (rd(fd, &a->slip1, 4) || rd(fd, &a->nt1, 4) || rd(fd, &a->slip2, 4) || rd(fd, &a->nt2, 4) ||
            rd(fd, &a->slip3, 4) || rd(fd, &a->nt3, 4))
            return srf_fail(b, "point slip words cut short", path);
        if (a->nt1 < 0 || a->nt2 < 0 || a->nt3 < 0) return srf_fail(b, "negative sample count", path);
        const int n[3] = {a->nt1, a->nt2, a->nt3};
        long long *off[3] = {&a->stf1, &a->stf2, &a->stf3};
        for (int q = 0; q < 3; q++) {
            if (pool_reserve(b, n[q])) return srf_fail(b, "out of host memory", path);
            *off[q] = b->npool;
            if (n[q] && rd(fd, b->pool + b->npool, sizeof(float) * (size_t)n[q]))
                return srf_fail(b, "slip-rate samples cut short", path);
            b->npool += n[q];
        }
    }
    return AWP_OK;
}

awp_status awp_srf_read(const char *path, int binary, awp_srf_point **pts, int *np, float **pool, long long *npool)
{
    if (!path || !pts || !np || !pool || !npool) return perr("awp_srf_read: null argument");
    srf_buf b = {0};
    awp_status st;
    if (binary) {
        const int fd = open(path, O_RDONLY);
        if (fd < 0) return srf_fail(&b, "cannot open", path);
        st = read_srf_binary(fd, path, &b);
        close(fd);
    } else {
        FILE *f = fopen(path, "r");
        if (!f) return srf_fail(&b, "cannot open", path);
        st = read_srf_text(f, path, &b);
        fclose(f);
    }
    if (st != AWP_OK) return st;
    if (!b.pool) b.pool = (float *)malloc(sizeof(float));
    *pts = b.p;
    *np = b.np;
    *pool = b.pool;
    *npool = b.npool;
    return AWP_OK;
}
