/*
 * synth_oracle.c -- CPU oracle of the reciprocity seismogram synthesis
 * (TEST INFRASTRUCTURE: only tests/, the smoke check and bench.py's CPU
 * baseline call it; nothing in the library does).
 *
 * A sequential restatement of CyberShake DirectSynth's worker step for one
 * rupture and one site, in the reference's own loop structure and float /
 * double evaluation order:
 *   geoprojection and grid lookup     DirectSynth/src/jbsim/geoproj_subs.c:10-197,
 *                                     jbsim/misc_subs.c:151-173
 *   bracketing SGT points             jbsim/sgt3d_subs.c:751-961 (find_sgt)
 *   lengths                           jbsim/jbsim3d.c:436-447
 *   per point, per variation          jbsim/jbsim3d.c:480-520:
 *     get_srfpars                     jbsim/srf_rupm.c:7-53
 *     mech_sgt                        jbsim/sgt3d_subs.c:1260-1422
 *     sum_sgt / timeshift_sgt         jbsim/sgt3d_subs.c:1121-1258
 *     srf_stf / do_cnvlv              jbsim/srf_rupm.c:55-153, jbsim/stf_subs.c:6-40
 * Points are processed in rupture order, as when one SGT handler holds every
 * point the rupture needs.  SRF resampling (srf_rupm.c:115-146) is not
 * restated; a variation whose sample interval differs from dtout is refused.
 *
 * Pinned: the reference's own functions for this path compile from their
 * sources with declaration-only stand-ins for the libraries they do not use
 * here (oracle/Makefile.ref, oracle/refinc, synth_ref_stubs.c), and
 * synth_ref_driver.c runs them in jbsim3d_synth's order; this restatement
 * equals them bit for bit on every case of tests/golden/synth (seismograms
 * they produced) and of the live comparisons in tests/test_synth.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int geoproj;
    float modellon, modellat, modelrot, xshift, yshift;
    int globnp, localnp, nt;
} o_master;
typedef struct {
    long long indx;
    int xsgt, ysgt, zsgt;
    float h;
} o_index;
typedef struct {
    long long indx;
    int geoproj;
    float modellon, modellat, modelrot, xshift, yshift;
    int nt;
    float xazim, dt, tst, h, src_lat, src_lon, src_dep;
    int xsrc, ysrc, zsrc;
    float sgt_lat, sgt_lon, sgt_dep;
    int xsgt, ysgt, zsgt;
    float cdist, lam, mu, rho, xmom, ymom, zmom;
} o_header;
typedef struct {
    float lon, lat, dep, stk, dip, area, tinit, dt, rake;
    float slip1, slip2, slip3;
    int nt1, nt2, nt3;
    long long stf1, stf2, stf3;
} o_point;

/* ---- geoprojection (geoproj 1) ---- */
typedef struct {
    double amat[9], ainv[9], g0, b0;
    float erad;
} o_geo;

static void o_gen_matrices(o_geo *g, float alpha, float ref_lon, float ref_lat)
{
    double rperd = 0.017453292, arg;
    arg = (double)(alpha)*rperd;
    double cosA = cos(arg), sinA = sin(arg);
    arg = (double)(90.0 - ref_lat) * rperd;
    double cosT = cos(arg), sinT = sin(arg);
    arg = (double)(ref_lon)*rperd;
    double cosP = cos(arg), sinP = sin(arg);
    double *amat = g->amat, *ainv = g->ainv;
    amat[0] = cosA * cosT * cosP + sinA * sinP;
    amat[1] = sinA * cosT * cosP - cosA * sinP;
    amat[2] = sinT * cosP;
    amat[3] = cosA * cosT * sinP - sinA * cosP;
    amat[4] = sinA * cosT * sinP + cosA * cosP;
    amat[5] = sinT * sinP;
    amat[6] = -cosA * sinT;
    amat[7] = -sinA * sinT;
    amat[8] = cosT;
    double det = amat[0] * (amat[4] * amat[8] - amat[7] * amat[5]) - amat[1] * (amat[3] * amat[8] - amat[6] * amat[5]) +
                 amat[2] * (amat[3] * amat[7] - amat[6] * amat[4]);
    det = 1.0 / det;
    ainv[0] = det * amat[0];
    ainv[1] = det * amat[3];
    ainv[2] = det * amat[6];
    ainv[3] = det * amat[1];
    ainv[4] = det * amat[4];
    ainv[5] = det * amat[7];
    ainv[6] = det * amat[2];
    ainv[7] = det * amat[5];
    ainv[8] = det * amat[8];
}

static void o_set_geoproj(const o_master *m, o_geo *g)
{
    float xlen = -2.0 * m->xshift, ylen = -2.0 * m->yshift;
    g->erad = 6378.139;
    o_gen_matrices(g, m->modelrot, m->modellon, m->modellat);
    g->g0 = (double)(0.5 * ylen) / (double)(g->erad);
    g->b0 = (double)(0.5 * xlen) / (double)(g->erad);
}

static void o_gcproj_inv(const o_geo *g, float *xf, float *yf, float rlon, float rlat)
{
    double rperd = 0.017453292, arg, cosG, sinG, cosB, sinB, xg, yg, zg, xp, yp;
    arg = rlon * rperd;
    cosG = cos(arg);
    sinG = sin(arg);
    arg = (90.0 - rlat) * rperd;
    cosB = cos(arg);
    sinB = sin(arg);
    xg = sinB * cosG;
    yg = sinB * sinG;
    zg = cosB;
    xp = xg * g->ainv[0] + yg * g->ainv[1] + zg * g->ainv[2];
    yp = xg * g->ainv[3] + yg * g->ainv[4] + zg * g->ainv[5];
    sinG = xp / sqrt(1.0 - yp * yp);
    sinB = yp / sqrt(1.0 - xp * xp);
    *xf = (double)(g->erad) * (asin(sinB) + g->b0);
    *yf = (double)(g->erad) * (asin(sinG) + g->g0);
}

static void o_get_indx(const o_geo *g, float lon, float lat, float dep, o_index *ix)
{
    float xr, yr;
    double invh = 1.0 / (double)(ix->h);
    o_gcproj_inv(g, &xr, &yr, lon, lat);
    ix->xsgt = (int)((double)(xr)*invh + 0.5);
    ix->ysgt = (int)((double)(yr)*invh + 0.5);
    ix->zsgt = (int)((double)(dep)*invh + 1.5);
    ix->indx = (long long)(ix->xsgt) * (long long)(1000000000000) + (long long)(ix->ysgt) * (long long)(1000000) +
               (long long)(ix->zsgt);
}

/* ---- find_sgt ---- */
typedef struct {
    int nsgt;
    long long indx[4];
    float wt[4];
    int ip[4];
} o_sgtpar;

static void o_find_sgt(o_sgtpar *sp, const o_index *sgtindx, int globnp, const o_index *eq, const o_index *st)
{
    int start = 0, end = globnp - 1, mid = (start + end) / 2, ip;
    while (end >= start) {
        mid = (start + end) / 2;
        if (eq->indx > sgtindx[mid].indx) start = mid + 1;
        else if (eq->indx < sgtindx[mid].indx) end = mid - 1;
        else break;
    }
    ip = mid;
    if (eq->indx == sgtindx[ip].indx) {
        sp->nsgt = 1;
        sp->indx[0] = sgtindx[ip].indx;
        sp->wt[0] = 1.0;
        sp->ip[0] = ip;
        return;
    }
    float xx, yy, zz, rng, zdp, rexact, zexact, del, delta[4], sum;
    int p[4] = {-1, -1, -1, -1}, i;
    sp->nsgt = 0;
    for (i = 0; i < 4; i++) delta[i] = 1.0e+15;
    xx = (eq->xsgt - st->xsgt);
    yy = (eq->ysgt - st->ysgt);
    rexact = xx * xx + yy * yy;
    zexact = (eq->zsgt - st->zsgt);
    for (ip = 0; ip < globnp; ip++) {
        xx = (sgtindx[ip].xsgt - st->xsgt);
        yy = (sgtindx[ip].ysgt - st->ysgt);
        rng = xx * xx + yy * yy;
        zdp = (sgtindx[ip].zsgt - st->zsgt);
        xx = (sgtindx[ip].xsgt - eq->xsgt);
        yy = (sgtindx[ip].ysgt - eq->ysgt);
        zz = (sgtindx[ip].zsgt - eq->zsgt);
        del = xx * xx + yy * yy + zz * zz;
        int q;
        if (rng <= rexact && zdp <= zexact) q = 0;
        else if (rng > rexact && zdp <= zexact) q = 1;
        else if (rng <= rexact && zdp > zexact) q = 2;
        else q = 3;
        if (p[q] < 0) {
            p[q] = sp->nsgt;
            sp->nsgt = sp->nsgt + 1;
        }
        if (del < delta[p[q]]) {
            delta[p[q]] = del;
            sp->indx[p[q]] = sgtindx[ip].indx;
            sp->wt[p[q]] = sqrt(del);
            sp->ip[p[q]] = ip;
        }
    }
    int zflag = -1;
    for (i = 0; i < sp->nsgt; i++)
        if (sp->wt[i] == 0.0) zflag = i;
    if (zflag >= 0) {
        for (i = 0; i < sp->nsgt; i++) sp->wt[i] = 0.0;
        sp->wt[zflag] = 1.0;
    } else {
        sum = 0.0;
        for (i = 0; i < sp->nsgt; i++) sum = sum + 1.0 / sp->wt[i];
        sum = 1.0 / sum;
        for (i = 0; i < sp->nsgt; i++) sp->wt[i] = sum / sp->wt[i];
    }
}

/* ---- mech_sgt ---- */
static void o_mech_sgt(float *gfmech, const o_sgtpar *sp, const o_header *const *hp, const float *const (*rows)[18],
                       int nts, int nmech, const int *flag, float stk, float dip, float rak, float *scl)
{
    float rperd = 0.017453293, two = 2.0, arg;
    float cxD, sxD, cxL, sxL, cxT, sxT, vx, vy, vz, u1, u2, u3, us, ud, ux, uy, uz, l2m;
    float mxx, myy, mzz, mxy, mxz, myz, cosA, sinA, xamp, yamp, zamp, sx, sy, sz, sum = 0.0;
    int im, ig, it;
    arg = dip * rperd;
    cxD = cos(arg);
    sxD = sin(arg);
    for (im = 0; im < nmech; im++) {
        u1 = u2 = u3 = 0;
        if (flag[im] == 1) u1 = 1;
        else if (flag[im] == 2) u2 = 1;
        else if (flag[im] == 3) u3 = 1;
        float *gfmptr = gfmech + im * 12 * nts;
        memset(gfmptr, 0, sizeof(float) * 12 * nts);
        arg = rak * rperd;
        cxL = cos(arg);
        sxL = sin(arg);
        sum = 0.0;
        for (ig = 0; ig < sp->nsgt; ig++) {
            const o_header *h = hp[ig];
            const float *const *r = rows[ig];
            arg = (stk - h->xazim) * rperd;
            cxT = cos(arg);
            sxT = sin(arg);
            vx = -sxD * sxT;
            vy = sxD * cxT;
            vz = -cxD;
            us = u1 * cxL - u2 * sxL;
            ud = u1 * sxL + u2 * cxL;
            ux = -(u3 * sxD - ud * cxD) * sxT + us * cxT;
            uy = (u3 * sxD - ud * cxD) * cxT + us * sxT;
            uz = -(u3 * cxD + ud * sxD);
            l2m = h->lam + two * h->mu;
            mxx = l2m * vx * ux + (h->lam) * vy * uy + (h->lam) * vz * uz;
            myy = (h->lam) * vx * ux + l2m * vy * uy + (h->lam) * vz * uz;
            mzz = (h->lam) * vx * ux + (h->lam) * vy * uy + l2m * vz * uz;
            mxy = (h->mu) * (vx * uy + vy * ux);
            mxz = (h->mu) * (vx * uz + vz * ux);
            myz = (h->mu) * (vy * uz + vz * uy);
            arg = h->xazim * rperd;
            cosA = cos(arg);
            sinA = sin(arg);
            float *gfv = gfmptr + 3 * ig * nts, *gfn = gfv + nts, *gfe = gfv + 2 * nts;
            sum = sum + (*scl) * (h->mu) * (sp->wt[ig]);
            xamp = 0.0;
            if (h->xmom > 0.0) xamp = (*scl) * (sp->wt[ig]) / (h->xmom);
            yamp = 0.0;
            if (h->ymom > 0.0) yamp = (*scl) * (sp->wt[ig]) / (h->ymom);
            zamp = 0.0;
            if (h->zmom > 0.0) zamp = (*scl) * (sp->wt[ig]) / (h->zmom);
            for (it = 0; it < h->nt; it++) {
                sx = xamp * (r[0][it] * mxx + r[1][it] * myy + r[2][it] * mzz + r[3][it] * mxy + r[4][it] * mxz +
                             r[5][it] * myz);
                sy = yamp * (r[6][it] * mxx + r[7][it] * myy + r[8][it] * mzz + r[9][it] * mxy + r[10][it] * mxz +
                             r[11][it] * myz);
                sz = zamp * (r[12][it] * mxx + r[13][it] * myy + r[14][it] * mzz + r[15][it] * mxy +
                             r[16][it] * mxz + r[17][it] * myz);
                gfe[it] = sx * sinA + sy * cosA;
                gfn[it] = sx * cosA - sy * sinA;
                gfv[it] = -sz;
            }
        }
    }
    *scl = sum;
}

/* ---- sum_sgt / timeshift_sgt ---- */
static void o_timeshift(float *seis, int ntout, float *gf, int ntsum, const float *t0, const float *bt0,
                        const o_sgtpar *sp, const o_header *const *hp)
{
    int taplen = 10, i, ig, it, tapst, itshift, it0;
    float pi = 3.141592654, half = 0.5, one = 1.0, arg, fac, tsh;
    float *sv = seis, *sn = seis + ntout, *se = seis + 2 * ntout;
    for (ig = 0; ig < sp->nsgt; ig++) {
        float *gf0 = gf + 3 * ig * ntsum, *gf1 = gf0 + ntsum, *gf2 = gf0 + 2 * ntsum;
        const o_header *h = hp[ig];
        tapst = h->nt - taplen;
        arg = pi / (float)(taplen);
        for (it = tapst + 1; it < h->nt; it++) {
            fac = half * (one + cos(arg * (it - tapst)));
            gf0[it] = fac * gf0[it];
            gf1[it] = fac * gf1[it];
            gf2[it] = fac * gf2[it];
        }
        tsh = t0[ig] + *bt0;
        if (tsh >= 0.0) itshift = (int)(tsh / h->dt + 0.5);
        else itshift = (int)(tsh / h->dt - 0.5);
        it0 = h->nt + itshift;
        if (it0 > ntsum) it0 = ntsum;
        if (it0 > ntout) it0 = ntout;
        if (itshift < 0) {
            for (i = 0; i < it0; i++) {
                sv[i] = sv[i] + gf0[i - itshift];
                sn[i] = sn[i] + gf1[i - itshift];
                se[i] = se[i] + gf2[i - itshift];
            }
        } else {
            for (i = it0 - 1; i >= itshift; i--) {
                sv[i] = sv[i] + gf0[i - itshift];
                sn[i] = sn[i] + gf1[i - itshift];
                se[i] = se[i] + gf2[i - itshift];
            }
        }
    }
}

static void o_sum_sgt(float *seis, int ntout, float *gfmech, const o_sgtpar *sp, const o_header *const *hp, int ntsum,
                      float rupt, float tstart, int nmech)
{
    float pbar = 0.0, maxgft = -1.0e+15, backt0 = 0.0, t0[4], gft[4];
    int ig, im;
    for (ig = 0; ig < sp->nsgt; ig++) pbar = pbar + sqrt(hp[ig]->rho / hp[ig]->mu);
    pbar = pbar / (float)(sp->nsgt);
    for (ig = 0; ig < sp->nsgt; ig++) {
        gft[ig] = pbar * hp[ig]->cdist;
        if (gft[ig] > maxgft) maxgft = gft[ig];
    }
    for (ig = 0; ig < sp->nsgt; ig++) {
        t0[ig] = maxgft - gft[ig];
        backt0 = backt0 - t0[ig] * sp->wt[ig];
        t0[ig] = t0[ig] + hp[ig]->tst;
    }
    backt0 = backt0 + rupt - tstart;
    for (im = 0; im < nmech; im++)
        o_timeshift(seis + 3 * im * ntout, ntout, gfmech + 12 * im * ntsum, ntsum, t0, &backt0, sp, hp);
}

/* ---- srf_stf / do_cnvlv ---- */
static void o_cnvlv(float *s, const float *u, int nt, const float *stf, int nstf)
{
    const float *uv = u, *un = u + nt, *ue = u + 2 * nt;
    float *sv = s, *sn = s + nt, *se = s + 2 * nt;
    for (int it = 0; it < nt; it++) {
        int kend = it + 1;
        if (kend > nstf) kend = nstf;
        float acc[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < kend; k++) {
            acc[0] += stf[k] * uv[it - k];
            acc[1] += stf[k] * un[it - k];
            acc[2] += stf[k] * ue[it - k];
        }
        sv[it] += acc[0];
        sn[it] += acc[1];
        se[it] += acc[2];
    }
}

/*
 * One rupture: nv variations of np points each (pts[v * np + i]); each
 * variation's slip-rate offsets index pool + pool_off[v].  sgt[q] are the
 * [globnp][6][nt] arrays of the x, y, z components (NULL beyond ncomp); hd
 * are the x component's headers.  seis receives nv * 3 * ntout floats.
 * Returns 0, or -1 for a variation the restatement refuses (resampling), -2
 * for a slip rate longer than ntout, -3 for allocation failure.
 */
int orc_synth(const o_master *m, const o_index *ix, const o_header *hd_in, int ncomp, const float *sx,
              const float *sy, const float *sz, float slon, float slat, float dtout, int ntout_in, float tstart,
              int nv, int np, const o_point *pts, const float *pool, const long long *pool_off, float *seis,
              int *ntout_out)
{
    const int globnp = m->globnp, nt = m->nt;
    o_header *hd = (o_header *)malloc(sizeof(o_header) * (size_t)globnp);
    if (!hd) return -3;
    memcpy(hd, hd_in, sizeof(o_header) * (size_t)globnp);
    for (int i = 0; i < globnp; i++) {               /* synth.c:545-557 */
        if (ncomp >= 2) hd[i].ymom = hd[i].xmom;
        if (ncomp == 3) hd[i].zmom = hd[i].xmom;
    }
    const float *src[3] = {sx, sy, sz};
    float *zero = (float *)calloc((size_t)nt, sizeof(float));

    o_geo geo;
    o_set_geoproj(m, &geo);
    o_index stat, eq;
    stat.h = ix[0].h;
    eq.h = ix[0].h;
    o_get_indx(&geo, slon, slat, 0.0f, &stat);
    o_sgtpar *sp = (o_sgtpar *)malloc(sizeof(o_sgtpar) * (size_t)(np ? np : 1));
    for (int ip = 0; ip < np; ip++) {
        o_get_indx(&geo, pts[ip].lon, pts[ip].lat, pts[ip].dep, &eq);
        o_find_sgt(&sp[ip], ix, globnp, &eq, &stat);
    }

    int maxnt = hd[0].nt;
    float mindt = hd[0].dt;
    if (dtout < mindt) maxnt = (maxnt * mindt / dtout);
    int ntsum = 2;
    while (ntsum < 4 * maxnt) ntsum = ntsum * 2;
    const int ntout = ntout_in > 0 ? ntout_in : ntsum;
    *ntout_out = ntout;

    const int maxmech = 3;
    float *gfmech = (float *)malloc(sizeof(float) * (size_t)maxmech * 12 * ntsum);
    float *subseis = (float *)malloc(sizeof(float) * (size_t)maxmech * 3 * ntout);
    float *stf = (float *)malloc(sizeof(float) * (size_t)ntout);
    int rc = 0;
    if (!gfmech || !subseis || !stf || !zero || !sp) rc = -3;
    if (!rc) memset(seis, 0, sizeof(float) * (size_t)nv * 3 * ntout);
    float ratio_tol = 0.00001, pratio_tol = 1.0 + ratio_tol, mratio_tol = 1.0 - ratio_tol;

    for (int ip = 0; ip < np && !rc; ip++) {
        const o_header *hp[4];
        const float *rows[4][18];
        for (int ig = 0; ig < sp[ip].nsgt; ig++) {
            const int p = sp[ip].ip[ig];
            hp[ig] = &hd[p];
            for (int q = 0; q < 3; q++)
                for (int r = 0; r < 6; r++)
                    rows[ig][6 * q + r] = q < ncomp ? src[q] + ((size_t)p * 6 + r) * nt : zero;
        }
        for (int v = 0; v < nv && !rc; v++) {
            const o_point *a = &pts[(size_t)v * np + ip];
            const float *vp = pool + pool_off[v];
            /* get_srfpars */
            int nmech = 0, flag[3] = {0, 0, 0};
            if (a->nt1 > 0) flag[nmech++] = 1;
            if (a->nt2 > 0) flag[nmech++] = 2;
            if (a->nt3 > 0) flag[nmech++] = 3;
            float scale = 1.0f * a->area;
            memset(subseis, 0, sizeof(float) * (size_t)maxmech * 3 * ntout);
            o_mech_sgt(gfmech, &sp[ip], hp, (const float *const(*)[18])rows, ntsum, nmech, flag, a->stk, a->dip,
                       a->rake, &scale);
            o_sum_sgt(subseis, ntout, gfmech, &sp[ip], hp, ntsum, a->tinit, tstart, nmech);
            /* srf_stf */
            float *sv = seis + (size_t)v * 3 * ntout;
            for (int im = 0; im < nmech; im++) {
                int nstf;
                const float *sptr;
                if (flag[im] == 1) nstf = a->nt1, sptr = vp + a->stf1;
                else if (flag[im] == 2) nstf = a->nt2, sptr = vp + a->stf2;
                else nstf = a->nt3, sptr = vp + a->stf3;
                if (nstf > ntout) {
                    rc = -2;
                    break;
                }
                memset(stf, 0, sizeof(float) * (size_t)ntout);
                for (int it = 0; it < nstf; it++) stf[it] = dtout * sptr[it];
                if (dtout / a->dt > pratio_tol || dtout / a->dt < mratio_tol) {
                    rc = -1;
                    break;
                }
                o_cnvlv(sv, subseis + 3 * im * ntout, ntout, stf, nstf);
            }
        }
    }
    free(gfmech);
    free(subseis);
    free(stf);
    free(zero);
    free(sp);
    free(hd);
    return rc;
}

/* the grid lookup alone, for the tests of the projection */
void orc_synth_get_indx(const o_master *m, float h, float lon, float lat, float dep, long long *indx, int *xyz)
{
    o_geo geo;
    o_set_geoproj(m, &geo);
    o_index o;
    o.h = h;
    o_get_indx(&geo, lon, lat, dep, &o);
    *indx = o.indx;
    xyz[0] = o.xsgt;
    xyz[1] = o.ysgt;
    xyz[2] = o.zsgt;
}
