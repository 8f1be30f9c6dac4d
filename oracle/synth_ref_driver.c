/*
 * synth_ref_driver.c -- TEST INFRASTRUCTURE: runs CyberShake DirectSynth's own
 * synthesis functions on in-memory inputs, to pin the synthesis oracle
 * (synth_oracle.c) and to make golden fixtures.
 *
 * Built only where the reference sources are present (oracle/Makefile.ref)
 * together with DirectSynth/src/jbsim/{sgt3d_subs,srf_rupm,stf_subs,
 * geoproj_subs,misc_subs}.c into oracle/_ref/libsynth_ref.so.  This file is
 * the glue a single-handler DirectSynth worker would run between those
 * functions: it replays jbsim3d_synth's loop (jbsim/jbsim3d.c:436-520) --
 * set_geoproj / get_indx / find_sgt for the site and the points (synth.c:35-74),
 * then per point and per variation get_srfpars, mech_sgt, sum_sgt and srf_stf
 * -- with the SGT buffer laid out as request_sgt leaves it (synth.c:520-557:
 * [point][component][6][nt], the x headers with ymom / zmom set to xmom).
 * The arithmetic is the reference's; only the loop and the data plumbing are
 * written here.
 */
#include "include.h"
#include "defs.h"
#include "structure.h"
#include "srf_structure.h"
#include "function.h"

/* defined in the reference sources, not declared in their headers */
void mech_sgt(float *gfmech, struct sgtparams *sgtpar, int nts, struct mechparam mp, float *scl);
void sum_sgt(float *seis, int ntout, float *gfmech, struct sgtparams *sgtpar, int ntsum, float *rupt, float *tstart,
             struct mechparam mp, int srf_index);
void srf_stf(struct standrupformat *srf, int off, int ip, float *s, float *u, float *stf, int nt, float *dt,
             struct mechparam mp, float *space);
void zapit(float *s, int n);

/* the synthesis ABI's rupture point record (awp_srf_point) */
typedef struct {
    float lon, lat, dep, stk, dip, area, tinit, dt, rake;
    float slip1, slip2, slip3;
    int nt1, nt2, nt3;
    long long stf1, stf2, stf3;
} drv_point;

static int find_pos(const struct sgtindex *ix, int np, long long indx)
{
    int lo = 0, hi = np - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) / 2;
        if (ix[mid].indx < indx) lo = mid + 1;
        else if (ix[mid].indx > indx) hi = mid - 1;
        else return mid;
    }
    return -1;
}

/* Same arguments and result as orc_synth (synth_oracle.c).  Returns 0, or
 * -1 when an SGT index is missing, -3 on allocation failure. */
int ref_synth(const struct sgtmaster *m_in, const struct sgtindex *ix_in, const struct sgtheader *hd_in, int ncomp,
              const float *sx, const float *sy, const float *sz, float slon, float slat, float dtout, int ntout_in,
              float tstart, int nv, int np, const drv_point *pts, const float *pool, const long long *pool_off,
              float *seis_out, int *ntout_out)
{
    struct sgtmaster m = *m_in;
    const int globnp = m.globnp, nt = m.nt;
    struct sgtindex *ix = (struct sgtindex *)malloc(sizeof(*ix) * (size_t)globnp);
    struct sgtheader *hd = (struct sgtheader *)malloc(sizeof(*hd) * (size_t)globnp);
    float *sgtbuf = (float *)calloc((size_t)globnp * 18 * nt, sizeof(float));
    if (!ix || !hd || !sgtbuf) return -3;
    memcpy(ix, ix_in, sizeof(*ix) * (size_t)globnp);
    memcpy(hd, hd_in, sizeof(*hd) * (size_t)globnp);
    const float *src[3] = {sx, sy, sz};
    for (int p = 0; p < globnp; p++) {
        if (ncomp >= 2) hd[p].ymom = hd[p].xmom;
        if (ncomp == 3) hd[p].zmom = hd[p].xmom;
        for (int q = 0; q < ncomp; q++)
            memcpy(sgtbuf + ((size_t)p * 18 + 6 * q) * nt, src[q] + (size_t)p * 6 * nt, sizeof(float) * 6 * nt);
    }

    struct geoprojection geop;
    set_geoproj(&m, &geop);
    struct sgtindex statindx, eqindx;
    statindx.h = ix[0].h;
    eqindx.h = ix[0].h;
    float sdep = 0.0f;
    get_indx(&slon, &slat, &sdep, &statindx, &geop);

    struct sgtparams *sp = (struct sgtparams *)calloc((size_t)(np ? np : 1), sizeof(*sp));
    float maxdelta = 0.0f, fweight = 1.0f;
    for (int ip = 0; ip < np; ip++) {
        float elon = pts[ip].lon, elat = pts[ip].lat, edep = pts[ip].dep;
        get_indx(&elon, &elat, &edep, &eqindx, &geop);
        find_sgt(&sp[ip], &m, ix, &eqindx, &statindx, &maxdelta, &fweight);
        for (int i = 0; i < sp[ip].nsgt; i++) {
            const int pos = find_pos(ix, globnp, sp[ip].indx[i]);
            if (pos < 0) return -1;
            sp[ip].sgt_head_ptrs[i] = hd + pos;
            sp[ip].sgtbuf_ptrs[i] = sgtbuf + (size_t)18 * nt * pos;
        }
    }

    /* jbsim3d.c:436-447 */
    int maxnt = hd[0].nt;
    const float mindt = hd[0].dt;
    if (dtout < mindt) maxnt = (maxnt * mindt / dtout);
    int ntsum = 2;
    while (ntsum < 4 * maxnt) ntsum = ntsum * 2;
    const int ntout = ntout_in > 0 ? ntout_in : ntsum;
    *ntout_out = ntout;

    const int maxmech = 3;
    float *gfmech = (float *)malloc(sizeof(float) * (size_t)maxmech * 12 * ntsum);
    float *space = (float *)malloc(sizeof(float) * 2 * (size_t)ntsum);
    float *subseis = (float *)malloc(sizeof(float) * (size_t)maxmech * 3 * ntout);
    float *stf = (float *)malloc(sizeof(float) * (size_t)ntout);
    struct standrupformat *srf = (struct standrupformat *)calloc((size_t)(nv ? nv : 1), sizeof(*srf));
    struct srf_apointvalues *apv = (struct srf_apointvalues *)calloc((size_t)nv * (np ? np : 1), sizeof(*apv));
    if (!gfmech || !space || !subseis || !stf || !srf || !apv) return -3;
    for (int v = 0; v < nv; v++) {
        srf[v].srf_apnts.np = np;
        srf[v].srf_apnts.apntvals = apv + (size_t)v * np;
        for (int ip = 0; ip < np; ip++) {
            const drv_point *a = &pts[(size_t)v * np + ip];
            struct srf_apointvalues *o = &apv[(size_t)v * np + ip];
            o->lon = a->lon, o->lat = a->lat, o->dep = a->dep, o->stk = a->stk, o->dip = a->dip;
            o->area = a->area, o->tinit = a->tinit, o->dt = a->dt, o->rake = a->rake;
            o->slip1 = a->slip1, o->nt1 = a->nt1, o->slip2 = a->slip2, o->nt2 = a->nt2;
            o->slip3 = a->slip3, o->nt3 = a->nt3;
            const float *vp = pool + pool_off[v];
            o->stf1 = (float *)(vp + a->stf1);
            o->stf2 = (float *)(vp + a->stf2);
            o->stf3 = (float *)(vp + a->stf3);
        }
    }
    memset(seis_out, 0, sizeof(float) * (size_t)nv * 3 * ntout);

    /* jbsim3d.c:480-520, points in rupture order */
    const float slip_conv = 1.0f;
    for (int ip = 0; ip < np; ip++)
        for (int v = 0; v < nv; v++) {
            struct mechparam mechpar;
            float rt, vslip, scale;
            zapit(subseis, maxmech * 3 * ntout);
            get_srfpars(&srf[v], 0, ip, &rt, &vslip, &mechpar.stk, &mechpar.dip, &mechpar.rak, &mechpar, 0);
            scale = slip_conv * srf[v].srf_apnts.apntvals[ip].area;
            mech_sgt(gfmech, &sp[ip], ntsum, mechpar, &scale);
            sum_sgt(subseis, ntout, gfmech, &sp[ip], ntsum, &rt, &tstart, mechpar, ip);
            srf_stf(&srf[v], 0, ip, seis_out + (size_t)v * 3 * ntout, subseis, stf, ntout, &dtout, mechpar, space);
        }
    free(gfmech), free(space), free(subseis), free(stf), free(srf), free(apv), free(sp);
    free(ix), free(hd), free(sgtbuf);
    return 0;
}
