/*
 * awp_synth_internal.h -- records shared by the synthesis set-up (C, host)
 * and its kernels (CUDA).
 *
 * One "term" is one (rupture variation, rupture point, slip component): the
 * unit jbsim3d_synth handles with one mech_sgt + timeshift_sgt + do_cnvlv
 * sequence (DirectSynth/src/jbsim/jbsim3d.c:480-520, srf_rupm.c:95-151).
 */
#ifndef AWP_SYNTH_INTERNAL_H
#define AWP_SYNTH_INTERNAL_H

#include "../../include/awp_synth.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { SY_MXX, SY_MYY, SY_MZZ, SY_MXY, SY_MXZ, SY_MYZ, SY_XAMP, SY_YAMP, SY_ZAMP, SY_COSA, SY_SINA, SY_NC };
#define SY_TAPLEN 10          /* samples of the cosine taper at the end of an SGT (sgt3d_subs.c:1186) */

/* what the first kernel needs of a term: the bracketing SGT points, their
 * shifts and the mechanism coefficients of mech_sgt for each */
typedef struct {
    int nsgt;
    int pt[4];                /* position of the SGT point in the device set      */
    int shift[4];             /* itshift (sgt3d_subs.c:1215-1219)                 */
    int lo[4], hi[4];         /* output samples [lo, hi) the SGT reaches          */
    float c[4][SY_NC];
} awp_synth_gterm;

/* what the convolution needs: the slip-rate samples (already times dtout) */
typedef struct {
    long long stf;            /* offset in the run's sample pool                  */
    int nstf;
    int lo, hi;               /* output samples the SGTs reach; the rest are +0   */
    int slot;                 /* where the combination kernel put the trace       */
} awp_synth_cterm;

typedef struct {
    float lon, lat, dep;
} awp_synth_loc;

/* geoproj 1 projection and grid lookup (DirectSynth/src/jbsim/geoproj_subs.c,
 * misc_subs.c:151-173) */
typedef struct {
    double amat[9], ainv[9];
    double g0, b0;
    float erad;
} awp_synth_geo;

awp_status awp_synth_geo_init(const awp_sgtmaster *m, awp_synth_geo *g);
void awp_synth_get_indx(const awp_synth_geo *g, float lon, float lat, float dep, float h, awp_sgtindex *out);

/* bracketing SGT points of one rupture point (sgt3d_subs.c:751-961) */
typedef struct {
    int nsgt;
    long long indx[4];
    float wt[4];
    int pos[4];               /* position in the SGT index                        */
} awp_synth_bracket;

void awp_synth_find_sgt(const awp_sgtindex *ix, int np, const awp_sgtindex *eq, const awp_sgtindex *stat,
                        awp_synth_bracket *out);

/* One variation's terms for points ip0 .. ip1 - 1: for each point in order,
 * its slip components.
 * gt/ct/stf are caller-sized with awp_synth_count_terms / pool sizes.
 * Returns AWP_OK or AWP_ERR_PARAM (text set) on an SRF the path rejects. */
typedef struct {
    const awp_sgtheader *hd;  /* x-component headers, moments already fixed       */
    const awp_synth_bracket *br;
    int np;
    int nt, ntsum, ntout;
    float dtout, tstart;
    const float *taper;       /* SY_TAPLEN factors, index it - tapst              */
} awp_synth_plan_ctx;

long long awp_synth_count_terms(const awp_srf_point *pts, int np);
awp_status awp_synth_plan_variation(const awp_synth_plan_ctx *cx, const awp_srf_point *pts, const float *pool,
                                    long long npool, int ip0, int ip1, awp_synth_gterm *gt, awp_synth_cterm *ct,
                                    float *stf, long long stf_base, long long *nterms, long long *nstf_used,
                                    long long *macs);

void awp_synth_taper(int nt, float *fac);

#ifdef __cplusplus
}
#endif
#endif /* AWP_SYNTH_INTERNAL_H */
