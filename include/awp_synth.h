/*
 * awp_synth.h -- C ABI of the reciprocity seismogram synthesis in libawpsgt:
 * the consumer of the SGTs, CyberShake's DirectSynth worker step.
 *
 * DirectSynth (DirectSynth/src/synth.c:27-170 run_synth, jbsim/jbsim3d.c:40-577
 * jbsim3d_synth) turns the site's SGTs and a rupture's variations into one
 * seismogram per variation.  For every rupture point it finds the SGT
 * point(s) that bracket it (jbsim/sgt3d_subs.c:751-961 find_sgt), combines the
 * SGT with the point's fault mechanism (sgt3d_subs.c:1260-1422 mech_sgt),
 * tapers, time-shifts and sums the bracketing SGTs (sgt3d_subs.c:1121-1258
 * sum_sgt / timeshift_sgt) and convolves the result with the point's slip-rate
 * function into the seismogram (jbsim/srf_rupm.c:55-153 srf_stf,
 * jbsim/stf_subs.c:6-40 do_cnvlv).  The reference spreads the SGTs over MPI
 * "handler" ranks and streams them to workers; here the SGT set stays
 * resident in device memory and every variation of a rupture is synthesised
 * against it in one pass.
 *
 * Conventions shared with the reference:
 *   - SGT data per component is float32 [point][6][nt] in the RWG order of
 *     the .sgthead point list (the "separate header" files read by
 *     DirectSynth/src/sgt_handler.c:276-333);
 *   - the x component's SGT headers are used for every component, with ymom
 *     and zmom set to its xmom (synth.c:545-557), and the components' moments
 *     must agree (sgt_handler.c:226-242);
 *   - a seismogram is float32 [3][ntout] in the order vertical, north, east
 *     (sgt3d_subs.c:1190-1192); the output file keeps the components that
 *     the SGT files supply (jbsim3d.c:616-660);
 *   - rupture variations are SRF point lists (jbsim/srf_subs.c:521-690).
 *
 * Ownership and threading: a synthesis object owns its device memory (the SGT
 * set, per-chunk term buffers, the seismograms) and its three CUDA streams;
 * calls on one object must not overlap, separate objects may run from
 * separate host threads.  Errors are status codes with awp_last_error().
 *
 * Not on the path and rejected with AWP_ERR_PARAM: an SRF sample interval
 * that differs from dtout by more than the reference's 1e-5 ratio (the
 * reference resamples, srf_rupm.c:115-146; CyberShake generates the
 * variations at dtout so the branch is not taken), and map projections other
 * than geoproj 1 (great-circle arcs, the one CyberShake writes).
 */
#ifndef AWP_SYNTH_H
#define AWP_SYNTH_H

#include "awp_sgt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct awp_synth awp_synth;

typedef struct {
    int device;          /* CUDA device ordinal                                     */
    float slon, slat;    /* site longitude / latitude (synth.c:27 slon, slat)        */
    float dtout;         /* output sample interval, s (jbsim3d.c:136, required > 0)  */
    int ntout;           /* output samples; <= 0 selects ntsum (jbsim3d.c:441-447)   */
    float tstart;        /* start time of the output, s (jbsim3d.c:137, default 0)   */
    int rv_batch;        /* variations per device pass; 0 = all at once              */
} awp_synth_params;

/* One rupture point (jbsim/srf_structure.h srf_apointvalues).  stf1..3 are
 * offsets of the point's slip-rate samples in the variation's sample pool. */
typedef struct {
    float lon, lat, dep, stk, dip, area, tinit, dt, rake;
    float slip1, slip2, slip3;
    int nt1, nt2, nt3;
    long long stf1, stf2, stf3;
} awp_srf_point;

/* Seismogram record header (DirectSynth/src/jbsim/structure.h seisheader,
 * 56 bytes), written before every variation's samples. */
typedef struct {
    char version[8];
    char site_name[8];
    char padding[8];
    int source_id, rupture_id, rup_var_id;
    float dt;
    int nt, comps;
    float det_max_freq, stoch_max_freq;
} awp_seisheader;

typedef struct {
    int ntout;           /* samples per output component                        */
    int ntsum;           /* working length (power of two >= 4 * SGT nt)         */
    int nsgt_points;     /* distinct SGT points the rupture needs (synth.c nm)  */
    int non_exact;       /* rupture points without an exact SGT match           */
    int nvariations;     /* variations synthesised by the last run              */
    int ncomp;           /* SGT components loaded (1..3)                        */
    long long terms;     /* (variation, point, slip component) convolutions     */
    long long macs;      /* multiply-adds the convolutions performed (components
                            with SGTs; a run without z SGTs skips the vertical,
                            which is +0 throughout)                              */
    double seconds_plan; /* host set-up of the last run                         */
    double seconds_device; /* device time of the last run (events)              */
    double seconds_conv; /* device time of the convolution kernels              */
    int gpu_launches;    /* kernels launched by the last run                    */
    double seconds_gf;   /* device time of the SGT combination kernels          */
} awp_synth_info;

awp_status awp_synth_create(const awp_synth_params *p, awp_synth **out);
void awp_synth_destroy(awp_synth *s);

/* SGT set from host memory: the x component's master record, point index and
 * headers (globnp entries each) and ncomp data arrays of [globnp][6][nt]
 * floats for the x, y and z components in that order (y and z may be NULL
 * when ncomp is smaller).  The data is copied to the device; the arrays may be
 * freed on return.  Replaces get_SGT_data / readSGT_MPI
 * (DirectSynth/src/sgt_handler.c:202-333). */
awp_status awp_synth_set_sgt(awp_synth *s, const awp_sgtmaster *m, const awp_sgtindex *ix,
                             const awp_sgtheader *hd, int ncomp, const float *x, const float *y, const float *z);

/* The same from files: per component a .sgthead header file and its SGT data
 * file; the y and z pairs may be NULL.  Moments of the components must agree
 * (sgt_handler.c:226-242). */
awp_status awp_synth_load_sgt_files(awp_synth *s, const char *xhead, const char *xdata, const char *yhead,
                                    const char *ydata, const char *zhead, const char *zdata);

/* Adds one rupture variation: np points and the pool of slip-rate samples the
 * points' stf offsets index.  Every variation of a rupture has the same
 * point list; the first variation's positions place the points (synth.c:44-74
 * reads them from the rupture geometry file).  The data is copied. */
awp_status awp_synth_add_variation(awp_synth *s, int rup_var_id, const awp_srf_point *pts, int np,
                                   const float *pool, long long npool);

/* The same without a copy: the library reads pts and pool in place, so they
 * must stay valid and unchanged while the variation is listed, that is until
 * awp_synth_clear_variations or awp_synth_destroy (no reference
 * counterpart). */
awp_status awp_synth_add_variation_borrowed(awp_synth *s, int rup_var_id, const awp_srf_point *pts, int np,
                                            const float *pool, long long npool);

/* Reads an SRF file (text when binary == 0; jbsim/srf_subs.c:521-690) and adds
 * it as a variation. */
awp_status awp_synth_add_srf_file(awp_synth *s, int rup_var_id, const char *path, int binary);

/* Drops every variation added so far (the SGT set stays). */
awp_status awp_synth_clear_variations(awp_synth *s);

/* Synthesises every variation added: jbsim3d_synth's loop over rupture
 * points and variations (jbsim3d.c:339-577). */
awp_status awp_synth_run(awp_synth *s);

/* Seismograms of the last run: [nvariations][3][ntout] floats (vertical,
 * north, east), in the order the variations were added.  n is the capacity
 * of out in floats. */
awp_status awp_synth_seismograms(awp_synth *s, float *out, size_t n);

/* Writes the last run's seismograms as the reference's merged output: per
 * variation a seisheader (from tmpl, with rup_var_id, dt, nt and comps set)
 * followed by the components the SGTs supply (jbsim3d.c:616-660). */
awp_status awp_synth_write_grm(awp_synth *s, const char *path, const awp_seisheader *tmpl);

awp_status awp_synth_get_info(awp_synth *s, awp_synth_info *out);

/* SRF reader on its own: *pts and *pool are malloc'ed (free with awp_free). */
awp_status awp_srf_read(const char *path, int binary, awp_srf_point **pts, int *np, float **pool, long long *npool);

#ifdef __cplusplus
}
#endif
#endif /* AWP_SYNTH_H */
