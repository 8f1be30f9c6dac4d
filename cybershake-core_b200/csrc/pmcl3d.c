/*
 * pmcl3d.c -- drop-in driver for the AWP-ODC-SGT strain-Green-tensor run.
 *
 * Accepts both reference command lines:
 *   pmcl3d [IN3D [SOURCE [MEDIA [CHKP [CHKJ ...]]]]]     (AWP-ODC-SGT/src/set_names.f)
 *   pmcl3d -T <TMAX> --IGREEN <g> --DH .. -o <OUT> ...    (AWP-GPU-SGT/src/command.c)
 * and writes the same files:
 *   IN3D form: the raw SGT file SGTGRO with the offsets of pmcl3d.f:1589-1601,
 *              CHKP (io.f:481-536) and CHKJ (pmcl3d.f:1478-1479);
 *   GPU form:  OUT/SGT%07d per WRITE_STEP chunk, layout [point][6][WRITE_STEP]
 *              (AWP-GPU-SGT/src/pmcl3d.c:462-492, 932-958), and CHKFILE
 *              (AWP-GPU-SGT/src/io.c:7-35).
 * Everything runs on one GPU; NPX/NPY/NPZ are read and ignored.  With
 * AWP_RWG_SGT=x|y|z in the environment the SGTs are written in RWG component
 * order (SgtHead/src/reformat_awp_mpi.c:104-122), so no separate reformat
 * pass is needed.  With AWP_AUTOTUNE_CACHE=<file> the launch shapes are tuned
 * for the job's grid before the solve (awp_autotune on the homogeneous
 * medium, a few seconds once per grid and GPU model) and kept in that file.
 * CHECKPOINT > 0 in IN3D resumes from output_ckp/ when a checkpoint is there
 * and writes one every CHECKPOINT steps (pmcl3d.f:1018-1097, 1967-2045).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "../../include/awp_sgt.h"

static int fail(awp_status st, const char *what)
{
    fprintf(stderr, "pmcl3d: %s failed: %s (%s)\n", what, awp_status_string(st), awp_last_error());
    return 1;
}

/* Fortran Ew.d (d significant digits, leading "0.") */
static void fmt_e(char *out, size_t cap, double v, int w, int d)
{
    char body[64];
    if (v == 0.0 || !isfinite(v)) {
        if (!isfinite(v)) { snprintf(out, cap, "%*s", w, "NaN"); return; }
        char z[32];
        memset(z, '0', (size_t)d); z[d] = 0;
        snprintf(body, sizeof body, "0.%sE+00", z);
    } else {
        char tmp[64];
        snprintf(tmp, sizeof tmp, "%.*e", d - 1, fabs(v));   /* D.DDDe+XX */
        int ex = atoi(strchr(tmp, 'e') + 1) + 1;
        char dig[32];
        int n = 0;
        for (const char *p = tmp; *p && *p != 'e'; p++)
            if (*p >= '0' && *p <= '9') dig[n++] = *p;
        dig[n] = 0;
        if (ex >= -99 && ex <= 99)
            snprintf(body, sizeof body, "%s0.%sE%c%02d", v < 0 ? "-" : "", dig, ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
        else
            snprintf(body, sizeof body, "%s0.%s%c%03d", v < 0 ? "-" : "", dig, ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    }
    snprintf(out, cap, "%*s", w, body);
}

/* Fortran Gw.d: F editing, (d - k) decimals and four trailing blanks, when
 * the value rounded to d significant digits lies in [0.1, 10^d) with k its
 * number of integer digits (zero: F with d - 1 decimals); Ew.d otherwise */
static void fmt_g(char *out, size_t cap, double v, int w, int d)
{
    if (v == 0.0) { snprintf(out, cap, "%*.*f    ", w - 4, d - 1, 0.0); return; }
    char tmp[64];
    snprintf(tmp, sizeof tmp, "%.*e", d - 1, fabs(v));
    const int k = atoi(strchr(tmp, 'e') + 1) + 1;
    if (k >= 0 && k <= d) snprintf(out, cap, "%*.*f    ", w - 4, d - k, v);
    else fmt_e(out, cap, v, w, d);
}

/* Fortran Iw: asterisks when the number does not fit */
static const char *fmt_i(char *out, size_t cap, long v, int w)
{
    char tmp[32];
    const int n = snprintf(tmp, sizeof tmp, "%*ld", w, v);
    if (n > w) {
        memset(tmp, '*', (size_t)w);
        tmp[w] = 0;
    }
    snprintf(out, cap, "%s", tmp);
    return out;
}

static void mkdir_for(const char *path)
{
    char buf[1200];
    snprintf(buf, sizeof buf, "%s", path);
    for (char *p = buf + 1; *p; p++)
        if (*p == '/') { *p = 0; mkdir(buf, 0755); *p = '/'; }
}

static void write_chkp_fortran(const awp_in3d *in, const awp_stats *st)
{
    mkdir_for(in->chkp);
    FILE *f = fopen(in->chkp, "w");
    if (!f) return;
    char b1[64], b2[64], b3[64], ib[32];
    /* list-directed: blank, the string, a blank separator, I11 (gfortran) */
    fprintf(f, " igreen =  %11d\n", in->igreen);
    fmt_e(b1, sizeof b1, st->vp_max * in->dt / in->dh, 15, 7);
    fprintf(f, "STABILITY CRITERIA .5 > CMAX*DT/DX = %s\n", b1);
    fprintf(f, "# OF X NODES PER PROC%s\n", fmt_i(ib, sizeof ib, in->nx / (in->npx > 0 ? in->npx : 1), 5));
    fprintf(f, "# OF Y NODES PER PROC%s\n", fmt_i(ib, sizeof ib, in->ny / (in->npy > 0 ? in->npy : 1), 5));
    fprintf(f, "# OF Z NODES PER PROC%s\n", fmt_i(ib, sizeof ib, in->nz / (in->npz > 0 ? in->npz : 1), 5));
    fprintf(f, "# OF TIME STEPS%s\n", fmt_i(ib, sizeof ib, in->nt, 5));
    fprintf(f, "DISCRETIZATION IN SPACE%10.4f\n", in->dh);
    fprintf(f, "DISCRETIZATION IN TIME%10.4f\n", in->dt);
    fmt_g(b1, sizeof b1, in->arbc, 13, 4);
    fprintf(f, "PML REFLECTION COEFFICIENT%s\n", b1);
    fprintf(f, "HIGHEST P-VELOCITY ENCOUNTERED%10.2f\n", st->vp_max);
    fprintf(f, "LOWEST P-VELOCITY ENCOUNTERED%10.2f\n", st->vp_min);
    fprintf(f, "HIGHEST S-VELOCITY ENCOUNTERED%10.2f\n", st->vs_max);
    fprintf(f, "LOWEST S-VELOCITY ENCOUNTERED%10.2f\n", st->vs_min);
    fprintf(f, "HIGHEST DENSITY ENCOUNTERED%15.2f\n", st->rho_max);
    fprintf(f, "LOWEST  DENSITY ENCOUNTERED%15.2f\n", st->rho_min);
    fprintf(f, "SKIP OF SEISMOGRAMS IN TIME (LOOP COUNTER)%s\n", fmt_i(ib, sizeof ib, in->ntiskp, 5));
    fprintf(f, "ABC CONDITION, PML=1 OR CERJAN=0:%s\n", fmt_i(ib, sizeof ib, in->npc, 5));
    fprintf(f, "FD SCHEME, VISCO=1 OR ELASTIC=0:%s\n", fmt_i(ib, sizeof ib, in->nve, 5));
    fmt_g(b1, sizeof b1, in->fl, 14, 5);
    fmt_g(b2, sizeof b2, in->fp, 14, 5);
    fmt_g(b3, sizeof b3, in->fh, 14, 5);
    fprintf(f, "Q, FL,FP,FH:%s%s%s\n", b1, b2, b3);
    fclose(f);
}

static void write_chkp_gpu(const awp_in3d *in, const awp_stats *st)
{
    mkdir_for(in->chkp);
    FILE *f = fopen(in->chkp, "w");
    if (!f) return;
    fprintf(f, "STABILITY CRITERIA .5 > CMAX*DT/DX:\t%f\n", st->vp_max * in->dt / in->dh);
    fprintf(f, "# OF X,Y,Z NODES PER PROC:\t%d, %d, %d\n", in->nx, in->ny, in->nz);
    fprintf(f, "# OF TIME STEPS:\t%d\n", in->nt);
    fprintf(f, "DISCRETIZATION IN SPACE:\t%f\n", in->dh);
    fprintf(f, "DISCRETIZATION IN TIME:\t%f\n", in->dt);
    fprintf(f, "PML REFLECTION COEFFICIENT:\t%f\n", in->arbc);
    fprintf(f, "HIGHEST P-VELOCITY ENCOUNTERED:\t%f\n", st->vp_max);
    fprintf(f, "LOWEST P-VELOCITY ENCOUNTERED:\t%f\n", st->vp_min);
    fprintf(f, "HIGHEST S-VELOCITY ENCOUNTERED:\t%f\n", st->vs_max);
    fprintf(f, "LOWEST S-VELOCITY ENCOUNTERED:\t%f\n", st->vs_min);
    fprintf(f, "HIGHEST DENSITY ENCOUNTERED:\t%f\n", st->rho_max);
    fprintf(f, "LOWEST  DENSITY ENCOUNTERED:\t%f\n", st->rho_min);
    fprintf(f, "SKIP OF SEISMOGRAMS IN TIME (LOOP COUNTER):\t%d\n", in->ntiskp);
    fprintf(f, "ABC CONDITION, PML=1 OR CERJAN=0:\t%d\n", in->npc);
    fprintf(f, "FD SCHEME, VISCO=1 OR ELASTIC=0:\t%d\n", in->nve);
    fprintf(f, "Q, FL,FP,FH:\t%f, %f, %f\n", in->fl, in->fp, in->fh);
    fclose(f);
}

/* Surface velocity recording of the GPU command line, one rank
 * (AWP-GPU-SGT/src/pmcl3d.c:300-320, calcRecordingPoints :1336-1395 and the
 * NTISKP block :962-1031): after every step that is a multiple of NTISKP,
 * u1 v1 w1 on the NBG*:NSKP*:NED* window (z counted in depth from the free
 * surface, z = 1 the surface) are stored as sample (step/NTISKP - 1) mod
 * WRITE_STEP of a buffer [WRITE_STEP][depth][y][x] per component; a full
 * buffer goes to OUT/SX%07ld, SY, SZ named by the step.  The CHKFILE gets
 * "step :\tu\tv\tw" at x = y = ND+1, depth ND below the surface, and "END"
 * when the run is over. */
typedef struct {
    int bg[3], skp[3], cnt[3];   /* 0-based first index, stride, count: x, y, depth */
    int ws;
    size_t rec;                  /* floats per sample and component */
    float *buf[3], *plane;
    FILE *chk;
} surf_rec;

/* rec_nbg / rec_ned / rec_n* of calcRecordingPoints for the one rank that
 * holds the whole axis of n points */
static int rec_axis(int n, int nbg, int ned, int nskp, int lateral, int *bg, int *cnt)
{
    if (ned == -1) ned = n;
    if (nskp < 1 || nbg < 1) return -1;
    ned = ned - (ned - nbg) % nskp;
    *bg = nbg - 1;
    if (nbg > n || (lateral && ned < 1)) { *cnt = 0; return 0; }
    int ed;
    if (!lateral) ed = ned - 1;
    else if (n <= ned) ed = (n + nbg - 1) % nskp - nskp + n;
    else ed = ned - 1;
    if (ed > n - 1) return -1;
    *cnt = ed < *bg ? 0 : (ed - *bg) / nskp + 1;
    return 0;
}

static int surf_open(surf_rec *r, const awp_in3d *in, const awp_params *p)
{
    memset(r, 0, sizeof *r);
    const int n[3] = {p->nx, p->ny, p->nz};
    const int bg[3] = {in->nbgx, in->nbgy, in->nbgz}, ed[3] = {in->nedx, in->nedy, in->nedz};
    const int sk[3] = {in->nskpx, in->nskpy, in->nskpz};
    for (int a = 0; a < 3; a++) {
        r->skp[a] = sk[a];
        if (rec_axis(n[a], bg[a], ed[a], sk[a], a < 2, &r->bg[a], &r->cnt[a]) != 0) {
            fprintf(stderr, "pmcl3d: recording window NBG/NED/NSKP outside the grid on axis %c\n", "XYZ"[a]);
            return -1;
        }
    }
    if (!r->cnt[0] || !r->cnt[1] || !r->cnt[2]) r->cnt[0] = r->cnt[1] = r->cnt[2] = 0;
    r->ws = p->write_step > 0 ? p->write_step : 1;
    r->rec = (size_t)r->cnt[0] * r->cnt[1] * r->cnt[2];
    for (int c = 0; c < 3; c++) r->buf[c] = (float *)calloc(r->rec * r->ws + 1, sizeof(float));
    r->plane = (float *)malloc(sizeof(float) * (size_t)p->nx * p->ny);
    r->chk = fopen(in->chkp, "a");
    if (!r->buf[0] || !r->buf[1] || !r->buf[2] || !r->plane) return -1;
    return 0;
}

static int surf_record(surf_rec *r, awp_solver *s, const awp_in3d *in, const awp_params *p, int step)
{
    static const char *base[3] = {"SX", "SY", "SZ"};
    const int sample = (step / in->ntiskp + r->ws - 1) % r->ws;
    float probe[3] = {0, 0, 0};
    const int kp = p->nz - in->nd;
    for (int c = 0; c < 3; c++) {
        float *dst = r->buf[c] + (size_t)sample * r->rec;
        for (int dz = 0; dz < r->cnt[2]; dz++) {
            if (awp_get_plane(s, 0, c, p->nz - (r->bg[2] + dz * r->skp[2]), r->plane) != AWP_OK) return -1;
            for (int jy = 0; jy < r->cnt[1]; jy++)
                for (int ix = 0; ix < r->cnt[0]; ix++)
                    *dst++ = r->plane[(size_t)(r->bg[1] + jy * r->skp[1]) * p->nx + r->bg[0] + ix * r->skp[0]];
        }
        if (r->chk && kp >= 1 && in->nd < p->nx && in->nd < p->ny) {
            if (awp_get_plane(s, 0, c, kp, r->plane) != AWP_OK) return -1;
            probe[c] = r->plane[(size_t)in->nd * p->nx + in->nd];
        }
    }
    if (r->chk) {
        fprintf(r->chk, "%ld :\t%e\t%e\t%e\n", (long)step, probe[0], probe[1], probe[2]);
        fflush(r->chk);
    }
    if ((step / in->ntiskp) % r->ws == 0) {
        for (int c = 0; c < 3; c++) {
            char name[1100];
            snprintf(name, sizeof name, "%s/%s%07ld", in->out_dir, base[c], (long)step);
            mkdir_for(name);
            FILE *f = fopen(name, "wb");
            if (!f || fwrite(r->buf[c], sizeof(float), r->rec * r->ws, f) != r->rec * r->ws) {
                fprintf(stderr, "pmcl3d: cannot write %s\n", name);
                if (f) fclose(f);
                return -1;
            }
            fclose(f);
        }
    }
    return 0;
}

static void surf_close(surf_rec *r)
{
    if (r->chk) { fprintf(r->chk, "END\n"); fclose(r->chk); }
    for (int c = 0; c < 3; c++) free(r->buf[c]);
    free(r->plane);
}

static int write_chkj(const char *path, const float *chkj, int nt)
{
    mkdir_for(path);
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    char a[32], b[32], c[32];
    for (int i = 0; i < nt; i++) {
        fmt_e(a, sizeof a, chkj[3 * i], 10, 3);
        fmt_e(b, sizeof b, chkj[3 * i + 1], 10, 3);
        fmt_e(c, sizeof c, chkj[3 * i + 2], 10, 3);
        char ib[32];
        fprintf(f, "%s%s%s%s\n", fmt_i(ib, sizeof ib, i + 1, 6), a, b, c);
    }
    fclose(f);
    return 0;
}

int main(int argc, char **argv)
{
    awp_in3d in;
    awp_status st = awp_parse_command_line(argc, argv, &in);
    if (st != AWP_OK) return fail(st, "reading parameters");
    if (in.ifault != 0 && in.ifault != 1 && in.ifault != 5) {
        fprintf(stderr, "pmcl3d: IFAULT=%d is not supported (0, 1 or 5)\n", in.ifault);
        return 1;
    }
    if (in.ifault == 5 && in.nst != 2) {   /* AWP-GPU-SGT/src/pmcl3d.c:509-515 */
        fprintf(stderr, "pmcl3d: IFAULT=5 requires NST = READ_STEP = 2\n");
        return 1;
    }

    awp_params p;
    awp_params_from_in3d(&in, &p);
    const char *dev = getenv("AWP_DEVICE");
    if (dev) p.device = atoi(dev);

    int *sxyz = (int *)malloc(sizeof(int) * 3 * (size_t)(in.nsrc > 0 ? in.nsrc : 1));
    float *stf = (float *)malloc(sizeof(float) * 6 * (size_t)(in.nsrc > 0 ? in.nsrc : 1) * (size_t)(in.nst > 0 ? in.nst : 1));
    st = awp_read_source(in.insrc, in.ifault, in.nsrc, in.nst, sxyz, stf);
    if (st != AWP_OK) return fail(st, "reading the source");

    int npts = 0, *pxyz = NULL;
    if (in.igreen != -1) {
        FILE *t = fopen(in.insgt, "r");   /* io.f:422-440: no cordfile -> no SGT output */
        if (t) {
            fclose(t);
            st = awp_read_cordfile(in.insgt, &npts, &pxyz);
            if (st != AWP_OK) return fail(st, "reading the cordfile");
            printf("Use SGT output mode, sgt_numsta=%d\n", npts);
        } else {
            printf("Station list does not exist. Use normal output mode\n");
        }
    }

    awp_tuning tuned;
    const char *tune_cache = getenv("AWP_AUTOTUNE_CACHE");
    if (tune_cache && *tune_cache) {
        double rate = 0.0;
        if ((st = awp_autotune(&p, NULL, 20, tune_cache, &tuned, &rate)) != AWP_OK) return fail(st, "tuning");
        printf("Launch shapes tuned: %.2f Gcell-updates/s in trial (cache %s)\n", rate, tune_cache);
    }

    awp_solver *s = NULL;
    if ((st = awp_create(&p, &s)) != AWP_OK) return fail(st, "creating the solver");
    if (tune_cache && *tune_cache && (st = awp_set_tuning(s, &tuned)) != AWP_OK) return fail(st, "applying the tuning");
    /* MEDIASTART 1 and 2 read INVEL; 3 reads the rank's partition file, which
     * on one GPU is the whole domain (AWP-GPU-SGT/src/mesh.c:97-118) */
    const char *media_path = p.mediastart == 3 ? "input_rst/mediapart/media0000000.bin" : in.invel;
    if ((st = awp_load_media_file(s, media_path)) != AWP_OK) return fail(st, "loading the media");
    if ((st = awp_set_source(s, 0, in.nsrc, sxyz, stf)) != AWP_OK) return fail(st, "setting the source");
    if ((st = awp_set_points(s, npts, pxyz)) != AWP_OK) return fail(st, "setting the SGT points");

    awp_stats stats;
    awp_get_stats(s, &stats);
    if (in.gpu_cli) write_chkp_gpu(&in, &stats);
    else write_chkp_fortran(&in, &stats);

    /* pmcl3d.f:1018-1097: with CHECKPOINT > 0 resume from output_ckp/ when a
     * checkpoint is there; pmcl3d.f:1967-2045: a checkpoint after every step i
     * with mod(i, CHECKPOINT) == 0.  The GPU command line records the surface
     * every NTISKP steps.  The time loop runs in segments between those
     * steps. */
    int t0 = 0;
    if (in.checkpoint > 0) {
        mkdir("output_ckp", 0755);
        if ((st = awp_checkpoint_read(s, "output_ckp", &t0)) != AWP_OK) return fail(st, "reading the checkpoint");
        if (t0 > 0) printf("Checkpoint found, starting from step %d\n", t0);
    }
    surf_rec rec;
    const int rec_every = in.gpu_cli && in.ntiskp > 0 ? in.ntiskp : 0;
    if (in.gpu_cli && surf_open(&rec, &in, &p) != 0) return fail(AWP_ERR_PARAM, "setting up the surface recording");
    if (!in.gpu_cli && in.ntiskp > 0 && in.ntiskp <= p.nt)
        fprintf(stderr, "pmcl3d: NTISKP %d <= NT: the IN3D form's velocity output files are not written\n", in.ntiskp);
    for (int done = t0; done < p.nt;) {
        int n = p.nt - done;
        if (in.checkpoint > 0 && in.checkpoint - done % in.checkpoint < n) n = in.checkpoint - done % in.checkpoint;
        if (rec_every && rec_every - done % rec_every < n) n = rec_every - done % rec_every;
        if ((st = awp_run(s, n, NULL)) != AWP_OK) return fail(st, "time stepping");
        done += n;
        if (in.checkpoint > 0 && done % in.checkpoint == 0) {
            printf("Writing checkpoint file\n");
            if ((st = awp_checkpoint_write(s, "output_ckp")) != AWP_OK) return fail(st, "writing the checkpoint");
        }
        if (rec_every && done % rec_every == 0 && surf_record(&rec, s, &in, &p, done) != 0)
            return fail(AWP_ERR_IO, "recording the surface");
    }
    if (in.gpu_cli) surf_close(&rec);
    awp_get_stats(s, &stats);
    printf("time loop: %d steps in %.3f s, %.3f Gcell-updates/s\n", (int)stats.steps_done, stats.seconds_loop,
           stats.gcell_updates_per_s);

    if (!in.gpu_cli) {
        float *chkj = (float *)malloc(sizeof(float) * 3 * (size_t)p.nt);
        if ((st = awp_get_chkj(s, 0, chkj)) != AWP_OK) return fail(st, "reading CHKJ");
        write_chkj(in.chkj, chkj, p.nt);
        free(chkj);
    }

    if (npts > 0 && in.io_opt == 1) {
        const int64_t nf = awp_sgt_file_floats(s);
        float *img = (float *)malloc(sizeof(float) * (size_t)(nf > 0 ? nf : 1));
        /* AWP_RWG_SGT=x|y|z: the file image in RWG order (the z-force run scaled
         * by -2), which folds SgtHead's reformat_awp pass into the run */
        const char *rwg = getenv("AWP_RWG_SGT");
        if (rwg && *rwg) st = awp_get_sgt_rwg(s, 0, rwg[0] == 'z', img);
        else st = awp_get_sgt(s, 0, img);
        if (st != AWP_OK) return fail(st, "reading the SGTs");
        if (!in.gpu_cli) {
            mkdir_for(in.sgtgro);
            FILE *f = fopen(in.sgtgro, "wb");
            if (!f || fwrite(img, sizeof(float), (size_t)nf, f) != (size_t)nf) { fprintf(stderr, "pmcl3d: cannot write %s\n", in.sgtgro); return 1; }
            fclose(f);
        } else {
            /* one file per WRITE_STEP chunk, [point][6][WRITE_STEP] */
            const int ws = p.write_step;
            const int nchunk = (p.nt / p.ntiskp_sgt) / ws;
            const int64_t ntf = ((int64_t)(p.nt / ws) * ws) / p.ntiskp_sgt;
            float *chunk = (float *)malloc(sizeof(float) * (size_t)npts * 6 * (size_t)ws);
            for (int c = 0; c < nchunk; c++) {
                for (int n = 0; n < npts; n++)
                    for (int q = 0; q < 6; q++) {
                        int64_t off = (int64_t)n * 6 * ntf + (int64_t)q * ntf + (int64_t)c * ws;
                        memcpy(chunk + ((size_t)n * 6 + q) * ws, img + off, sizeof(float) * (size_t)ws);
                    }
                char name[1100];
                snprintf(name, sizeof name, "%s/SGT%07ld", in.out_dir, (long)(c + 1) * ws * p.ntiskp_sgt);
                mkdir_for(name);
                FILE *f = fopen(name, "wb");
                if (!f || fwrite(chunk, sizeof(float), (size_t)npts * 6 * ws, f) != (size_t)npts * 6 * ws) {
                    fprintf(stderr, "pmcl3d: cannot write %s\n", name);
                    return 1;
                }
                fclose(f);
            }
            free(chunk);
        }
        free(img);
    }
    awp_destroy(s);
    free(sxyz); free(stf); free(pxyz);
    return 0;
}
