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

/* Fortran Gw.d for the magnitudes CHKP prints */
static void fmt_g(char *out, size_t cap, double v, int w, int d)
{
    double a = fabs(v);
    if (a >= 0.1 && a < pow(10.0, d)) {
        int e = (int)floor(log10(a)) + 1;
        char f[64];
        snprintf(f, sizeof f, "%*.*f    ", w - 4, d - e, v);
        snprintf(out, cap, "%s", f);
    } else {
        fmt_e(out, cap, v, w, d);
    }
}

static void mkdir_for(const char *path)
{
    char buf[1024];
    snprintf(buf, sizeof buf, "%s", path);
    for (char *p = buf + 1; *p; p++)
        if (*p == '/') { *p = 0; mkdir(buf, 0755); *p = '/'; }
}

static void write_chkp_fortran(const awp_in3d *in, const awp_stats *st)
{
    mkdir_for(in->chkp);
    FILE *f = fopen(in->chkp, "w");
    if (!f) return;
    char b1[64], b2[64], b3[64];
    fprintf(f, " igreen = %11d\n", in->igreen);
    fmt_e(b1, sizeof b1, st->vp_max * in->dt / in->dh, 15, 7);
    fprintf(f, "STABILITY CRITERIA .5 > CMAX*DT/DX = %s\n", b1);
    fprintf(f, "# OF X NODES PER PROC%5d\n", in->nx / (in->npx > 0 ? in->npx : 1));
    fprintf(f, "# OF Y NODES PER PROC%5d\n", in->ny / (in->npy > 0 ? in->npy : 1));
    fprintf(f, "# OF Z NODES PER PROC%5d\n", in->nz / (in->npz > 0 ? in->npz : 1));
    fprintf(f, "# OF TIME STEPS%5d\n", in->nt);
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
    fprintf(f, "SKIP OF SEISMOGRAMS IN TIME (LOOP COUNTER)%5d\n", in->ntiskp);
    fprintf(f, "ABC CONDITION, PML=1 OR CERJAN=0:%5d\n", in->npc);
    fprintf(f, "FD SCHEME, VISCO=1 OR ELASTIC=0:%5d\n", in->nve);
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
        fprintf(f, "%6d%s%s%s\n", i + 1, a, b, c);
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

    if (in.checkpoint > 0) {
        /* pmcl3d.f:1018-1097: resume from output_ckp/ when a checkpoint is
         * there; pmcl3d.f:1967-2045: a checkpoint after every step i with
         * mod(i, CHECKPOINT) == 0 */
        mkdir("output_ckp", 0755);
        int t0 = 0;
        if ((st = awp_checkpoint_read(s, "output_ckp", &t0)) != AWP_OK) return fail(st, "reading the checkpoint");
        if (t0 > 0) printf("Checkpoint found, starting from step %d\n", t0);
        for (int done = t0; done < p.nt;) {
            int n = in.checkpoint - done % in.checkpoint;
            if (n > p.nt - done) n = p.nt - done;
            if ((st = awp_run(s, n, NULL)) != AWP_OK) return fail(st, "time stepping");
            done += n;
            if (done % in.checkpoint == 0) {
                printf("Writing checkpoint file\n");
                if ((st = awp_checkpoint_write(s, "output_ckp")) != AWP_OK) return fail(st, "writing the checkpoint");
            }
        }
    } else if ((st = awp_run(s, p.nt, NULL)) != AWP_OK) {
        return fail(st, "time stepping");
    }
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
