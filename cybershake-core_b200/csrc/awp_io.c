/*
 * awp_io.c -- reference file formats and command lines of the pmcl3d driver.
 *
 *   IN3D reader          AWP-ODC-SGT/src/io.f:327-441 (ordered list-directed reads)
 *   positional CLI       AWP-ODC-SGT/src/set_names.f:17-50, io.f:459-479
 *   GPU getopt CLI       AWP-GPU-SGT/src/command.c:60-340
 *   source file          AWP-ODC-SGT/src/source.f:170-198 (IFAULT 0, text)
 *                        AWP-GPU-SGT/src/source.c:52-71    (IFAULT 1, binary)
 *   cordfile             AWP-ODC-SGT/src/io.f:420-441, AWP-GPU-SGT/src/sgt.c:24-32
 */
#define _GNU_SOURCE
#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/awp_sgt.h"

/* the error text is kept by the solver translation unit (awp_last_error) */
void awp_set_error_text(const char *msg);

static awp_status ioerr(awp_status st, const char *fmt, const char *a)
{
    char buf[512];
    snprintf(buf, sizeof buf, fmt, a ? a : "");
    awp_set_error_text(buf);
    return st;
}

/* ------------------------------------------------------------------ */
/* IN3D                                                                */
/* ------------------------------------------------------------------ */

typedef enum { T_INT, T_REAL, T_STR } ftype;
typedef struct { const char *name; ftype t; size_t off; } field;

#define FI(n, m) {n, T_INT, offsetof(awp_in3d, m)}
#define FR(n, m) {n, T_REAL, offsetof(awp_in3d, m)}
#define FS(n, m) {n, T_STR, offsetof(awp_in3d, m)}

/* exact read order of rddt3d, io.f:327-417 */
static const field in3d_fields[] = {
    FI("igreen", igreen), FR("TMAX", tmax), FR("DH", dh), FR("DT", dt), FI("NPC", npc),
    FI("ND", nd), FR("ARBC", arbc), FR("PHT", pht),
    FI("NSRC", nsrc), FI("NST", nst),
    FI("NX", nx), FI("NY", ny), FI("NZ", nz),
    FI("NPX", npx), FI("NPY", npy), FI("NPZ", npz),
    FI("IFAULT", ifault), FI("CHECKPOINT", checkpoint), FI("ISFCVLM", isfcvlm), FI("IMD5", imd5),
    FI("IVELOCITY", ivelocity), FI("MEDIARESTART", mediarestart), FI("NVAR", nvar), FI("IOST", iost),
    FI("PARTDEG", partdeg), FI("IO_OPT", io_opt), FI("PERF_MEAS", iperf), FI("IDYNA", idyna),
    FI("SOCALQ", socalq),
    FI("NVE", nve),
    FR("MU_S", mu_s), FR("MU_D", mu_d),
    FR("FL", fl), FR("FH", fh), FR("FP", fp),
    FI("READ_STEP", read_step), FI("WRITE_STEP", write_step), FI("WRITE_STEP2", write_step2),
    FI("NBGX", nbgx), FI("NEDX", nedx), FI("NSKPX", nskpx),
    FI("NBGY", nbgy), FI("NEDY", nedy), FI("NSKPY", nskpy),
    FI("NBGZ", nbgz), FI("NEDZ", nedz), FI("NSKPZ", nskpz),
    FI("NTISKP", ntiskp),
    FI("NBGX2", nbgx2), FI("NEDX2", nedx2), FI("NSKPX2", nskpx2),
    FI("NBGY2", nbgy2), FI("NEDY2", nedy2), FI("NSKPY2", nskpy2),
    FI("NBGZ2", nbgz2), FI("NEDZ2", nedz2), FI("NSKPZ2", nskpz2),
    FI("NTISKP2", ntiskp2), FI("NTISKP_SGT", ntiskp_sgt),
    FS("CHKP", chkp), FS("CHKJ", chkj), FS("INSRC", insrc), FS("INVEL", invel), FS("INSGT", insgt),
    FS("SXGRO", sxgro), FS("SYGRO", sygro), FS("SZGRO", szgro),
    FS("SXGRO2", sxgro2), FS("SYGRO2", sygro2), FS("SZGRO2", szgro2),
    FS("SGTGRO", sgtgro), FS("SGSN", sgsn),
};

/* first list-directed item of a line: a quoted string, or text up to a blank
 * or comma.  Returns 0 for a blank line. */
static int first_item(const char *line, char *out, size_t cap)
{
    const char *p = line;
    while (*p && isspace((unsigned char)*p)) p++;
    if (!*p) return 0;
    size_t n = 0;
    if (*p == '\'' || *p == '"') {
        char q = *p++;
        while (*p && *p != q && n + 1 < cap) out[n++] = *p++;
    } else {
        while (*p && !isspace((unsigned char)*p) && *p != ',' && n + 1 < cap) out[n++] = *p++;
    }
    out[n] = 0;
    return 1;
}

/* Fortran reads of REAL accept d/D exponents */
static double fortran_real(const char *s, int *ok)
{
    char buf[128];
    size_t n = strlen(s);
    if (n >= sizeof buf) { *ok = 0; return 0; }
    for (size_t i = 0; i <= n; i++) buf[i] = (s[i] == 'd' || s[i] == 'D') ? 'e' : s[i];
    char *end;
    errno = 0;
    double v = strtod(buf, &end);
    *ok = (end != buf && *end == 0 && errno == 0);
    return v;
}

static int nint_f(float x) { return (int)(x >= 0 ? floorf(x + 0.5f) : -floorf(-x + 0.5f)); }

awp_status awp_read_in3d(const char *path, awp_in3d *o)
{
    memset(o, 0, sizeof *o);
    FILE *f = fopen(path, "r");
    if (!f) return ioerr(AWP_ERR_IO, "cannot open IN3D file %s", path);
    char line[4096], item[1024];
    size_t nf = sizeof in3d_fields / sizeof in3d_fields[0];
    size_t k = 0;
    while (k < nf && fgets(line, sizeof line, f)) {
        if (!first_item(line, item, sizeof item)) continue;   /* blank record */
        const field *fd = &in3d_fields[k];
        char *dst = (char *)o + fd->off;
        int ok = 1;
        if (fd->t == T_INT) {
            char *end;
            long v = strtol(item, &end, 10);
            if (end == item || *end) ok = 0;
            *(int *)dst = (int)v;
        } else if (fd->t == T_REAL) {
            *(float *)dst = (float)fortran_real(item, &ok);
        } else {
            /* string fields are 512 bytes: longer names are cut there */
            snprintf(dst, 512, "%.511s", item);
        }
        if (!ok) { fclose(f); return ioerr(AWP_ERR_IO, "IN3D: bad value for %s", fd->name); }
        k++;
    }
    fclose(f);
    if (k < nf) return ioerr(AWP_ERR_IO, "IN3D: file ends before %s", in3d_fields[k].name);
    o->nt = nint_f(o->tmax / o->dt) + 1;   /* pmcl3d.f:287 */
    o->gpu_cli = 0;
    return AWP_OK;
}

/* ------------------------------------------------------------------ */
/* command lines                                                       */
/* ------------------------------------------------------------------ */

typedef struct { const char *lng; char shrt; ftype t; size_t off; } opt;
#define OI(l, s, m) {l, s, T_INT, offsetof(awp_in3d, m)}
#define OR(l, s, m) {l, s, T_REAL, offsetof(awp_in3d, m)}
#define OS(l, s, m) {l, s, T_STR, offsetof(awp_in3d, m)}

/* long options of AWP-GPU-SGT/src/command.c:144-188 */
static const opt gpu_opts[] = {
    OR("TMAX", 'T', tmax), OR("DH", 'H', dh), OR("DT", 't', dt), OR("ARBC", 'A', arbc), OR("PHT", 'P', pht),
    OI("NPC", 'M', npc), OI("ND", 'D', nd), OI("NSRC", 'S', nsrc), OI("NST", 'N', nst), OI("NVE", 'V', nve),
    OI("MEDIASTART", 'B', mediarestart), OI("NVAR", 'n', nvar), OI("IFAULT", 'I', ifault),
    OI("READ_STEP", 'R', read_step), OI("READ_STEP_GPU", 'Q', read_step),
    OI("NX", 'X', nx), OI("NY", 'Y', ny), OI("NZ", 'Z', nz), OI("PX", 'x', npx), OI("PY", 'y', npy),
    OI("NBGX", 0, nbgx), OI("NEDX", 0, nedx), OI("NSKPX", 0, nskpx),
    OI("NBGY", 0, nbgy), OI("NEDY", 0, nedy), OI("NSKPY", 0, nskpy),
    OI("NBGZ", 0, nbgz), OI("NEDZ", 0, nedz), OI("NSKPZ", 0, nskpz),
    OI("IDYNA", 'i', idyna), OI("SoCalQ", 's', socalq), OR("FL", 'l', fl), OR("FH", 'h', fh), OR("FP", 'p', fp),
    OI("NTISKP", 'r', ntiskp), OI("WRITE_STEP", 'W', write_step),
    OS("INSRC", 0, insrc), OS("INVEL", 0, invel), OS("OUT", 'o', out_dir), OS("CHKFILE", 'c', chkp),
    OI("IGREEN", 'G', igreen), OI("NTISKP_SGT", 0, ntiskp_sgt), OS("INSGT", 0, insgt),
};

static void gpu_defaults(awp_in3d *o)
{
    /* AWP-GPU-SGT/src/command.c:60-115 */
    memset(o, 0, sizeof *o);
    o->tmax = 20.0f; o->dh = 200.0f; o->dt = 0.01f; o->arbc = 0.92f; o->pht = 0.1f;
    o->npc = 0; o->nd = 20; o->nsrc = 1; o->nst = 91; o->nvar = 3; o->nve = 1;
    o->mediarestart = 0; o->ifault = 1; o->read_step = 91; o->ntiskp = 10; o->write_step = 10;
    o->nx = 224; o->ny = 224; o->nz = 1024; o->npx = 1; o->npy = 1; o->npz = 1;
    o->nbgx = 1; o->nedx = -1; o->nskpx = 1; o->nbgy = 1; o->nedy = -1; o->nskpy = 1;
    o->nbgz = 1; o->nedz = 1; o->nskpz = 1;
    o->idyna = 0; o->socalq = 1; o->fl = 0.005f; o->fh = 5.0f; o->fp = 2.5f;
    snprintf(o->insrc, sizeof o->insrc, "input/FAULTPOW");
    snprintf(o->invel, sizeof o->invel, "input/media");
    snprintf(o->out_dir, sizeof o->out_dir, "output_sfc");
    snprintf(o->chkp, sizeof o->chkp, "output_sfc/CHKP");
    o->igreen = -1; o->ntiskp_sgt = 1;
    snprintf(o->insgt, sizeof o->insgt, "input/SGT");
    o->io_opt = 1;
}

static int set_opt(awp_in3d *o, const opt *op, const char *val)
{
    char *dst = (char *)o + op->off;
    if (op->t == T_INT) *(int *)dst = atoi(val);
    else if (op->t == T_REAL) *(float *)dst = (float)atof(val);
    else snprintf(dst, 512, "%s", val);
    return 0;
}

static awp_status parse_gpu_cli(int argc, char **argv, awp_in3d *o)
{
    gpu_defaults(o);
    const size_t nopt = sizeof gpu_opts / sizeof gpu_opts[0];
    for (int a = 1; a < argc; a++) {
        const char *s = argv[a];
        const opt *hit = NULL;
        const char *val = NULL;
        if (s[0] == '-' && s[1] == '-') {
            const char *name = s + 2;
            const char *eq = strchr(name, '=');
            size_t len = eq ? (size_t)(eq - name) : strlen(name);
            for (size_t k = 0; k < nopt; k++)
                if (strlen(gpu_opts[k].lng) == len && strncmp(gpu_opts[k].lng, name, len) == 0) { hit = &gpu_opts[k]; break; }
            if (eq) val = eq + 1;
        } else if (s[0] == '-' && s[1] && !s[2]) {
            for (size_t k = 0; k < nopt; k++)
                if (gpu_opts[k].shrt == s[1]) { hit = &gpu_opts[k]; break; }
        }
        if (!hit) return ioerr(AWP_ERR_PARAM, "unknown option %s", s);
        if (!val) {
            if (a + 1 >= argc) return ioerr(AWP_ERR_PARAM, "option %s needs a value", s);
            val = argv[++a];
        }
        set_opt(o, hit, val);
    }
    o->nt = (int)(o->tmax / o->dt) + 1;   /* AWP-GPU-SGT/src/pmcl3d.c:265 */
    o->gpu_cli = 1;
    o->npz = 1;
    return AWP_OK;
}

awp_status awp_parse_command_line(int argc, char **argv, awp_in3d *out)
{
    for (int a = 1; a < argc; a++)
        if (argv[a][0] == '-') return parse_gpu_cli(argc, argv, out);
    /* set_names.f: #1 IN3D, #2 source, #3 media, #4 CHKP, #5 CHKJ, #6.. SSX3D.. */
    const char *in3d = (argc >= 2) ? argv[1] : "IN3D";
    awp_status st = awp_read_in3d(in3d, out);
    if (st != AWP_OK) return st;
    if (argc >= 3) snprintf(out->insrc, sizeof out->insrc, "%s", argv[2]);
    if (argc >= 4) snprintf(out->invel, sizeof out->invel, "%s", argv[3]);
    if (argc >= 5) snprintf(out->chkp, sizeof out->chkp, "%s", argv[4]);
    if (argc >= 6) snprintf(out->chkj, sizeof out->chkj, "%s", argv[5]);
    if (argc >= 7) snprintf(out->sxgro, sizeof out->sxgro, "%s", argv[6]);
    if (argc >= 8) snprintf(out->sygro, sizeof out->sygro, "%s", argv[7]);
    if (argc >= 9) snprintf(out->szgro, sizeof out->szgro, "%s", argv[8]);
    if (argc >= 10) snprintf(out->sxgro2, sizeof out->sxgro2, "%s", argv[9]);
    if (argc >= 11) snprintf(out->sygro2, sizeof out->sygro2, "%s", argv[10]);
    if (argc >= 12) snprintf(out->szgro2, sizeof out->szgro2, "%s", argv[11]);
    return AWP_OK;
}

void awp_params_from_in3d(const awp_in3d *in, awp_params *p)
{
    awp_params_default(p);
    p->nx = in->nx; p->ny = in->ny; p->nz = in->nz;
    p->dh = in->dh; p->dt = in->dt; p->nt = in->nt;
    p->nd = in->nd; p->arbc = in->arbc;
    p->fl = in->fl; p->fh = in->fh; p->fp = in->fp;
    p->socalq = in->socalq; p->nve = in->nve;
    p->mediastart = in->mediarestart; p->nvar = in->nvar; p->idyna = in->idyna;
    p->kinematic = in->ifault == 5;
    p->nst = in->nst; p->ntiskp_sgt = in->ntiskp_sgt; p->write_step = in->write_step;
    p->ncomp = 1; p->igreen[0] = in->igreen;
    p->npc = in->npc; p->pht = in->pht;
}

/* ------------------------------------------------------------------ */
/* source and cordfile                                                 */
/* ------------------------------------------------------------------ */

/* next number of a list-directed text stream (blanks and commas separate) */
static int next_number(FILE *f, double *v)
{
    char buf[128];
    int c, n = 0;
    do { c = fgetc(f); } while (c != EOF && (isspace(c) || c == ','));
    if (c == EOF) return 0;
    while (c != EOF && !isspace(c) && c != ',' && n + 1 < (int)sizeof buf) { buf[n++] = (char)c; c = fgetc(f); }
    buf[n] = 0;
    int ok;
    *v = fortran_real(buf, &ok);
    return ok;
}

awp_status awp_read_source(const char *path, int ifault, int nsrc, int nst, int *xyz, float *stf)
{
    if (ifault != 0 && ifault != 1 && ifault != 5)
        return ioerr(AWP_ERR_PARAM, "IFAULT %s: only 0 (text), 1 and 5 (binary) sources are read", "");
    if (ifault == 5) ifault = 1;   /* the subfault table has the binary IFAULT=1 layout (source.c:42-71) */
    FILE *f = fopen(path, ifault == 1 ? "rb" : "r");
    if (!f) return ioerr(AWP_ERR_IO, "cannot open source file %s", path);
    for (int s = 0; s < nsrc; s++) {
        float *t = stf + (size_t)s * nst * 6;
        if (ifault == 1) {
            if (fread(&xyz[3 * s], sizeof(int), 3, f) != 3 || fread(t, sizeof(float), (size_t)nst * 6, f) != (size_t)nst * 6) {
                fclose(f);
                return ioerr(AWP_ERR_IO, "source file %s is short", path);
            }
        } else {
            double v;
            for (int q = 0; q < 3; q++) {
                if (!next_number(f, &v)) { fclose(f); return ioerr(AWP_ERR_IO, "source file %s: bad position line", path); }
                xyz[3 * s + q] = (int)v;
            }
            for (size_t q = 0; q < (size_t)nst * 6; q++) {
                if (!next_number(f, &v)) { fclose(f); return ioerr(AWP_ERR_IO, "source file %s is short", path); }
                t[q] = (float)v;
            }
        }
    }
    fclose(f);
    return AWP_OK;
}

awp_status awp_read_cordfile(const char *path, int *npts, int **xyz)
{
    *npts = 0; *xyz = NULL;
    FILE *f = fopen(path, "r");
    if (!f) return ioerr(AWP_ERR_IO, "cannot open cordfile %s", path);
    char line[4096];
    long n = -1;
    while (fgets(line, sizeof line, f)) {
        char *p = line;
        while (*p && isspace((unsigned char)*p)) p++;
        if (*p == '#' || !*p) continue;
        n = strtol(p, NULL, 10);
        break;
    }
    if (n < 0) { fclose(f); return ioerr(AWP_ERR_IO, "cordfile %s has no point count", path); }
    int *a = (int *)malloc(sizeof(int) * 3 * (size_t)(n > 0 ? n : 1));
    for (long i = 0; i < n; i++) {
        if (fscanf(f, " %d %d %d", &a[3 * i], &a[3 * i + 1], &a[3 * i + 2]) != 3) {
            free(a); fclose(f);
            return ioerr(AWP_ERR_IO, "cordfile %s is short", path);
        }
    }
    fclose(f);
    *npts = (int)n;
    *xyz = a;
    return AWP_OK;
}
