/*
 * awp_sgthead.c -- the RWG SGT header file (sgtmaster, sgtindex[np],
 * sgtheader[np]) that CyberShake's post-processing reads next to the SGT.
 *
 * Follows SgtHead/src/write_head.c:48-469 (field values, media sampling and
 * the great-circle projection of head_subs.c:3-126, 158-246 with geoproj 1),
 * keeping the reference's float / double evaluation points so that the file
 * is byte-identical.  The records are the structs of SgtHead/src/structure.h:
 * 164-220 (x86-64 layout: 36, 24 and 128 bytes).
 */
#define _FILE_OFFSET_BITS 64
#include <errno.h>
#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../../include/awp_sgt.h"

void awp_set_error_text(const char *msg);

static awp_status io_err(const char *fmt, const char *what)
{
    char b[1200];
    snprintf(b, sizeof b, fmt, what);
    awp_set_error_text(b);
    return AWP_ERR_IO;
}

#define DEG 0.01745329            /* radians per degree, as head_subs.c uses it */
#define EARTH_RADIUS 6378.139f    /* km */

/* geoproj 1: great-circle projection of the model box */
typedef struct {
    double a[9], ainv[9];
    double g0, b0;
    float erad;
} gc_proj;

/* rotation of the model frame: azimuth alpha of the y axis, origin (lon, lat) */
static void gc_matrices(gc_proj *p, float alpha, float lon, float lat)
{
    const double ca = cos((double)alpha * DEG), sa = sin((double)alpha * DEG);
    const double ct = cos((double)(90.0 - lat) * DEG), st = sin((double)(90.0 - lat) * DEG);
    const double cp = cos((double)lon * DEG), sp = sin((double)lon * DEG);
    double *m = p->a;
    m[0] = ca * ct * cp + sa * sp;
    m[1] = sa * ct * cp - ca * sp;
    m[2] = st * cp;
    m[3] = ca * ct * sp - sa * cp;
    m[4] = sa * ct * sp + ca * cp;
    m[5] = st * sp;
    m[6] = -ca * st;
    m[7] = -sa * st;
    m[8] = ct;
    double det = m[0] * (m[4] * m[8] - m[7] * m[5]) - m[1] * (m[3] * m[8] - m[6] * m[5]) +
                 m[2] * (m[3] * m[7] - m[6] * m[4]);
    det = 1.0 / det;
    /* transpose scaled by 1/det (the matrix is a rotation) */
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) p->ainv[3 * r + c] = det * m[3 * c + r];
}

/* model-frame (x, y) in km to longitude / latitude in degrees */
static void gc_xy_to_lonlat(const gc_proj *p, float x, float y, float *lon, float *lat)
{
    double arg = x / p->erad - p->b0;
    const double cb = cos(arg), sb = sin(arg);
    arg = y / p->erad - p->g0;
    const double cg = cos(arg), sg = sin(arg);
    arg = sqrt(1.0 + sb * sb * sg * sg);
    const double xp = sg * cb * arg, yp = sb * cg * arg;
    const double zp = sqrt(1.0 - xp * xp - yp * yp);
    const double *m = p->a;
    const double xg = xp * m[0] + yp * m[1] + zp * m[2];
    const double yg = xp * m[3] + yp * m[4] + zp * m[5];
    const double zg = xp * m[6] + yp * m[7] + zp * m[8];
    arg = sqrt(xg * xg + yg * yg) / zg;
    *lat = 90.0 - atan(arg) / DEG;
    *lon = xg != 0.0 ? atan(yg / xg) / DEG : 0.0;
    if (xg < 0.0) *lon = *lon - 180.0;
    while (*lon < -180.0) *lon = *lon + 360.0;
}

/* the 5th line of the model-box file: "mlon= <lon> mlat= <lat> mrot= <rot>" */
static awp_status read_modelbox(const char *path, float *lon, float *lat, float *rot)
{
    FILE *f = fopen(path, "r");
    if (!f) return io_err("cannot open model box file %s", path);
    char line[1024] = {0};
    for (int n = 0; n < 5; n++)
        if (!fgets(line, sizeof line, f)) {
            fclose(f);
            return io_err("model box file %s has fewer than 5 lines", path);
        }
    fclose(f);
    char *tok[6];
    int nt = 0;
    for (char *t = strtok(line, "= "); t && nt < 6; t = strtok(NULL, "= ")) tok[nt++] = t;
    if (nt < 6) return io_err("model box file %s: line 5 is not 'mlon= . mlat= . mrot= .'", path);
    *lon = (float)atof(tok[1]);
    *lat = (float)atof(tok[3]);
    *rot = (float)atof(tok[5]);
    return AWP_OK;
}

/* nx, ny, nz of a grid file: a line, "nx=N", N + 2 lines, "ny=N", N + 2 lines, "nz=N" */
static awp_status read_gridout(const char *path, int *nx, int *ny, int *nz)
{
    FILE *f = fopen(path, "r");
    if (!f) return io_err("cannot open grid file %s", path);
    char line[1024];
    int ok = fgets(line, sizeof line, f) != NULL && fscanf(f, "nx=%d", nx) == 1;
    for (int i = 0; ok && i < *nx + 2; i++) ok = fgets(line, sizeof line, f) != NULL;
    ok = ok && fscanf(f, "ny=%d", ny) == 1;
    for (int i = 0; ok && i < *ny + 2; i++) ok = fgets(line, sizeof line, f) != NULL;
    ok = ok && fscanf(f, "nz=%d", nz) == 1;
    fclose(f);
    if (!ok || *nx < 1 || *ny < 1 || *nz < 1) return io_err("grid file %s: cannot read nx / ny / nz", path);
    return AWP_OK;
}

static int read_at(int fd, void *dst, size_t bytes, off_t off)
{
    unsigned char *p = (unsigned char *)dst;
    while (bytes > 0) {
        ssize_t r = pread(fd, p, bytes, off);
        if (r <= 0) return -1;
        p += r;
        bytes -= (size_t)r;
        off += r;
    }
    return 0;
}


awp_status awp_write_sgt_header(const awp_sgthead_args *a, const char *outfile)
{
    if (!a || !outfile || !a->modelbox || !a->coordfile || !a->fdloc || !a->gridout || !a->media_file ||
        !a->component) {
        awp_set_error_text("awp_write_sgt_header: null argument");
        return AWP_ERR_PARAM;
    }
    if (a->sgt_tinc < 1) {
        awp_set_error_text("awp_write_sgt_header: time decimation must be >= 1");
        return AWP_ERR_PARAM;
    }
    float mlon = 0.0f, mlat = 0.0f, mrot = 0.0f;
    awp_status st = read_modelbox(a->modelbox, &mlon, &mlat, &mrot);
    if (st != AWP_OK) return st;
    int xsrc = 0, ysrc = 0;
    {
        FILE *f = fopen(a->fdloc, "r");
        if (!f) return io_err("cannot open source location file %s", a->fdloc);
        const int n = fscanf(f, "%d %d", &xsrc, &ysrc);
        fclose(f);
        if (n != 2) return io_err("source location file %s: expected 'x y'", a->fdloc);
    }
    int nx, ny, nz;
    st = read_gridout(a->gridout, &nx, &ny, &nz);
    if (st != AWP_OK) return st;

    /* model frame (geoproj 1: origin at the box centre) */
    const float h = a->spacing;
    const float xlen = nx * h, ylen = ny * h;
    gc_proj gp;
    gp.erad = EARTH_RADIUS;
    gc_matrices(&gp, mrot, mlon, mlat);
    gp.g0 = (double)(0.5 * ylen) / (double)gp.erad;
    gp.b0 = (double)(0.5 * xlen) / (double)gp.erad;

    awp_sgtmaster m;
    memset(&m, 0, sizeof m);
    m.geoproj = 1;
    m.modellon = mlon;
    m.modellat = mlat;
    m.modelrot = mrot;
    m.xshift = -0.5 * xlen;
    m.yshift = -0.5 * ylen;

    /* RWG cordfile: '#' comments, the point count, then "x y z indx lon lat dep" */
    FILE *cf = fopen(a->coordfile, "r");
    if (!cf) return io_err("cannot open SGT coordinate file %s", a->coordfile);
    char line[1024];
    do {
        if (!fgets(line, sizeof line, cf)) {
            fclose(cf);
            return io_err("SGT coordinate file %s: no point count", a->coordfile);
        }
    } while (line[0] == '#');
    if (sscanf(line, "%d", &m.globnp) != 1 || m.globnp < 0) {
        fclose(cf);
        return io_err("SGT coordinate file %s: bad point count", a->coordfile);
    }
    m.localnp = m.globnp;
    m.nt = a->nt / a->sgt_tinc;
    const int np = m.globnp;
    awp_sgtindex *ix = (awp_sgtindex *)calloc(np > 0 ? (size_t)np : 1, sizeof *ix);
    awp_sgtheader *hd = (awp_sgtheader *)calloc(np > 0 ? (size_t)np : 1, sizeof *hd);
    if (!ix || !hd) {
        fclose(cf);
        free(ix);
        free(hd);
        awp_set_error_text("awp_write_sgt_header: host allocation failed");
        return AWP_ERR_OOM;
    }
    for (int i = 0; i < np; i++) {
        float lon, lat;
        if (!fgets(line, sizeof line, cf) ||
            sscanf(line, "%d %d %d %lld %f %f %f", &ix[i].xsgt, &ix[i].ysgt, &ix[i].zsgt, &ix[i].indx, &lon, &lat,
                   &hd[i].sgt_dep) != 7 ||
            ix[i].xsgt < 0 || ix[i].xsgt >= nx || ix[i].ysgt < 0 || ix[i].ysgt >= ny || ix[i].zsgt < 0 ||
            ix[i].zsgt >= nz) {
            fclose(cf);
            free(ix);
            free(hd);
            char b[160];
            snprintf(b, sizeof b, "SGT coordinate file: bad or missing point record %d", i);
            awp_set_error_text(b);
            return AWP_ERR_IO;
        }
    }
    fclose(cf);

    /* media file: float [z][x][y][vp vs rho] in m/s and kg/m^3 (AWP order, y fastest) */
    const int fd = open(a->media_file, O_RDONLY);
    if (fd < 0) {
        free(ix);
        free(hd);
        return io_err("cannot open media file %s", a->media_file);
    }
    const size_t plane = (size_t)3 * nx * ny;
    float *vel = (float *)malloc(2 * plane * sizeof(float));
    if (!vel) {
        close(fd);
        free(ix);
        free(hd);
        awp_set_error_text("awp_write_sgt_header: host allocation failed");
        return AWP_ERR_OOM;
    }
    const float sf = 0.001f;      /* m/s -> km/s, kg/m^3 -> g/cm^3 */
    const float conv = 1.0e+10f;  /* -> dyne/cm^2 */
    const float fh = 25.0f, fp = 1.0f;
    int loaded = -1;
    st = AWP_OK;
    for (int i = 0; i < np && st == AWP_OK; i++) {
        awp_sgtheader *s = &hd[i];
        ix[i].h = h;
        s->indx = ix[i].indx;
        s->geoproj = m.geoproj;
        s->modellon = m.modellon;
        s->modellat = m.modellat;
        s->modelrot = m.modelrot;
        s->xshift = m.xshift;
        s->yshift = m.yshift;
        s->xazim = 90.0 + m.modelrot;
        s->nt = m.nt;
        s->dt = a->dt * a->sgt_tinc;
        s->h = h;
        s->xsrc = xsrc;
        s->ysrc = ysrc;
        s->zsrc = 1;
        s->xsgt = ix[i].xsgt;
        s->ysgt = ix[i].ysgt;
        s->zsgt = ix[i].zsgt;
        s->xmom = s->ymom = s->zmom = 0.0f;
        if (strcmp(a->component, "x") == 0) s->xmom = a->moment;
        else if (strcmp(a->component, "y") == 0) s->ymom = a->moment;
        else if (strcmp(a->component, "z") == 0) s->zmom = a->moment;
        s->tst = -3.0 / a->flo;
        float xx = s->xsrc * h, yy = s->ysrc * h;
        gc_xy_to_lonlat(&gp, xx, yy, &s->src_lon, &s->src_lat);
        s->src_dep = (s->zsrc - 1) * h;
        xx = s->xsgt * h;
        yy = s->ysgt * h;
        gc_xy_to_lonlat(&gp, xx, yy, &s->sgt_lon, &s->sgt_lat);
        const float dx = s->xsgt - s->xsrc, dy = s->ysgt - s->ysrc, dz = s->zsgt - s->zsrc;
        s->cdist = h * sqrt(dx * dx + dy * dy + dz * dz);

        /* material at the point: plane z-1 (plane 0 at the surface) and the plane after it */
        const int z0 = s->zsgt != 0 ? s->zsgt - 1 : 0;
        if (z0 != loaded) {
            const int nplanes = z0 + 1 < nz ? 2 : 1;
            if (read_at(fd, vel, nplanes * plane * sizeof(float), (off_t)z0 * plane * sizeof(float)) != 0) {
                st = io_err("media file %s is shorter than the grid", a->media_file);
                break;
            }
            loaded = z0;
        }
        const int yr = s->ysgt == 0 ? 1 : 0;     /* density from y = 1 at y = 0 */
        const size_t vp_i = (size_t)3 * ((size_t)s->xsgt * ny + s->ysgt), vs_i = vp_i + 1;
        const size_t rho_i = (size_t)3 * ((size_t)s->xsgt * ny + s->ysgt + yr) + 2;
        const size_t rho_x = (size_t)3 * ((size_t)(s->xsgt + 1) * ny + s->ysgt + yr) + 2;
        const size_t rho_y = (size_t)3 * ((size_t)s->xsgt * ny + s->ysgt + 1) + 2;
        const size_t rho_z = plane + rho_i;
        float mu;
        if (a->mu_corr) {
            const float qs = 0.05 * vel[vs_i];
            const float vs_corr = vel[vs_i] * sf * (1 + (log(fh / fp) / (qs * 3.14159)));
            mu = vel[rho_i] * sf * vs_corr * vs_corr;
        } else {
            mu = vel[vs_i] * sf * vel[vs_i] * sf * vel[rho_i] * sf;
        }
        const float lam = vel[vp_i] * sf * vel[vp_i] * sf * vel[rho_i] * sf - 2 * mu;
        s->mu = conv * mu;
        s->lam = conv * lam;
        const float r0 = vel[rho_i] * sf;
        if (s->xsgt == nx - 1 || s->zsgt == nz - 1) {
            s->rho = r0;
        } else {
            const float rx = vel[rho_x] * sf, ry = vel[rho_y] * sf, rz = vel[rho_z] * sf;
            const float bx = 2.0 / (r0 + rx), by = 2.0 / (r0 + ry), bz = 2.0 / (r0 + rz);
            s->rho = 3.0 / (bx + by + bz);
        }
    }
    free(vel);
    close(fd);
    if (st == AWP_OK) {
        FILE *out = fopen(outfile, "wb");
        if (!out) {
            st = io_err("cannot create header file %s", outfile);
        } else {
            const int ok = fwrite(&m, sizeof m, 1, out) == 1 &&
                           (np == 0 || fwrite(ix, sizeof *ix, (size_t)np, out) == (size_t)np) &&
                           (np == 0 || fwrite(hd, sizeof *hd, (size_t)np, out) == (size_t)np);
            if (fclose(out) != 0 || !ok) st = io_err("cannot write header file %s", outfile);
        }
    }
    free(ix);
    free(hd);
    return st;
}
