/*
 * gpusgt_step_driver.cpp -- runs the reference CUDA stepper's own velocity and
 * stress kernels (dvelcx, dstrqc of AWP-GPU-SGT/src/kernel_kp1_fix_havg_ifault5.cu,
 * with its SetDeviceConstValue set-up) on the host CPU, to pin the oracle's
 * time-loop arithmetic to code the reference ships.
 *
 * TEST INFRASTRUCTURE ONLY.  tests/ and the fixture generator under
 * tests/golden/ load the library built from this file; the product never
 * does.  oracle/Makefile.ref extracts the two __global__ functions, the
 * __constant__ declarations and SetDeviceConstValue from the reference file
 * where it lies (nothing of it is copied into this repository) into
 * oracle/_ref/, and compiles them with this driver, which supplies host
 * stand-ins for the CUDA built-ins they use:
 *   - blockIdx / threadIdx are host variables that the driver's loops set, one
 *     emulated thread per interior (j, k) column, so the launch covers exactly
 *     the interior (the reference launches ceil(nzt / BLOCK_SIZE_Z) blocks of
 *     BLOCK_SIZE_Z threads with no bounds check, which assumes nzt is a
 *     multiple of BLOCK_SIZE_Z);
 *   - __constant__ values are host variables, cudaMemcpyToSymbol an assignment;
 *   - the texture reads tex1Dfetch(p_vx1 / p_vx2, pos) are array reads.
 * The threads of one kernel run one after the other; dvelcx and the interior
 * part of dstrqc do not depend on that order (each thread writes only its
 * own column, except dstrqc's free-surface branch, whose cells the tests
 * leave out of the comparison).
 *
 * Layout of the reference stepper (AWP-GPU-SGT/src/pmcl3d.c:384-411,
 * kernel_kp1_fix_havg_ifault5.cu:23-53): z fastest with `align` padding cells
 * below and above, then y, then x, with 2 + 4*loop ghost columns in x and y;
 * Fortran cell (i, j, k) of one rank is at x = i + 1 + 4*loop,
 * y = j + 1 + 4*loop, z = align + k - 1 (k = nz the free surface).
 *
 * Built with -ffp-contract=off: the host evaluates each expression with the
 * roundings C++ gives it (float arithmetic, and double where the reference
 * writes double literals such as 8.0/(...)); the device binary of the
 * reference may contract multiply-adds, so comparisons are within a stated
 * tolerance, not bit for bit.
 */
#include <stdlib.h>
#include <string.h>

#include "pmcl3d_cons.h"   /* BLOCK_SIZE_Y, BLOCK_SIZE_Z, align, loop (the reference's header) */

struct HostIdx {
    unsigned x, y, z;
};
static HostIdx blockIdx, threadIdx;

#define __global__ static
#define __constant__ static
#define register
#define tex1Dfetch(tex, i) ((tex)[i])
#define cudaMemcpyToSymbol(sym, src, n) memcpy(&(sym), (src), (n))

static const float *p_vx1, *p_vx2;

#include "gpusgt_const.inc"   /* __constant__ declarations                    */
#include "gpusgt_setconst.inc" /* SetDeviceConstValue                          */
#include "gpusgt_dvelcx.inc"   /* dvelcx                                       */
#include "gpusgt_dstrqc.inc"   /* dstrqc                                       */

namespace {

/* field numbering of the oracle: u1 v1 w1 xx yy zz xy xz yz r1..r6 lam mu d1 qp qs */
enum { U1, V1, W1, XX, YY, ZZ, XY, XZ, YZ, R1, R2, R3, R4, R5, R6, LAM, MU, D1, QP, QS, NF };

struct Ref {
    int nx, ny, nz;
    int sx, sy, sz;   /* extents: x (slowest), y, z (fastest) */
    float *f[NF];
    float *vx1, *vx2, *cx, *cy, *cz;
    long at(int i, int j, int k) const
    {
        return ((long)(i + 1 + 4 * loop) * sy + (j + 1 + 4 * loop)) * sz + (align + k - 1);
    }
};

}  // namespace

extern "C" {

void *gsr_create(int nx, int ny, int nz, float dh, float dt)
{
    Ref *r = (Ref *)calloc(1, sizeof(Ref));
    if (!r) return NULL;
    r->nx = nx; r->ny = ny; r->nz = nz;
    r->sx = nx + 4 + 8 * loop;
    r->sy = ny + 4 + 8 * loop;
    r->sz = nz + 2 * align;
    const size_t n = (size_t)r->sx * r->sy * r->sz;
    for (int a = 0; a < NF; a++) r->f[a] = (float *)calloc(n, sizeof(float));
    r->vx1 = (float *)calloc(n, sizeof(float));
    r->vx2 = (float *)calloc(n, sizeof(float));
    r->cx = (float *)calloc(r->sx, sizeof(float));
    r->cy = (float *)calloc(r->sy, sizeof(float));
    r->cz = (float *)calloc(r->sz, sizeof(float));
    for (int i = 0; i < r->sx; i++) r->cx[i] = 1.f;
    for (int j = 0; j < r->sy; j++) r->cy[j] = 1.f;
    for (int k = 0; k < r->sz; k++) r->cz[k] = 1.f;
    SetDeviceConstValue(dh, dt, nx, ny, nz);
    return r;
}

void gsr_destroy(void *h)
{
    Ref *r = (Ref *)h;
    if (!r) return;
    for (int a = 0; a < NF; a++) free(r->f[a]);
    free(r->vx1); free(r->vx2); free(r->cx); free(r->cy); free(r->cz);
    free(r);
}

/* one field from / to the padded host layout in[(k+1)][(j+1)][(i+1)],
 * extents (nz+4, ny+4, nx+4) */
int gsr_set(void *h, int fid, const float *in)
{
    Ref *r = (Ref *)h;
    if (fid < 0 || fid >= NF) return -1;
    const int wx = r->nx + 4, wy = r->ny + 4;
    for (int k = -1; k <= r->nz + 2; k++)
        for (int j = -1; j <= r->ny + 2; j++)
            for (int i = -1; i <= r->nx + 2; i++)
                r->f[fid][r->at(i, j, k)] = in[((size_t)(k + 1) * wy + (j + 1)) * wx + (i + 1)];
    return 0;
}

int gsr_get(void *h, int fid, float *out)
{
    const Ref *r = (const Ref *)h;
    if (fid < 0 || fid >= NF) return -1;
    const int wx = r->nx + 4, wy = r->ny + 4;
    for (int k = -1; k <= r->nz + 2; k++)
        for (int j = -1; j <= r->ny + 2; j++)
            for (int i = -1; i <= r->nx + 2; i++)
                out[((size_t)(k + 1) * wy + (j + 1)) * wx + (i + 1)] = r->f[fid][r->at(i, j, k)];
    return 0;
}

/* relaxation coefficients per cell: t1 / t2 [itz][ity][itx] with the parity
 * itx = i mod 2, ity = j mod 2, itz = (nz + 1 - k) mod 2 (viscoop.f:93-101) */
void gsr_set_tau(void *h, const float *t1, const float *t2)
{
    Ref *r = (Ref *)h;
    for (int k = 1; k <= r->nz; k++)
        for (int j = 1; j <= r->ny; j++)
            for (int i = 1; i <= r->nx; i++) {
                const int it = ((((r->nz + 1 - k) & 1) * 2 + (j & 1)) * 2) + (i & 1);
                r->vx1[r->at(i, j, k)] = t1[it];
                r->vx2[r->at(i, j, k)] = t2[it];
            }
}

/* Cerjan factors of cells 1..n of each axis */
void gsr_set_sponge(void *h, const float *cx, const float *cy, const float *cz)
{
    Ref *r = (Ref *)h;
    for (int i = 1; i <= r->nx; i++) r->cx[i + 1 + 4 * loop] = cx[i - 1];
    for (int j = 1; j <= r->ny; j++) r->cy[j + 1 + 4 * loop] = cy[j - 1];
    for (int k = 1; k <= r->nz; k++) r->cz[align + k - 1] = cz[k - 1];
}

/* nsteps of the reference's loop order for one rank without neighbours
 * (pmcl3d.c:864-876): dvelcx over x = xvs..xve, then dstrqc over
 * x = xls..xre, y from yls, every interior column */
void gsr_run(void *h, int nsteps)
{
    Ref *r = (Ref *)h;
    float **f = r->f;
    const int s_i = 2 + 4 * loop, e_i = r->nx + 4 * loop + 1, s_j = 2 + 4 * loop;
    p_vx1 = r->vx1;
    p_vx2 = r->vx2;
    for (int n = 0; n < nsteps; n++) {
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                blockIdx.x = k / BLOCK_SIZE_Z; threadIdx.x = k % BLOCK_SIZE_Z;
                blockIdx.y = j / BLOCK_SIZE_Y; threadIdx.y = j % BLOCK_SIZE_Y;
                dvelcx(f[U1], f[V1], f[W1], f[XX], f[YY], f[ZZ], f[XY], f[XZ], f[YZ], r->cx, r->cy, r->cz, f[D1],
                       s_i, e_i);
            }
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                blockIdx.x = k / BLOCK_SIZE_Z; threadIdx.x = k % BLOCK_SIZE_Z;
                blockIdx.y = j / BLOCK_SIZE_Y; threadIdx.y = j % BLOCK_SIZE_Y;
                dstrqc(f[XX], f[YY], f[ZZ], f[XY], f[XZ], f[YZ], f[R1], f[R2], f[R3], f[R4], f[R5], f[R6], f[U1],
                       f[V1], f[W1], f[LAM], f[MU], f[QP], f[QS], r->cx, r->cy, r->cz, NULL, r->nx, 0, 0, s_i, e_i,
                       s_j);
            }
    }
}

}  /* extern "C" */
