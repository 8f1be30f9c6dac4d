/*
 * gpusgt_ref_driver.c -- TEST INFRASTRUCTURE: runs the host set-up functions
 * of the reference's CUDA stepper (AWP-GPU-SGT/src/mesh.c inimesh and tausub,
 * cerjan.c inicrj, grid.c allocators) on one rank, to pin the oracle's media
 * transform, relaxation times and sponge factors (awp_oracle.c, which follows
 * the Fortran of AWP-ODC-SGT) and to make golden fixtures.
 *
 * Built only where the reference sources are present (oracle/Makefile.ref).
 * The arrays are allocated and initialised as pmcl3d.c:561-612 does; the
 * results come back in the media file's order ([z][y][x], z = 0 at the
 * surface) and, for the sponge, indexed from the low face (z from the bottom).
 */
#include <string.h>

#include "pmcl3d.h"

Grid3D Alloc3D(int nx, int ny, int nz);
Grid1D Alloc1D(int nx);
void Delloc3D(Grid3D U);
void Delloc1D(Grid1D U);

/* MEDIASTART = 1 from `invel` (a path under 40 characters, as mesh.c's
 * filename buffer takes); ext6 = vs min/max, vp min/max, rho min/max;
 * taumm = taumin, taumax.  Returns 0. */
int ref_inimesh(int nx, int ny, int nz, int nvar, int nve, int socalq, float fp, float fl, float fh,
                const char *invel, float *lam, float *mu, float *d1, float *qp, float *qs, float *ext6, float *taumm)
{
    const int X = nx + 4 + 8 * loop, Y = ny + 4 + 8 * loop, Z = nz + 2 * align;
    Grid3D D1 = Alloc3D(X, Y, Z), MU = Alloc3D(X, Y, Z), LAM = Alloc3D(X, Y, Z);
    Grid3D QP = Alloc3D(X, Y, Z), QS = Alloc3D(X, Y, Z);
    float taumax = 0.f, taumin = 0.f, vse[2], vpe[2], dde[2];
    int coords[2] = {0, 0};
    char path[256];
    strncpy(path, invel, sizeof path - 1);
    path[sizeof path - 1] = 0;
    inimesh(1, D1, MU, LAM, QP, QS, &taumax, &taumin, nvar, fp, fl, fh, nx, ny, nz, 1, 1, nx, ny, nz, coords,
            MPI_COMM_WORLD, 0, nve, socalq, path, vse, vpe, dde);
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const size_t o = ((size_t)k * ny + j) * nx + i;
                const int a = i + 2 + 4 * loop, b = j + 2 + 4 * loop, c = (nz + align - 1) - k;
                lam[o] = LAM[a][b][c];
                mu[o] = MU[a][b][c];
                d1[o] = D1[a][b][c];
                qp[o] = QP[a][b][c];
                qs[o] = QS[a][b][c];
            }
    ext6[0] = vse[0], ext6[1] = vse[1], ext6[2] = vpe[0], ext6[3] = vpe[1], ext6[4] = dde[0], ext6[5] = dde[1];
    taumm[0] = taumin, taumm[1] = taumax;
    Delloc3D(D1), Delloc3D(MU), Delloc3D(LAM), Delloc3D(QP), Delloc3D(QS);
    return 0;
}

/* tau8[idx][idy][idz] */
int ref_tausub(float taumin, float taumax, float *tau8)
{
    Grid3D t = Alloc3D(2, 2, 2);
    tausub(t, taumin, taumax);
    for (int x = 0; x < 2; x++)
        for (int y = 0; y < 2; y++)
            for (int z = 0; z < 2; z++) tau8[(x * 2 + y) * 2 + z] = t[x][y][z];
    Delloc3D(t);
    return 0;
}

/* cx[nx], cy[ny] from the low face; cz[nz] from the bottom */
int ref_inicrj(float arbc, int nx, int ny, int nz, int nd, float *cx, float *cy, float *cz)
{
    Grid1D x = Alloc1D(nx + 4 + 8 * loop), y = Alloc1D(ny + 4 + 8 * loop), z = Alloc1D(nz + 2 * align);
    for (int i = 0; i < nx + 4 + 8 * loop; i++) x[i] = 1.0f;
    for (int j = 0; j < ny + 4 + 8 * loop; j++) y[j] = 1.0f;
    for (int k = 0; k < nz + 2 * align; k++) z[k] = 1.0f;
    int coords[2] = {0, 0};
    inicrj(arbc, coords, nx, ny, nz, nx, ny, nd, x, y, z);
    for (int i = 0; i < nx; i++) cx[i] = x[i + 2 + 4 * loop];
    for (int j = 0; j < ny; j++) cy[j] = y[j + 2 + 4 * loop];
    for (int k = 0; k < nz; k++) cz[k] = z[k + align];
    Delloc1D(x), Delloc1D(y), Delloc1D(z);
    return 0;
}
