/*
 * awp_internal.h -- device data layout shared by the kernels and the solver.
 *
 * HBM layout of one field (one float32 array per field per component):
 *   x fastest, then y, then z;  element (i,j,k) of the Fortran index space
 *   (i = -1..nx+2, j = -1..ny+2, k = -1..nz+2, k = nz the free surface) lives
 *   at  (k+1)*plane + (j+1)*px + (i + XO - 1)  with XO = 8, so that x = 1
 *   starts on a 32-byte sector and every row of px floats is 32-byte aligned.
 *   px = round_up(nx + XO + 2, 8), plane = px * (ny + 4).
 * Ghost cells hold zeros for wavefields (the boundary values of a single
 * domain), the padded values of padmedia/afsmedia for media.
 */
#ifndef AWP_INTERNAL_H
#define AWP_INTERNAL_H

#include <stdint.h>

#define AWP_XO 8
#define AWP_NF_STATE 15   /* u v w xx yy zz xy xz yz r1..r6 */
#define AWP_NF_ARRAYS 16  /* the state plus the exponent words of 16-bit block floating point r1..r6 */

enum {
    AF_U = 0, AF_V, AF_W, AF_XX, AF_YY, AF_ZZ, AF_XY, AF_XZ, AF_YZ,
    AF_R1, AF_R2, AF_R3, AF_R4, AF_R5, AF_R6,
    AF_RX   /* AWP_STORE_BFP only: per cell, the exponents of (r1 r2 r3) and (r4 r5 r6) */
};
enum { AM_LAM = 0, AM_MU, AM_D1, AM_QP, AM_QS, AM_N };

struct AwpGeom {
    int nx, ny, nz;
    int px;      /* row pitch (floats)            */
    int py;      /* rows per plane (ny + 4)       */
    int plane;   /* px * py                       */
    int64_t vol; /* plane * (nz + 4)              */
#ifdef __CUDACC__
    __host__ __device__ __forceinline__
#endif
    int idx(int i, int j, int k) const { return (k + 1) * plane + (j + 1) * px + (i + AWP_XO - 1); }
};

struct AwpComp {
    float *f[AWP_NF_ARRAYS];
};

template <int NC>
struct AwpCompSet {
    AwpComp c[NC];
};

struct AwpMedia {
    float *m[AM_N];
};

/* storage type of the media arrays and of r1..r6.  AWP_STORE_BFP (r1..r6
 * only): 16-bit block floating point -- each memory variable an int16
 * mantissa, the three normal (r1 r2 r3) and the three shear (r4 r5 r6)
 * memory variables of a cell sharing one exponent each, both exponents in
 * one uint16 word per cell (AF_RX: low byte r1..r3, high byte r4..r6). */
enum { AWP_STORE_F32 = 0, AWP_STORE_BF16 = 1, AWP_STORE_F16 = 2, AWP_STORE_BFP = 3 };

/* bytes of the six memory variables of one cell in a storage type */
static inline int awp_r_bytes(int rstore) { return rstore == AWP_STORE_F32 ? 24 : (rstore == AWP_STORE_BFP ? 14 : 12); }

/* Block floating point of three values sharing an exponent, the host and
 * device rule: e = the float exponent field of the largest magnitude; with
 * e >= 15 each value v is stored as the integer nearest (ties to even) to
 * v * 2^(141 - e) clamped to [-32767, 32767] (|v| * 2^(141 - e) < 2^15), and
 * read back as m * 2^(max(e, 15) - 141); e < 15 stores zero mantissas and a
 * zero exponent.  Both scalings are powers of two (exact), and decoding then
 * encoding again returns the same mantissas and exponent. */
#define AWP_BFP_EMIN 15u

/* binary16 arrays hold value * scale (a power of two); inv = 1/scale */
struct AwpMediaScale {
    float scale[AM_N];
    float inv[AM_N];
};

/* media as the steppers read them: typed arrays plus their scales */
struct AwpMediaT {
    void *m[AM_N];
    int type;
    AwpMediaScale sc;
};

/* relaxation coefficients tau1/tau2 indexed [itz][ity][itx] flattened */
struct AwpTau {
    float t1[8];
    float t2[8];
};

/* per-component source description on the device */
struct AwpSrcDev {
    int igreen;
    int nsrc;
    const int *ijk;     /* [nsrc][3] Fortran (i,j,k), k = nz at the surface */
    const float *stf;   /* [nsrc][nst][6]                                    */
};

struct AwpPostArgs {
    AwpGeom g;
    int ncomp;
    int nst;
    int nt;
    float vtst, vtst1;
    int probe;          /* (nd+2) when inside the grid, else 0 */
    int *step;          /* device counter: completed steps      */
    float *chkj[3];     /* [nt][3] per component                */
    AwpSrcDev src[3];
    AwpComp comp[3];
    const void *d1;     /* typed density array                  */
    int media_type;     /* AWP_STORE_*                          */
    float d1_inv;       /* binary16 scale inverse               */
    int kinematic;      /* IFAULT=5 subfault sources            */
    float dt;
    const void *mu;     /* typed compliance 1/mu (kinematic)     */
    float mu_inv;
    float *kin[3];      /* [nsrc][6] per-step stress increments  */
};

struct AwpSgtArgs {
    AwpGeom g;
    int ncomp;
    int npts;
    int ntiskp;
    int nsamp_written;  /* samples that land in complete chunks  */
    int64_t nt_file;
    const int *pt_idx;  /* [npts] linear grid index              */
    const float *sg;    /* [npts][3] sg1 sg2 sg3                 */
    const int *step;
    float *file[3];     /* raw SGT file image per component      */
    AwpComp comp[3];
    int active[3];      /* 0 for moment sources (IGREEN = -1)    */
};

#endif
