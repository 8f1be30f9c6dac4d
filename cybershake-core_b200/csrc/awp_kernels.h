/* awp_kernels.h -- launchers of the stepper kernels (host side, C++). */
#ifndef AWP_KERNELS_H
#define AWP_KERNELS_H

#include <cuda_runtime.h>
#include "awp_internal.h"

/* tensor maps of the TMA-staged stepper (awp_staged.cu) */
struct AwpStaged;

/* error word bits the steppers set */
#define AWP_KERR_TMA_WAIT 1          /* a staged-tile barrier wait ran out */

/* the PML zones of the step (NPC = 1; awp_pml.cu) */
struct AwpPmlArgs {
    AwpGeom g;
    int ncomp, nd;
    float dt, dth, pht;
    const float *rf, *rh;         /* damping profiles, index 1..nd            */
    float *split[3];              /* split arrays of each component           */
    long long n[5], off[5];       /* cells of each plane S N W E B, offsets   */
    AwpComp comp[3];              /* wavefields (the two-sweep buffer)        */
    const float *d1, *lam, *mu;   /* FP32 media                               */
    /* the 17 zone boxes (zone, first cell and extent per axis) with their
     * first block and block count, then the 8 lateral boxes' columns for
     * the free-surface image (awp_pml_boxes) */
    struct Box { int zone, i0, ni, j0, nj, k0, nk, b0, nb; } box[17], col[8];
    int nblk, ncolblk;
};
/* fills a.box / a.col and the block counts from a.g and a.nd */
void awp_pml_boxes(AwpPmlArgs &a);
cudaError_t awp_launch_pml(const AwpPmlArgs &a, int part, cudaStream_t st);
void awp_pml_profiles(int nd, float arbc, float dh, float vs_min, float vs_max, float *rf, float *rh);

struct AwpStepArgs {
    AwpGeom g;
    AwpMediaT md;                /* typed media                             */
    int ncomp;
    AwpComp comp[3];             /* wavefields read (two-sweep: updated)    */
    AwpComp comp_new[3];         /* fused: wavefields written (ping-pong)   */
    const float *cx, *cy, *cz;   /* sponge factors, index 1..n              */
    const float *tau;            /* [16] tau1[8] then tau2[8]               */
    float dth, dt, dh1;
    int kchunk;                  /* z levels per fused work item            */
    int kchunk_sweep;            /* z levels per two-sweep work item        */
    int nve;
    int fused;                   /* 1: single-sweep stepper                 */
    int rtype;                   /* AWP_STORE_* of r1..r6                   */
    int ty;                      /* thread-block rows (4, 8 or 16)          */
    int unroll;                  /* two-sweep z-loop unroll (1 or 2)        */
    const AwpStaged *staged;     /* non-NULL: TMA-staged velocity/stress    */
    int kchunk_staged;           /* z levels per staged work item           */
    int staged_qslow;            /* staged items: one component at a time   */
    int staged_rpt;              /* staged stress sweep: tile rows per thread */
    int staged_rpt_vel;          /* staged velocity sweep: tile rows per thread */
    int staged_batch;            /* staged sweeps with the components side by side in one item:
                                    bit 0 stress, bit 1 velocity */
    int *kerr;                   /* device error word (AWP_KERR_*)          */
    int sm_limit;                /* persistent grids sized for this many SMs (0 = all) */
    int fma;                     /* staged sweeps compiled with multiply-add contraction */
    int staged_generic;          /* one-component staged sweeps read their rings with generic loads */
    const AwpPmlArgs *pml;       /* NPC = 1: the PML zones after each sweep (NULL: Cerjan) */
    unsigned long long wait_ns;  /* bound of one barrier wait of the staged sweeps */
    int withhold;                /* test injection, -1 = off: block 0's producer of the
                                    staged stress sweep issues no copies for ring use
                                    `withhold`, so its consumers' wait runs out */
};

cudaError_t awp_launch_media_interior(const AwpGeom &g, const AwpMedia &md, const float *raw, int zf0, int nzs,
                                      int nvar, int var_offset, int socalq, int nve, float pi, float lw,
                                      float tmp1, float tmp2, int *ext, cudaStream_t st);
cudaError_t awp_launch_media_ghosts(const AwpGeom &g, const AwpMedia &md, int nve, cudaStream_t st);
cudaError_t awp_launch_media_homo(const AwpGeom &g, const AwpMedia &md, float lam, float mu, float d1,
                                  cudaStream_t st);
cudaError_t awp_launch_media_range(const AwpGeom &g, const AwpMedia &md, unsigned *mx, unsigned *mn, cudaStream_t st);
cudaError_t awp_launch_media_convert(const AwpMedia &src, const AwpMediaT &dst, int64_t n, cudaStream_t st);
cudaError_t awp_launch_sg_coeffs(const AwpMediaT &md, int npts, const int *pt_idx, float *sg, cudaStream_t st);

/* the kernels of one step */
enum { AWP_PART_VEL = 0, AWP_PART_FSVEL = 1, AWP_PART_STR = 2, AWP_PART_FUSED = 3,
       AWP_PART_PML_VEL = 4, AWP_PART_PML_STR = 5 };   /* PML parts: awp_launch_pml */
cudaError_t awp_launch_part(const AwpStepArgs &s, int part, cudaStream_t st);
/* two-sweep: velocity, free-surface velocity, stress (+ fstr); fused: one kernel */
cudaError_t awp_launch_step(const AwpStepArgs &s, cudaStream_t st);
/* TMA-staged sweeps: FP32 media; maps built once over fixed device arrays */
cudaError_t awp_staged_create(AwpStaged **out, const AwpGeom &g, int ncomp, const AwpComp *comp, const AwpMediaT &md,
                              int rtype);
void awp_staged_destroy(AwpStaged *s);
cudaError_t awp_launch_vel_staged(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream);
cudaError_t awp_launch_str_staged(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream);
/* the same sweeps compiled with multiply-add contraction (AWP_KERNEL_STAGED_FMA) */
cudaError_t awp_launch_vel_staged_fma(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream);
cudaError_t awp_launch_str_staged_fma(const AwpStaged *st, const AwpStepArgs &s, cudaStream_t stream);
cudaError_t awp_launch_post(const AwpPostArgs &a, int initial, cudaStream_t st);
cudaError_t awp_launch_sgt(const AwpSgtArgs &a, cudaStream_t st);
/* one z-slab of RWG p/s/d volumes ([3][ny][n][nx]) to AWP media order
 * ([n][nx][ny][3], x 1000) */
cudaError_t awp_launch_rwg_slab(const float *rwg, float *awp, int nx, int ny, int n, cudaStream_t st);
/* SGT file images [point][6][nt] in RWG component order (z-force runs x -2) */
cudaError_t awp_launch_sgt_rwg(const float *in, float *out, int64_t npts, int nt, int zsrc, cudaStream_t st);

/* FP64 energy of (u, v, w) per component, two passes through `partial`
 * (nblocks * ncomp doubles of scratch); flag (may be NULL) set on NaN/Inf */
#define AWP_EN_BLOCK 256
#define AWP_EN_GRID 592
struct AwpEnergyArgs {
    AwpGeom g;
    int ncomp;
    const float *f[9];
};
cudaError_t awp_launch_energy(const AwpEnergyArgs &a, double *partial, int nblocks, double *out, int *flag,
                              cudaStream_t st);
/* n floats of bounded pseudo-random values in [-amp, amp) (autotuner trials) */
cudaError_t awp_launch_fill_noise(float *p, int64_t n, unsigned seed, float amp, cudaStream_t st);

#endif
