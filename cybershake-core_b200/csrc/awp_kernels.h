/* awp_kernels.h -- launchers of the stepper kernels (host side, C++). */
#ifndef AWP_KERNELS_H
#define AWP_KERNELS_H

#include <cuda_runtime.h>
#include "awp_internal.h"

struct AwpStepArgs {
    AwpGeom g;
    AwpMedia md;
    int ncomp;
    AwpComp comp[3];
    const float *cx, *cy, *cz;   /* sponge factors, index 1..n            */
    const float *tau;            /* [16] tau1[8] then tau2[8]              */
    float dth, dt, dh1;
    int kchunk;                  /* z levels per thread block              */
    int nve;
};

cudaError_t awp_launch_media_interior(const AwpGeom &g, const AwpMedia &md, const float *raw, int zf0, int nzs,
                                      int nvar, int var_offset, int socalq, int nve, float pi, float lw,
                                      float tmp1, float tmp2, int *ext, cudaStream_t st);
cudaError_t awp_launch_media_ghosts(const AwpGeom &g, const AwpMedia &md, int nve, cudaStream_t st);
cudaError_t awp_launch_media_homo(const AwpGeom &g, const AwpMedia &md, float lam, float mu, float d1,
                                  cudaStream_t st);
cudaError_t awp_launch_sg_coeffs(const AwpGeom &g, const AwpMedia &md, int npts, const int *pt_idx, float *sg,
                                 cudaStream_t st);
/* velocity sweep, free-surface velocity, stress sweep (+ fused fstr) */
cudaError_t awp_launch_step(const AwpStepArgs &s, cudaStream_t st);
cudaError_t awp_launch_post(const AwpPostArgs &a, int initial, cudaStream_t st);
cudaError_t awp_launch_sgt(const AwpSgtArgs &a, cudaStream_t st);

#endif
