/*
 * awp_sgt.h -- C ABI of libawpsgt, the B200 strain-Green-tensor (SGT) stepper.
 *
 * The reference has no plugin API: its boundary is the `pmcl3d` process plus
 * its files, and inside the CUDA variant an `extern "C"` launcher layer over
 * raw device pointers.  This header is the library form of that boundary.  The
 * `pmcl3d` executable built beside the library is a thin C driver over it that
 * accepts both reference command lines and writes the same files.
 *
 * Every entry point below names the reference code it replaces (paths are
 * inside the reference project SCECcode/cybershake-core).
 *
 * Conventions shared with the reference:
 *   - grid indices are 1-based; x = 1..NX, y = 1..NY, z = 1..NZ with z = 1 at
 *     the free surface for every coordinate a caller passes in (source
 *     position, cordfile points), as in the IN3D/cordfile formats;
 *   - the media array is float32 [z][y][x][nvar], z = 0 at the surface
 *     (file layout read by AWP-ODC-SGT/src/structure.f:142-173);
 *   - a source time function is float32 [nst][6] with columns
 *     axx ayy azz axz ayz axy (AWP-ODC-SGT/src/source.f:193);
 *   - the raw SGT output is float32 [point][6][NT] with components
 *     XX YY ZZ XY XZ YZ (AWP axes), NT = int(int(nt/WRITE_STEP)*WRITE_STEP/
 *     NTISKP_SGT), points in cordfile order (AWP-ODC-SGT/src/pmcl3d.f:1589-1601).
 *
 * Ownership and threading: the library allocates and owns all device memory of
 * a solver.  Calls on one solver must not overlap; separate solvers may be used
 * from separate host threads.  No entry point calls exit(); failures return a
 * status and awp_last_error() describes the latest failure of the calling
 * thread.
 */
#ifndef AWP_SGT_H
#define AWP_SGT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    AWP_OK = 0,
    AWP_ERR_IO = 1,        /* file missing, short or malformed               */
    AWP_ERR_PARAM = 2,     /* parameter out of range                         */
    AWP_ERR_OOM = 3,       /* device or host allocation failed               */
    AWP_ERR_CUDA = 4,      /* CUDA runtime error                             */
    AWP_ERR_UNSTABLE = 5,  /* stability monitor saw NaN/Inf or runaway growth */
    AWP_ERR_TIMEOUT = 6,   /* a bounded wait ran out                         */
    AWP_ERR_STATE = 7,     /* call made in the wrong order                   */
    AWP_ERR_BUSY = 8,      /* serving queue full / not enough device memory  */
    AWP_ERR_CANCELLED = 9  /* serving request was cancelled                  */
} awp_status;

/* Storage precision of the material coefficients and of the anelastic memory
 * variables r1..r6.  Wavefields and all stencil arithmetic stay FP32. */
typedef enum {
    AWP_PREC_F32 = 0,   /* plain FP32, bit-exact with the FP32 oracle        */
    AWP_PREC_BF16 = 1,  /* media and r1..r6 stored as bfloat16               */
    AWP_PREC_F16 = 2,   /* media as binary16 scaled by a power of two per
                           array, r1..r6 as bfloat16 (binary16 lacks the
                           exponent range for memory variables, whose size
                           follows the source amplitude)                     */
    AWP_PREC_MIXED = 3, /* media FP32, r1..r6 bfloat16                       */
    AWP_PREC_BFP = 4    /* media FP32, r1..r6 in 16-bit block floating point:
                           an int16 mantissa each, the normal (r1..r3) and
                           the shear (r4..r6) memory variables of a cell
                           sharing one exponent each (one 16-bit word per
                           cell); 14 bytes per cell instead of 24           */
} awp_precision;

/* Stepper implementation. */
typedef enum {
    AWP_KERNEL_AUTO = 0,      /* library picks: the staged stepper for FP32
                                 media, else the two-sweep stepper           */
    AWP_KERNEL_TWO_SWEEP = 1, /* velocity sweep, then stress sweep, in place   */
    AWP_KERNEL_FUSED = 2,     /* one z-march per tile: velocity on a 2-cell
                                 halo, then stress; ping-pong wavefields       */
    AWP_KERNEL_STAGED = 3,    /* the two sweeps with TMA-staged xy tiles and a
                                 z register queue (FP32 media only)           */
    AWP_KERNEL_STAGED_FMA = 4 /* the staged sweeps compiled with multiply-add
                                 contraction: fewer instructions, results
                                 within FP32 rounding of the others instead
                                 of bit-identical                              */
} awp_kernel;

#define AWP_MAX_COMP 3

/* Parameters of one solve.  Field names follow IN3D (AWP-ODC-SGT/src/io.f:327-417)
 * and the GPU command line (AWP-GPU-SGT/src/command.c:185-230). */
typedef struct {
    int nx, ny, nz;          /* NX NY NZ                                     */
    float dh, dt;            /* DH DT                                        */
    int nt;                  /* time steps (pmcl3d.f:287: nint(TMAX/DT)+1)   */
    int nd;                  /* ND    Cerjan sponge width                    */
    float arbc;              /* ARBC  Cerjan coefficient                     */
    float fl, fh, fp;        /* FL FH FP  Q band                             */
    int socalq;              /* SOCALQ velocity dispersion correction        */
    int nve;                 /* NVE   1 = viscoelastic, 0 = elastic          */
    int mediastart;          /* MEDIARESTART 0 = homogeneous, else media     */
    int nvar;                /* NVAR  3, 5 or 8                              */
    int idyna;               /* IDYNA (homogeneous medium choice only)       */
    int nst;                 /* NST   source time-function length            */
    int ntiskp_sgt;          /* NTISKP_SGT                                   */
    int write_step;          /* WRITE_STEP (SGT samples per chunk)           */
    int ncomp;               /* components stepped together (1..3)           */
    int igreen[AWP_MAX_COMP];/* IGREEN per component (1,2,3,-1,-2,4,5,6)     */
    int precision;           /* awp_precision                                */
    int kernel;              /* awp_kernel                                   */
    int device;              /* CUDA device ordinal                          */
    int monitor_every;       /* stability check period in steps (0 = off)    */
    int kinematic;           /* 1: IFAULT=5 kinematic source -- each source
                                row pair is a subfault (stf type, slip,
                                rupture time, rise time, area | strike, dip,
                                rake; NST = 2) whose moment rate is inserted
                                into the stresses after every stress update
                                (AWP-GPU-SGT kernel_kp1_fix_havg_ifault5.cu:
                                289-376); IGREEN then only selects the SGT
                                output                                        */
    int npc;                 /* NPC   0 = Cerjan sponge, 1 = PML absorbing
                                boundary of width ND (AWP-ODC-SGT/src/pml.f;
                                the two-sweep and staged steppers, FP32 media) */
    float pht;               /* PHT   PML damping ratio of the tangential splits */
} awp_params;

typedef struct {
    int64_t steps_done;
    double seconds_loop;         /* device time of the time loop (events)    */
    double gcell_updates_per_s;  /* nx*ny*nz*ncomp*steps / seconds_loop      */
    double bytes_per_cell_update;/* algorithmic bytes of the chosen stepper  */
    double device_bytes;         /* device memory held by the solver         */
    float vp_min, vp_max, vs_min, vs_max, rho_min, rho_max;  /* for CHKP     */
    double energy;               /* last stability-monitor value (FP64)      */
} awp_stats;

typedef struct awp_solver awp_solver;

/* Fills defaults (those of AWP-GPU-SGT/src/command.c:60-115 where they apply). */
void awp_params_default(awp_params *p);

/* Allocates a solver and its device fields.
 * Replaces: vsemem (AWP-ODC-SGT/src/memory.f:137-200), inicrj
 * (AWP-ODC-SGT/src/cerjan.f:4-247), tausub (AWP-ODC-SGT/src/relax.f:4-39) and the
 * device set-up of AWP-GPU-SGT/src/pmcl3d.c:640-823 and
 * SetDeviceConstValue (AWP-GPU-SGT/src/kernel_kp1_fix_havg_ifault5.cu:23-53). */
awp_status awp_create(const awp_params *p, awp_solver **out);

/* Loads media (float32 [nz][ny][nx][nvar], z = 0 at the surface, host memory),
 * applies the Q / SoCalQ transform and pads the ghost cells on the device.
 * Replaces: inimesh + padmedia + afsmedia (AWP-ODC-SGT/src/structure.f:13-707),
 * AWP-GPU-SGT/src/mesh.c:12-410.  With mediastart == 0 `media` may be NULL
 * (inihomo, structure.f:709-765). */
awp_status awp_load_media(awp_solver *s, const float *media);

/* Same, reading the media file (structure.f:142-173 record layout). */
awp_status awp_load_media_file(awp_solver *s, const char *path);

/* Sets the sources of component `comp`: xyz [nsrc][3] (1-based, z = 1 at the
 * surface) and stf [nsrc][nst][6].
 * Replaces: rdsrcpos/getsrc (AWP-ODC-SGT/src/source.f:132-470) and the source
 * upload of AWP-GPU-SGT/src/source.c:4-159. */
awp_status awp_set_source(awp_solver *s, int comp, int nsrc, const int *xyz, const float *stf);

/* Sets the SGT output points: xyz [npts][3] cordfile coordinates (1-based,
 * z = 1 at the surface), kept in cordfile order.
 * Replaces: getrec SGT part (AWP-ODC-SGT/src/station.f:31-80), inisgt
 * (AWP-GPU-SGT/src/sgt.c:4-73). */
awp_status awp_set_points(awp_solver *s, int npts, const int *xyz);

/* Advances every component by up to `nsteps` time steps (stops at nt).  When
 * sgt_out is not NULL the raw SGT file images of all components are copied to
 * it, one after the other ([comp][awp_sgt_file_floats()]).
 * Replaces: the time loop AWP-ODC-SGT/src/pmcl3d.f:1183-1611 (dvelc, addcrjvel,
 * fvelxy, fvelz, dstrqc, addcrjstr, addsrc, fstr, SGT gather) and its CUDA
 * launchers dvelcx_H, dstrqc_H, addsrc_H, ComputeSGT
 * (AWP-GPU-SGT/src/kernel_kp1_fix_havg_ifault5.cu:72-178, 379-419). */
awp_status awp_run(awp_solver *s, int nsteps, float *sgt_out);

/* Number of float32 values in one component's raw SGT file image. */
int64_t awp_sgt_file_floats(const awp_solver *s);

/* Copies the raw SGT file image of one component (pmcl3d.f:1582-1604). */
awp_status awp_get_sgt(awp_solver *s, int comp, float *out);

/* Copies the CHKJ series of one component: [nt][3] u1,v1,w1 at (ND+2,ND+2,ND+2)
 * after every step (AWP-ODC-SGT/src/pmcl3d.f:1474-1484). */
awp_status awp_get_chkj(awp_solver *s, int comp, float *out);

/* Test/diagnostic access: copies one field of one component into the padded
 * host layout out[(k+1)][(j+1)][(i+1)], extents (nz+4, ny+4, nx+4), as float32.
 * field: 0..8 = u1 v1 w1 xx yy zz xy xz yz, 9..14 = r1..r6,
 * 15..19 = lam mu d1 qp qs (compliances as stored by structure.f:488-519). */
awp_status awp_get_field(awp_solver *s, int comp, int field, float *out);

/* Copies the interior of one horizontal level of a wavefield or stress
 * (field 0..8, numbering as awp_get_field) after the steps done so far:
 * out[(j-1)*nx + (i-1)] = field(i, j, k), i = 1..nx, j = 1..ny, k = 1..nz
 * (k = nz is the free surface).  Replaces the reference's per-NTISKP device
 * copies of u1, v1, w1 for the surface velocity files and the CHKP statistics
 * line (AWP-GPU-SGT/src/pmcl3d.c:962-1031), moving one level instead of the
 * whole volume. */
awp_status awp_get_plane(awp_solver *s, int comp, int field, int k, float *out);

/* Sets one state field (0..14, numbering as awp_get_field) of one component
 * from the padded host layout in[(k+1)][(j+1)][(i+1)], extents (nz+4, ny+4,
 * nx+4), float32; memory variables stored in 16 bits are rounded to nearest
 * (bf16), or, in block floating point, their group of three (r1..r3 or
 * r4..r6) is encoded again with the new member -- values below the group
 * exponent's range become zero, so restoring decoded values needs all three
 * members, as awp_checkpoint_read sets them.
 * Used by the checkpoint restart below and to start a solve from a given
 * state.  Replaces the state part of the checkpoint read
 * (AWP-ODC-SGT/src/pmcl3d.f:1044-1056). */
awp_status awp_set_field(awp_solver *s, int comp, int field, const float *in);

/* Checkpoint of the state after the steps done so far, in the reference's
 * files (AWP-ODC-SGT/src/pmcl3d.f:1967-2045; the component index stands for
 * the MPI rank):
 *   dir/ckp<rank:7><step:7>.bin    records [u1 v1 w1] [xx yy zz] [xy xz yz]
 *                                  [r1 r2 r3] [r4 r5 r6], each array
 *                                  (nx+4)(ny+4)(nz+4) float32 with ghosts;
 *   dir/ckpdy<rank:7><step:7>.bin  u2, broken (zero: no dynamic rupture), mu;
 *   dir/ckp<rank:7>.hdr            the step, written last;
 * plus dir/ckpsgt<rank:7><step:7>.bin (this library's addition: the SGT file
 * image and CHKJ series so far, which the reference writes out as it goes)
 * so that a resumed solve ends with the files of an uninterrupted one. */
awp_status awp_checkpoint_write(awp_solver *s, const char *dir);

/* Restores the newest checkpoint in `dir` (the smallest step over the
 * components' .hdr files, as pmcl3d.f:1019-1036 takes the minimum over
 * ranks); *step receives it, 0 when there is none (then nothing changes).
 * Media, sources and points must be set first, as for a new solve.  Without
 * the ckpsgt file only the wavefield is restored.  The next awp_run continues
 * with step *step + 1 (pmcl3d.f:1103). */
awp_status awp_checkpoint_read(awp_solver *s, const char *dir, int *step);

/* Statistics of the solver (timers, throughput, media extremes for CHKP). */
awp_status awp_get_stats(awp_solver *s, awp_stats *st);

/* Rewinds to step 0 with zeroed wavefields, keeping media, sources and
 * points; the next awp_run starts a new solve. */
awp_status awp_reset(awp_solver *s);

/* Frees every resource of the solver. */
awp_status awp_destroy(awp_solver *s);

/* Asynchronous stepping: enqueues up to `nsteps` steps on the solver's CUDA
 * stream and returns at once.  awp_query returns 1 when all enqueued work has
 * finished (0 otherwise, negative on error); awp_sync waits for it and
 * reports the stability monitor's result.  No reference counterpart (the
 * reference loop is synchronous, AWP-GPU-SGT/src/pmcl3d.c:841-960). */
awp_status awp_run_async(awp_solver *s, int nsteps);
int awp_query(awp_solver *s);
awp_status awp_sync(awp_solver *s);

/* Device layout of the wavefield arrays (awp_internal.h): element (i,j,k)
 * of the 1-based Fortran index space is at (k+1)*plane + (j+1)*pitch + i + 7. */
typedef struct {
    int nx, ny, nz;
    int pitch;      /* floats per row                */
    int plane;      /* floats per z level            */
    int64_t vol;    /* floats per array              */
} awp_layout;

/* Device pointer and layout of one field of the current wavefield (field
 * numbering as awp_get_field).  The pointer stays valid until the next step
 * of the fused stepper, which alternates between two buffers. */
awp_status awp_device_field(awp_solver *s, int comp, int field, float **ptr, awp_layout *layout);

/* FP64 wavefield energy: out[q] = sum over interior cells of u^2 + v^2 + w^2
 * for component q, fields = {u0, v0, w0, u1, v1, w1, ...} device arrays in
 * the layout L, out a device array of ncomp doubles.  Two deterministic passes
 * (per-block partial sums, then a fixed-order sum); the partial sums live in
 * a scratch buffer this call allocates and frees on the calling thread's
 * current device.  The quantity of the stability monitor.  No reference
 * counterpart (the reference has no monitor). */
awp_status awp_field_energy(const float *const *fields, int ncomp, const awp_layout *L, double *out);

/* awp_field_energy without any allocation (no counterpart in the reference).
 * For callers that must not allocate device memory mid-run: a host that runs
 * several solves side by side on one device (cudaFree waits for the whole
 * device, stalling every other solve's stream) or that admits work against a
 * fixed device-memory budget (an allocation here could fail or overrun it).
 * Same passes and result as awp_field_energy, enqueued on `stream` (a
 * cudaStream_t; NULL = the default stream) without synchronizing: `out` is
 * ready once that stream's work completes.  The partial sums live in a static
 * device array of the library (592 x 3 doubles), so ncomp is at most 3 and a
 * larger count is rejected with AWP_ERR_PARAM.  The first call on a device
 * does a one-time set-up (looks up that array's device address) and should
 * come before any stream capture; its address is kept for the life of the
 * process, so the device must not be reset (cudaDeviceReset, or anything else
 * that destroys its primary context) between calls.  Calls on one device
 * share the array: calls that overlap in time, from other streams or threads,
 * race and must be serialized by the caller.  A CUDA error left pending by
 * earlier work of the calling thread is reported (AWP_ERR_CUDA) without being
 * cleared, and nothing is launched. */
awp_status awp_field_energy_noalloc(const float *const *fields, int ncomp, const awp_layout *L, double *out,
                                    void *stream);

/* Energy of a solver's current wavefield (host output, ncomp doubles). */
awp_status awp_energy(awp_solver *s, double *out);

/* Per-kernel timing of the stepper (diagnostic, no reference counterpart).
 * Advances the solve by `nsteps` steps exactly as awp_run does, but records
 * CUDA events around every launch on the solver's stream and returns, per
 * kernel class, the launch count, the average device time of one launch and
 * the algorithmic bytes one launch moves (the compulsory traffic of its
 * arrays; the basis of the HBM roofline). */
#define AWP_MAX_KERNELS 8
typedef struct {
    int nkernels;
    char name[AWP_MAX_KERNELS][32];
    int launches[AWP_MAX_KERNELS];
    double ms_per_launch[AWP_MAX_KERNELS];
    double bytes_per_launch[AWP_MAX_KERNELS];
} awp_kernel_times;

awp_status awp_profile_steps(awp_solver *s, int nsteps, awp_kernel_times *out);

/* Launch shapes of the steppers (no reference counterpart).  Every shape
 * gives bit-identical results; they differ only in speed.  awp_create fills
 * them from measured defaults (and the AWP_TUNE_* environment variables);
 * awp_set_tuning replaces them at any point of a solve (a captured time-loop
 * graph is rebuilt on the next step). */
typedef struct {
    int kchunk_staged;       /* staged sweeps: z levels per work item (8..nz)          */
    int staged_qslow;        /* staged sweeps: 1 = one component over all tiles first  */
    int staged_rpt;          /* staged stress sweep, one component per item: tile rows
                                per thread (1, 2)                                      */
    int staged_rpt_vel;      /* staged velocity sweep: tile rows per thread (1, 2)     */
    int unroll;              /* z-loop unroll of the sweeps (1, 2)                     */
    int ty;                  /* two-sweep / fused steppers: block rows (4, 8, 16)      */
    int kchunk;              /* fused stepper: z levels per work item (8..nz)          */
    int kchunk_sweep;        /* two-sweep stepper: z levels per work item (8..nz)      */
    int staged_batch;        /* staged sweeps with all components of a tile in one work
                                item, sharing media tiles and cell coefficients:
                                bit 0 the stress sweep, bit 1 the velocity sweep
                                (default 1 up to 32 GiB of solver state, else 0) */
    int sm_limit;            /* persistent grids sized for this many SMs (0 = every
                                SM of the device): solves that share a GPU each take
                                their share instead of time-slicing the whole device */
} awp_tuning;

awp_status awp_get_tuning(awp_solver *s, awp_tuning *t);
awp_status awp_set_tuning(awp_solver *s, const awp_tuning *t);

/* Autotuner: times candidate launch shapes on a solver of these parameters
 * (the caller's media, or a homogeneous medium when media is NULL; the
 * wavefield filled with bounded noise, since a zero wavefield runs at higher
 * clocks under the power cap) for trial_steps (1..100000) time steps each, by
 * coordinate descent over the fields of awp_tuning that the chosen stepper
 * uses, and returns the fastest with its Gcell-updates/s.  With a cache path,
 * a result stored there for the same grid, components, precision, NVE,
 * stepper and GPU model is returned without timing, and a new result is
 * appended.  Allocates one solver's device memory for the duration of the
 * call. */
awp_status awp_autotune(const awp_params *p, const float *media, int trial_steps, const char *cache_path,
                        awp_tuning *best, double *gcell_updates_per_s);

/* Device memory one solver of these parameters would hold (admission). */
int64_t awp_footprint_bytes(const awp_params *p, int npts);

/* Algorithmic bytes per cell-update of the stepper these parameters select. */
double awp_bytes_per_cell_update(const awp_params *p);

const char *awp_status_string(awp_status st);
const char *awp_last_error(void);

/* ------------------------------------------------------------------------- */
/* SGT post-processing formats (SgtHead).                                    */
/* ------------------------------------------------------------------------- */

/* One component's SGT file image in RWG order, straight from the device
 * image: per point [6][NT] with XX <- YY, YY <- XX, ZZ, XY, XZ <- -YZ,
 * YZ <- -XZ, and for the z-force run every value first scaled by -2
 * (z_source = 1).  Replaces the separate reformat_awp / reformat_awp_mpi
 * pass (SgtHead/src/reformat_awp_mpi.c:104-122); `out` holds
 * awp_sgt_file_floats() floats. */
awp_status awp_get_sgt_rwg(awp_solver *s, int comp, int z_source, float *out);

/* The same reordering of a host SGT file image of npts points x [6][nt],
 * done on the current device (the reformat_awp tool's transform). */
awp_status awp_sgt_reorder_rwg(const float *in, int64_t npts, int nt, int z_source, float *out);

/* Media from RWG velocity volumes prefix.p, prefix.s, prefix.d (float,
 * x fastest, then z from the surface, then y; km/s and g/cm^3), transposed
 * to the AWP order on the device slab by slab and then transformed as
 * awp_load_media does; NVAR must be 3, RWG (nx, ny) = AWP (ny, nx).  Replaces
 * SgtHead's reformat_velocity pass plus the media read
 * (SgtHead/src/reformat_velocity.c:30-80, structure.f:107-116). */
awp_status awp_load_media_rwg(awp_solver *s, const char *prefix);

/* The AWP media file ([z][x][y][vp vs rho], y fastest, values x 1000) written
 * from RWG volumes of nx x ny x nz, the transpose done on the current device:
 * the reformat_velocity tool (SgtHead/src/reformat_velocity.c). */
awp_status awp_reformat_velocity(int nx, int ny, int nz, const char *prefix, const char *out);

/* Records of the RWG SGT header file (SgtHead/src/structure.h:164-220). */
typedef struct {
    int geoproj;
    float modellon, modellat, modelrot, xshift, yshift;
    int globnp, localnp, nt;
} awp_sgtmaster;
typedef struct {
    long long indx;
    int xsgt, ysgt, zsgt;
    float h;
} awp_sgtindex;
typedef struct {
    long long indx;
    int geoproj;
    float modellon, modellat, modelrot, xshift, yshift;
    int nt;
    float xazim, dt, tst, h, src_lat, src_lon, src_dep;
    int xsrc, ysrc, zsrc;
    float sgt_lat, sgt_lon, sgt_dep;
    int xsgt, ysgt, zsgt;
    float cdist, lam, mu, rho, xmom, ymom, zmom;
} awp_sgtheader;

/* Inputs of the header writer, the arguments of SgtHead's write_head. */
typedef struct {
    const char *modelbox;    /* model box file; line 5: "mlon= . mlat= . mrot= ." */
    const char *coordfile;   /* RWG SGT coordinate file: x y z indx lon lat dep   */
    const char *fdloc;       /* "xsrc ysrc" of the site (the reciprocal source)   */
    const char *gridout;     /* grid file with nx=, ny=, nz=                      */
    float spacing;           /* grid spacing (km)                                 */
    int nt;                  /* time steps of the run                             */
    float dt;                /* time step (s)                                     */
    int sgt_tinc;            /* SGT time decimation                               */
    const char *component;   /* "x", "y" or "z"                                   */
    float moment;            /* force moment of the run                           */
    float flo;               /* source filter frequency (Hz)                      */
    const char *media_file;  /* AWP media file (vp vs rho, m/s and kg/m^3)        */
    int mu_corr;             /* 1: unrelaxed mu (the -c option)                   */
} awp_sgthead_args;

/* Writes sgtmaster, sgtindex[np] and sgtheader[np] (the .sgthead file),
 * byte-identical to write_head (SgtHead/src/write_head.c:48-469). */
awp_status awp_write_sgt_header(const awp_sgthead_args *a, const char *outfile);

/* ------------------------------------------------------------------------- */
/* Serving: continuous batching of SGT solves on one GPU.                    */
/* No reference counterpart (the reference runs one solve per job).          */
/*                                                                           */
/* A request is admitted (arrival order, or shortest total work first) when  */
/* its device footprint (awp_footprint_bytes) fits in the server's HBM       */
/* budget, fewer than max_active solves are resident and the resident solves */
/* do not already fill the GPU; it is built (allocation, media, sources,     */
/* points) while the resident solves keep stepping.  Every resident solve    */
/* keeps its fields on the device and advances a chunk of steps at a time on */
/* its own CUDA stream, so the kernels of different requests overlap on the  */
/* GPU.  A finished request's SGT file images are copied into the caller's   */
/* buffer and its memory is released for the next admission.  Each          */
/* request's result is identical to running it alone (separate buffers,      */
/* fixed order).                                                             */
/* ------------------------------------------------------------------------- */

typedef struct awp_server awp_server;

typedef struct {
    awp_params params;
    const float *media;                  /* host [nz][ny][nx][nvar]; NULL if mediastart == 0 */
    int nsrc[AWP_MAX_COMP];
    const int *src_xyz[AWP_MAX_COMP];    /* [nsrc][3] per component           */
    const float *stf[AWP_MAX_COMP];      /* [nsrc][nst][6] per component      */
    int npts;
    const int *pts;                      /* [npts][3] cordfile coordinates    */
    float *sgt_out;                      /* caller-owned, ncomp * awp_sgt_floats_for() floats;
                                            must stay valid until the request ends */
} awp_request;

enum { AWP_REQ_QUEUED = 0, AWP_REQ_RUNNING = 1, AWP_REQ_DONE = 2, AWP_REQ_FAILED = 3, AWP_REQ_CANCELLED = 4 };

typedef struct {
    int state;                 /* AWP_REQ_*                                  */
    awp_status status;         /* final status (AWP_OK when DONE)            */
    double t_submit, t_admit, t_done;   /* seconds on the server's clock     */
    int64_t steps_done;
    int64_t footprint;         /* device bytes reserved for the request      */
} awp_request_info;

/* Device blocks freed by awp_destroy stay on the device for the next solver of
 * the process (a block serves a request of its size or up to 1/8 smaller; a
 * failed allocation returns them first;
 * AWP_DEVICE_CACHE_MB bounds the idle bytes per device, default half the device
 * memory, 0 = off).  This returns every idle block to the driver.  Work that
 * uses a solver's device pointers (awp_device_field) must be complete before
 * awp_destroy.  No reference counterpart (the reference runs one solve per
 * process). */
void awp_release_cached_memory(void);

/* Device memory of this library on a device: bytes held by live solvers and
 * bytes idle in the block cache (diagnostic; no reference counterpart). */
awp_status awp_device_memory(int device, int64_t *live_bytes, int64_t *idle_bytes);

/* hbm_budget <= 0: 90 % of the device's free memory at creation.
 * chunk_steps: fewest steps a resident solve advances per chunk. */
awp_status awp_server_create(int device, int64_t hbm_budget, int max_active, int chunk_steps, awp_server **out);

enum { AWP_SERVE_FIFO = 0, AWP_SERVE_SJF = 1, AWP_SERVE_FIFO_SRPT = 2 };
/* Admission order (AWP_SERVE_FIFO: arrival; AWP_SERVE_SJF: least total work,
 * cells x components x steps, first; AWP_SERVE_FIFO_SRPT: arrival, and of the
 * n >= 2 resident solves the one with the least remaining work has its grids
 * sized for 2/(n+1) of the SMs, the others for 1/(n+1) each, instead of equal
 * shares -- short solves leave sooner, long ones are still admitted in
 * order); fill_cells: resident cells x components
 * at which the GPU counts as full, so that a request is admitted next to
 * others only while their sum stays below it (default 32e6); chunk_cells:
 * cell-updates per chunk (default 4e8; at least chunk_steps steps).  Values
 * <= 0 keep the current setting. */
awp_status awp_server_configure(awp_server *sv, int policy, double fill_cells, double chunk_cells);
/* Copies the request description (host arrays must stay valid until the
 * request ends); returns its id. */
awp_status awp_submit(awp_server *sv, const awp_request *rq, int64_t *id);
awp_status awp_poll(awp_server *sv, int64_t id, awp_request_info *info);
/* Cancels a queued or running request; its output buffer is left as is. */
awp_status awp_cancel(awp_server *sv, int64_t id);
/* Waits until the request ends or timeout_s passes (AWP_ERR_TIMEOUT). */
awp_status awp_wait(awp_server *sv, int64_t id, double timeout_s, awp_request_info *info);
/* Seconds on the server's clock. */
double awp_server_time(awp_server *sv);
/* Stops the scheduler after cancelling what is still queued or running. */
awp_status awp_server_destroy(awp_server *sv);
/* Floats of one component's SGT file image for these parameters. */
int64_t awp_sgt_floats_for(const awp_params *p, int npts);

/* ------------------------------------------------------------------------- */
/* File formats of the drop-in driver (pmcl3d).                              */
/* ------------------------------------------------------------------------- */

/* Everything the IN3D file carries (AWP-ODC-SGT/src/io.f:327-417, in order). */
typedef struct {
    int igreen; float tmax, dh, dt; int npc, nd; float arbc, pht;
    int nsrc, nst, nx, ny, nz, npx, npy, npz;
    int ifault, checkpoint, isfcvlm, imd5, ivelocity, mediarestart, nvar, iost,
        partdeg, io_opt, iperf, idyna, socalq, nve;
    float mu_s, mu_d, fl, fh, fp;
    int read_step, write_step, write_step2;
    int nbgx, nedx, nskpx, nbgy, nedy, nskpy, nbgz, nedz, nskpz, ntiskp;
    int nbgx2, nedx2, nskpx2, nbgy2, nedy2, nskpy2, nbgz2, nedz2, nskpz2, ntiskp2;
    int ntiskp_sgt;
    char chkp[512], chkj[512], insrc[512], invel[512], insgt[512];
    char sxgro[512], sygro[512], szgro[512], sxgro2[512], sygro2[512], szgro2[512];
    char sgtgro[512], sgsn[512];
    char out_dir[512];   /* GPU command line -o / --OUT                      */
    int gpu_cli;         /* 1 when parsed from the GPU getopt command line   */
    int nt;              /* derived number of time steps                     */
} awp_in3d;

/* Reads an IN3D file: one "value NAME" per line in the fixed order of
 * AWP-ODC-SGT/src/io.f:327-417, blank lines allowed, quoted file names. */
awp_status awp_read_in3d(const char *path, awp_in3d *out);

/* Parses a pmcl3d command line in either reference form:
 *   pmcl3d [IN3D [SOURCE [MEDIA [CHKP [CHKJ]]]]]   (AWP-ODC-SGT/src/set_names.f:17-50)
 *   pmcl3d -T .. --IGREEN .. --DH ..               (AWP-GPU-SGT/src/command.c:117-340) */
awp_status awp_parse_command_line(int argc, char **argv, awp_in3d *out);

/* Fills solver parameters from a parsed IN3D. */
void awp_params_from_in3d(const awp_in3d *in, awp_params *p);

/* Reads a source file: IFAULT 0 text (first line x y z, then nst lines of six
 * comma/space separated values; AWP-ODC-SGT/src/source.f:170-198) or IFAULT 1
 * binary (int32[3] then float32[nst*6] per source; AWP-GPU-SGT/src/source.c:52-71).
 * xyz must hold 3*nsrc ints, stf nsrc*nst*6 floats. */
awp_status awp_read_source(const char *path, int ifault, int nsrc, int nst, int *xyz, float *stf);

/* Reads a cordfile: optional '#' lines, the point count, then "x y z" lines
 * (AWP-ODC-SGT/src/io.f:424-434).  *xyz is malloc'ed; free with awp_free. */
awp_status awp_read_cordfile(const char *path, int *npts, int **xyz);

void awp_free(void *p);

#ifdef __cplusplus
}
#endif
#endif /* AWP_SGT_H */
