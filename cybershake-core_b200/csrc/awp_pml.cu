/*
 * awp_pml.cu -- the PML absorbing boundary (NPC = 1) on the device.
 *
 * With NPC = 1 the reference steps the interior zone with its 4th-order
 * operators and 17 boundary zones (five planes, eight edges, four bottom
 * corners, width ND) with 2nd-order split-field PML routines
 * (AWP-ODC-SGT/src/pmcl3d.f:1234-1333, pml.f, bound.f:837-893).  Here the
 * usual sweeps step every cell without a sponge, and two kernels then
 * recompute the boundary zones from the same inputs: k_pml<0> after the
 * velocity sweep (before the free-surface velocity), k_pml<1> after the
 * stress sweep, followed by k_pml_fstr, the free-surface stress image of the
 * lateral columns it rewrote (fstr, operator.f:594-606).  The sweeps' values
 * in the boundary zones are overwritten; their memory variables there are
 * never read (the PML is elastic and r is a point quantity).
 *
 * The lateral zones (x or y within ND of a face) span the whole depth, under
 * the interior columns only the bottom ND levels are PML.  The 17 zones are
 * boxes of cells; each box gets its own run of thread blocks, one thread per
 * cell with x fastest, so every warp runs one zone's routine on consecutive
 * cells and a launch covers the PML volume and nothing else.  The split
 * arrays of a component sit in one device buffer, plane after plane (S N W E
 * B), each plane [split T/H][field][cells of the plane] with the plane's own
 * addressing (memory.f:217-300): S, N nx x ND x nz (N counted from the north
 * face), W, E ND x ny x nz (E from the east face), B nx x ny x ND.
 * Compiled without multiply-add contraction: bit-identical to the oracle.
 */
#include <cuda_runtime.h>

#include "awp_internal.h"
#include "awp_kernels.h"

namespace {

enum { PS = 0, PN = 1, PW = 2, PE = 3, PB = 4 };
enum { T_ = 0, H_ = 1 };
enum { PU, PV, PW_, PXX, PYY, PZZ, PXY, PXZ, PYZ };

/* one cell of one component, as the zone routines see it */
struct PmlCell {
    float *u1, *v1, *w1, *xx, *yy, *zz, *xy, *xz, *yz;
    const float *d1, *lam, *mu, *rf, *rh;
    float *split;
    const long long *n, *off;
    long long pidx[5];
    long c, SY, SZ;
    int i, j, k, nx, ny;
    float dt, dth, pht;
};

#define R(v) ((float)(v))
#define PML(pl, sp, fd) x.split[x.off[pl] + ((sp) * 9 + (fd)) * x.n[pl] + x.pidx[pl]]
#define PML_CELL_LOCALS                                                                             \
    float *u1 = x.u1, *v1 = x.v1, *w1 = x.w1, *xx = x.xx, *yy = x.yy, *zz = x.zz;                  \
    float *xy = x.xy, *xz = x.xz, *yz = x.yz;                                                       \
    const float *d1 = x.d1, *lam = x.lam, *mu = x.mu, *rf = x.rf, *rh = x.rh;                       \
    const long c = x.c, SX = 1, SY = x.SY, SZ = x.SZ;                                               \
    const int i = x.i, j = x.j, k = x.k, nx = x.nx, ny = x.ny;                                      \
    const float dt = x.dt, dth = x.dth, pht = x.pht;                                                \
    float d, dc, xl, xl2m, xm;                                                                      \
    (void)u1; (void)v1; (void)w1; (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz;       \
    (void)d1; (void)lam; (void)mu; (void)rf; (void)rh; (void)SX; (void)SY; (void)SZ; (void)i;       \
    (void)j; (void)k; (void)nx; (void)ny; (void)pht; (void)d; (void)dc; (void)xl; (void)xl2m; (void)xm;

#include "awp_pml_zones.cuh"

/* zone of a cell (bound.f:837-893): xs / ys 1 = within ND of the west /
 * south face, 2 = of the east / north face; zs 1 = within ND of the bottom */
__host__ __device__ __forceinline__ int pml_zone(int xs, int ys, int zs)
{
    if (!zs) {
        if (!xs) return ys == 1 ? 1 : (ys == 2 ? 3 : 18);
        if (!ys) return xs == 1 ? 2 : 4;
        return xs == 1 ? (ys == 1 ? 6 : 7) : (ys == 1 ? 8 : 9);
    }
    if (!xs && !ys) return 5;
    if (!xs) return ys == 1 ? 10 : 12;
    if (!ys) return xs == 1 ? 11 : 13;
    return xs == 1 ? (ys == 1 ? 14 : 15) : (ys == 1 ? 16 : 17);
}

/* pmlvel (pml.f:49-146) for one cell */
__device__ __forceinline__ void pml_vel_cell(int zone, const PmlCell &x)
{
    switch (zone) {
    case 1: m_us(x); m_vs(x); m_ws(x); break;
    case 2: m_uw(x); m_vw(x); m_ww(x); break;
    case 3: m_un(x); m_vn(x); m_wn(x); break;
    case 4: m_ue(x); m_ve(x); m_we(x); break;
    case 5: m_ub(x); m_vb(x); m_wb(x); break;
    case 6: m_usw(x); m_vsw(x); m_wsw(x); break;
    case 7: m_unw(x); m_vnw(x); m_wnw(x); break;
    case 8: m_use(x); m_vse(x); m_wse(x); break;
    case 9: m_une(x); m_vne(x); m_wne(x); break;
    case 10: m_usb(x); m_vsb(x); m_wsb(x); break;
    case 11: m_uwb(x); m_vwb(x); m_wwb(x); break;
    case 12: m_unb(x); m_vnb(x); m_wnb(x); break;
    case 13: m_ueb(x); m_veb(x); m_web(x); break;
    case 14: m_uswb(x); m_vswb(x); m_wswb(x); break;
    case 15: m_unwb(x); m_vnwb(x); m_wnwb(x); break;
    case 16: m_useb(x); m_vseb(x); m_wseb(x); break;
    case 17: m_uneb(x); m_vneb(x); m_wneb(x); break;
    default: break;
    }
}

/* pmlstr (pml.f:148-263) for one cell */
__device__ __forceinline__ void pml_str_cell(int zone, const PmlCell &x)
{
    switch (zone) {
    case 1: m_xyzs(x); m_xzs(x); m_yzs(x); m_xys(x); break;
    case 2: m_xyzw(x); m_xzw(x); m_yzw(x); m_xyw(x); break;
    case 3: m_xyzn(x); m_xzn(x); m_yzn(x); m_xyn(x); break;
    case 4: m_xyze(x); m_xze(x); m_yze(x); m_xye(x); break;
    case 5: m_xyzb(x); m_xzb(x); m_yzb(x); m_xyb(x); break;
    case 6: m_xyzsw(x); m_xzsw(x); m_yzsw(x); m_xysw(x); break;
    case 7: m_xyznw(x); m_xznw(x); m_yznw(x); m_xynw(x); break;
    case 8: m_xyzse(x); m_xzse(x); m_yzse(x); m_xyse(x); break;
    case 9: m_xyzne(x); m_xzne(x); m_yzne(x); m_xyne(x); break;
    case 10: m_xyzsb(x); m_xzsb(x); m_yzsb(x); m_xysb(x); break;
    case 11: m_xyzwb(x); m_xzwb(x); m_yzwb(x); m_xywb(x); break;
    case 12: m_xyznb(x); m_xznb(x); m_yznb(x); m_xynb(x); break;
    case 13: m_xyzeb(x); m_xzeb(x); m_yzeb(x); m_xyeb(x); break;
    case 14: m_xyzswb(x); m_xzswb(x); m_yzswb(x); m_xyswb(x); break;
    case 15: m_xyznwb(x); m_xznwb(x); m_yznwb(x); m_xynwb(x); break;
    case 16: m_xyzseb(x); m_xzseb(x); m_yzseb(x); m_xyseb(x); break;
    case 17: m_xyzneb(x); m_xzneb(x); m_yzneb(x); m_xyneb(x); break;
    default: break;
    }
}

constexpr int PML_BLOCK = 256;
/* Register budgets: the zone kernels wait on global loads, so resident warps
 * count for more than spills to L1.  Measured per step on 400x400x200 with
 * three components (velocity + stress part): 1.23 + 2.17 ms at 54 registers
 * (4 blocks per SM), 1.04 + 1.94 at 48 (5), 0.93 + 1.72 at 40 (6), 0.95 +
 * 1.68 at 32 (8, more spills). */
constexpr int PML_MINB_VEL = 6, PML_MINB_STR = 8;

/* the box a block belongs to: every thread of a block works in one zone, so
 * the zone dispatch below never diverges within a warp */
template <int N>
__device__ __forceinline__ const AwpPmlArgs::Box &pml_box_of(const AwpPmlArgs::Box (&box)[N], int b)
{
    int n = 0;
#pragma unroll
    for (int z = 1; z < N; ++z)
        if (b >= box[z].b0) n = z;
    return box[n];
}

/* PART 0: velocities of the boundary zones; PART 1: their stresses.  One
 * thread per cell of a zone box, x fastest, so a warp reads consecutive
 * cells of each array; blockIdx.y = component.  Cells are independent within
 * a part (a velocity update reads stresses and its own splits, a stress
 * update velocities and its own splits). */
template <int PART>
__global__ void __launch_bounds__(PML_BLOCK, PART == 0 ? PML_MINB_VEL : PML_MINB_STR) k_pml(AwpPmlArgs a)
{
    const AwpGeom &g = a.g;
    const AwpPmlArgs::Box &bx = pml_box_of(a.box, (int)blockIdx.x);
    const long long t = (long long)(blockIdx.x - bx.b0) * PML_BLOCK + threadIdx.x;
    const long long row = t / bx.ni;
    const int i = bx.i0 + (int)(t - row * bx.ni), j = bx.j0 + (int)(row % bx.nj), k = bx.k0 + (int)(row / bx.nj);
    if (k >= bx.k0 + bx.nk) return;
    const int q = blockIdx.y, nd = a.nd;
    const AwpComp &cp = a.comp[q];
    PmlCell x;
    x.u1 = cp.f[AF_U]; x.v1 = cp.f[AF_V]; x.w1 = cp.f[AF_W];
    x.xx = cp.f[AF_XX]; x.yy = cp.f[AF_YY]; x.zz = cp.f[AF_ZZ];
    x.xy = cp.f[AF_XY]; x.xz = cp.f[AF_XZ]; x.yz = cp.f[AF_YZ];
    x.d1 = a.d1; x.lam = a.lam; x.mu = a.mu; x.rf = a.rf; x.rh = a.rh;
    x.split = a.split[q]; x.n = a.n; x.off = a.off;
    x.SY = g.px; x.SZ = g.plane;
    x.i = i; x.j = j; x.nx = g.nx; x.ny = g.ny;
    x.dt = a.dt; x.dth = a.dth; x.pht = a.pht;
    x.k = k;
    x.c = g.idx(i, j, k);
    x.pidx[PS] = ((long long)(k - 1) * nd + (j - 1)) * g.nx + (i - 1);
    x.pidx[PN] = ((long long)(k - 1) * nd + (g.ny - j)) * g.nx + (i - 1);
    x.pidx[PW] = ((long long)(k - 1) * g.ny + (j - 1)) * nd + (i - 1);
    x.pidx[PE] = ((long long)(k - 1) * g.ny + (j - 1)) * nd + (g.nx - i);
    x.pidx[PB] = ((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1);
    if (PART == 0) pml_vel_cell(bx.zone, x);
    else pml_str_cell(bx.zone, x);
}

/* after the stress part: the free-surface image of each lateral column
 * (fstr, operator.f:594-606), which the stress sweep wrote from the values
 * the PML has since replaced; one thread per column of the lateral boxes */
__global__ void __launch_bounds__(PML_BLOCK) k_pml_fstr(AwpPmlArgs a)
{
    const AwpGeom &g = a.g;
    const AwpPmlArgs::Box &bx = pml_box_of(a.col, (int)blockIdx.x);
    const int t = (int)(blockIdx.x - bx.b0) * PML_BLOCK + (int)threadIdx.x;
    const int i = bx.i0 + t % bx.ni, j = bx.j0 + t / bx.ni;
    if (j >= bx.j0 + bx.nj) return;
    const AwpComp &cp = a.comp[blockIdx.y];
    const long sz = g.plane, ct = g.idx(i, j, g.nz);
    float *ZZ = cp.f[AF_ZZ], *XZ = cp.f[AF_XZ], *YZ = cp.f[AF_YZ];
    ZZ[ct + sz] = -ZZ[ct];
    ZZ[ct + 2 * sz] = -ZZ[ct - sz];
    XZ[ct + sz] = -XZ[ct - sz];
    XZ[ct + 2 * sz] = -XZ[ct - 2 * sz];
    YZ[ct + sz] = -YZ[ct - sz];
    YZ[ct + 2 * sz] = -YZ[ct - 2 * sz];
    XZ[ct] = 0.0f;
    YZ[ct] = 0.0f;
}

}  // namespace

/* The 17 zones as boxes: x (and y) within nd of the low face, of the high
 * face, or between; z within nd of the bottom or above.  Each box gets a
 * contiguous run of blocks, in increasing order (pml_box_of relies on it). */
void awp_pml_boxes(AwpPmlArgs &a)
{
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz, nd = a.nd;
    const int n3[3] = {nx, ny, nz};
    auto range = [&](int axis, int side, int &s0, int &n) {   /* side 1 low band, 2 high band, 0 between */
        const int N = n3[axis];
        if (axis == 2) { s0 = side ? 1 : nd + 1; n = side ? nd : N - nd; return; }
        if (side == 1) { s0 = 1; n = nd; }
        else if (side == 2) { s0 = N - nd + 1; n = nd; }
        else { s0 = nd + 1; n = N - 2 * nd; }
    };
    int nb = 0, nbox = 0, ncol = 0, ncb = 0;
    for (int zs = 1; zs >= 0; --zs)
        for (int ys = 0; ys < 3; ++ys)
            for (int xs = 0; xs < 3; ++xs) {
                if (!xs && !ys && !zs) continue;
                AwpPmlArgs::Box b;
                b.zone = pml_zone(xs, ys, zs);
                range(0, xs, b.i0, b.ni);
                range(1, ys, b.j0, b.nj);
                range(2, zs, b.k0, b.nk);
                const long long cells = (long long)b.ni * b.nj * b.nk;
                b.b0 = nb;
                b.nb = (int)((cells + PML_BLOCK - 1) / PML_BLOCK);
                nb += b.nb;
                a.box[nbox++] = b;
                if (!zs) {                                   /* a lateral box: its columns */
                    AwpPmlArgs::Box c = b;
                    c.b0 = ncb;
                    c.nb = (b.ni * b.nj + PML_BLOCK - 1) / PML_BLOCK;
                    ncb += c.nb;
                    a.col[ncol++] = c;
                }
            }
    a.nblk = nb;
    a.ncolblk = ncb;
}

cudaError_t awp_launch_pml(const AwpPmlArgs &a, int part, cudaStream_t st)
{
    const dim3 grid(a.nblk, a.ncomp), gcol(a.ncolblk, a.ncomp);
    if (a.nblk <= 0 || a.ncomp <= 0) return cudaErrorInvalidValue;
    if (part == 0) {
        k_pml<0><<<grid, PML_BLOCK, 0, st>>>(a);
    } else {
        k_pml<1><<<grid, PML_BLOCK, 0, st>>>(a);
        if (a.ncolblk > 0) k_pml_fstr<<<gcol, PML_BLOCK, 0, st>>>(a);
    }
    return cudaGetLastError();
}

/* inipml (pml.f:4-44) in FP32, the statement order of the Fortran: rf / rh
 * hold nd + 1 values, index 1 at the outer edge */
void awp_pml_profiles(int nd, float arbc, float dh, float vs_min, float vs_max, float *rf, float *rh)
{
    const float c0 = 0.f, c1 = 8.f / 15.f, c2 = -(3.f / 100.f), c3 = 1.f / 1500.f;
    const float f = c0 + (float)nd * c1 + (float)(nd * nd) * c2 + (float)(nd * nd * nd) * c3;
    const float v = 1.f / (0.5f * (1.f / vs_min + 1.f / vs_max));
    const float coef = arbc * f * v / ((float)nd * dh);
    for (int i = 1; i <= nd; i++) rf[nd + 1 - i] = coef * (float)i * (float)i / (float)(nd * nd);
    rh[1] = rf[1] + 0.50f * (rf[1] - rf[2]);
    for (int i = 2; i <= nd; i++) rh[i] = 0.5f * (rf[i - 1] + rf[i]);
}
