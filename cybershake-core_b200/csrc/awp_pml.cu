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
 * the interior columns only the bottom ND levels are PML.  One thread takes
 * up to eight levels of one (i, j) column: one launch covers the bottom ND
 * levels of every column, a second the levels above of the columns in the
 * tiles that touch a lateral band (a tile list made once per solver), so the
 * thread count follows the PML volume rather than the columns.  The split
 * arrays of a
 * component sit in one device buffer, plane after plane (S N W E B), each
 * plane [split T/H][field][cells of the plane] with the plane's own
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
__device__ __forceinline__ int pml_zone(int xs, int ys, int zs)
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

constexpr int PML_KC = 8;   /* z levels per thread */

/* PART 0: velocities of the boundary zones; PART 1: their stresses.  The
 * bottom launch (LATERAL 0) covers levels 1..nd of every column, the lateral
 * one levels nd+1..nz of the columns within nd of a lateral face, its blocks
 * taken from the tile list; blockIdx.z = chunk of PML_KC levels x component.
 * Cells are independent within a part (a velocity update reads stresses and
 * its own splits, a stress update velocities and its own splits). */
template <int PART, int LATERAL>
__global__ void __launch_bounds__(256) k_pml(AwpPmlArgs a)
{
    const AwpGeom &g = a.g;
    int tx, ty;
    if (LATERAL) {
        const int2 t = a.tiles[blockIdx.x];
        tx = t.x; ty = t.y;
    } else {
        tx = blockIdx.x; ty = blockIdx.y;
    }
    const int i = tx * 32 + threadIdx.x + 1, j = ty * 8 + threadIdx.y + 1;
    const int q = blockIdx.z % a.ncomp, kc = blockIdx.z / a.ncomp;
    if (i > g.nx || j > g.ny) return;
    const int nd = a.nd;
    const int xs = i <= nd ? 1 : (i > g.nx - nd ? 2 : 0), ys = j <= nd ? 1 : (j > g.ny - nd ? 2 : 0);
    int k0, k1;
    if (LATERAL) {
        if (!xs && !ys) return;
        k0 = nd + 1 + kc * PML_KC;
        k1 = min(g.nz, k0 + PML_KC - 1);
    } else {
        k0 = 1 + kc * PML_KC;
        k1 = min(nd, k0 + PML_KC - 1);
    }
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
    for (int k = k0; k <= k1; ++k) {
        x.k = k;
        x.c = g.idx(i, j, k);
        x.pidx[PS] = ((long long)(k - 1) * nd + (j - 1)) * g.nx + (i - 1);
        x.pidx[PN] = ((long long)(k - 1) * nd + (g.ny - j)) * g.nx + (i - 1);
        x.pidx[PW] = ((long long)(k - 1) * g.ny + (j - 1)) * nd + (i - 1);
        x.pidx[PE] = ((long long)(k - 1) * g.ny + (j - 1)) * nd + (g.nx - i);
        x.pidx[PB] = ((long long)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1);
        const int zone = pml_zone(xs, ys, k <= nd);
        if (PART == 0) pml_vel_cell(zone, x);
        else pml_str_cell(zone, x);
    }
}

/* after the stress part: the free-surface image of each lateral column
 * (fstr, operator.f:594-606), which the stress sweep wrote from the values
 * the PML has since replaced */
__global__ void __launch_bounds__(256) k_pml_fstr(AwpPmlArgs a)
{
    const AwpGeom &g = a.g;
    const int2 t = a.tiles[blockIdx.x];
    const int i = t.x * 32 + threadIdx.x + 1, j = t.y * 8 + threadIdx.y + 1, q = blockIdx.z;
    if (i > g.nx || j > g.ny || q >= a.ncomp) return;
    const int nd = a.nd;
    if (i > nd && i <= g.nx - nd && j > nd && j <= g.ny - nd) return;
    const AwpComp &cp = a.comp[q];
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

int awp_pml_lateral_tiles(int nx, int ny, int nd, int2 *out)
{
    int n = 0;
    for (int by = 0; by < (ny + 7) / 8; by++)
        for (int bx = 0; bx < (nx + 31) / 32; bx++) {
            const int i0 = bx * 32 + 1, i1 = bx * 32 + 32 < nx ? bx * 32 + 32 : nx;
            const int j0 = by * 8 + 1, j1 = by * 8 + 8 < ny ? by * 8 + 8 : ny;
            if (i0 <= nd || i1 > nx - nd || j0 <= nd || j1 > ny - nd) {
                if (out) out[n] = make_int2(bx, by);
                n++;
            }
        }
    return n;
}

cudaError_t awp_launch_pml(const AwpPmlArgs &a, int part, cudaStream_t st)
{
    const dim3 b(32, 8);
    const int nbot = (a.nd + PML_KC - 1) / PML_KC, nlat = (a.g.nz - a.nd + PML_KC - 1) / PML_KC;
    const dim3 gbot((a.g.nx + 31) / 32, (a.g.ny + 7) / 8, nbot * a.ncomp);
    const dim3 glat(a.ntiles, 1, nlat * a.ncomp);
    if (part == 0) {
        k_pml<0, 0><<<gbot, b, 0, st>>>(a);
        if (a.ntiles > 0 && nlat > 0) k_pml<0, 1><<<glat, b, 0, st>>>(a);
    } else {
        k_pml<1, 0><<<gbot, b, 0, st>>>(a);
        if (a.ntiles > 0 && nlat > 0) k_pml<1, 1><<<glat, b, 0, st>>>(a);
        if (a.ntiles > 0) k_pml_fstr<<<dim3(a.ntiles, 1, a.ncomp), b, 0, st>>>(a);
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
