/*
 * awp_oracle_pml.h -- the PML absorbing boundary (NPC = 1) of the oracle:
 * AWP-ODC-SGT/src/pml.f restated routine by routine.  TEST INFRASTRUCTURE
 * ONLY, included by awp_oracle.c (the same FP32 / FP64 builds).
 *
 * Single rank: the grid is cut into 18 zones (bound.f:837-893) -- the
 * interior zone 18 stepped by the usual 4th-order operators without a sponge
 * (dvel / dstrq, operator.f:4-45, viscoop.f:4-22), and 17 PML zones (five
 * planes S W N E B, eight edges, four bottom corners) stepped by these
 * 2nd-order split-field routines (elastic, cell-local moduli).  Each plane
 * keeps a T and an H split of all nine fields (memory.f:217-300); edges and
 * corners store their splits in the arrays of their planes.  The damping
 * profiles rf (full nodes) and rh (half nodes) come from inipml
 * (pml.f:4-44).  The free surface, the sources and the SGT gather are those
 * of the Cerjan runs.
 *
 * Every routine below restates the arithmetic statements of the pml.f
 * subroutine its comment names, in their order and grouping (R() marks a
 * real constant; PML(plane, split, field) is the routine's split array at the
 * cell; the field arrays are indexed from the cell c with strides SX SY SZ).
 * PARITY: no reference run pins this part (the Fortran cannot be built here
 * and the CUDA variant has no PML); tests/test_pml.py checks absorption and
 * the mirror symmetry of the zones' restatements.
 */

#define R(x) ((real)(x))
enum { PS = 0, PN = 1, PW = 2, PE = 3, PB = 4 };         /* planes: south north west east bottom */
enum { T_ = 0, H_ = 1 };                                  /* splits                               */
enum { PU, PV, PW_, PXX, PYY, PZZ, PXY, PXZ, PYZ };       /* fields of a split                    */
#define PML(pl, sp, fd) h->pml[pl][sp][fd][pidx[pl]]

/* one PML routine's loop over its zone r = {x0, x1, y0, y1, z0, z1}, with
 * the cell's index in every plane's arrays (pml.f's (i,j,k), (i,ny-j+1,k),
 * (nx-i+1,j,k) addressing) */
#define PML_BEGIN                                                                              \
    const orc_params *p = &h->p;                                                               \
    const int nx = p->nx, ny = p->ny, nd = p->nd;                                              \
    const real dt = (real)p->dt, dth = (real)p->dt / (real)p->dh, pht = (real)p->pht;          \
    const real *rf = h->rf, *rh = h->rh;                                                       \
    real *u1 = h->f[F_U1], *v1 = h->f[F_V1], *w1 = h->f[F_W1];                                 \
    real *xx = h->f[F_XX], *yy = h->f[F_YY], *zz = h->f[F_ZZ];                                 \
    real *xy = h->f[F_XY], *xz = h->f[F_XZ], *yz = h->f[F_YZ];                                 \
    const real *d1 = h->f[F_D1], *lam = h->f[F_LAM], *mu = h->f[F_MU];                         \
    const long SX = 1, SY = h->sx, SZ = (long)h->sx * h->sy;                                   \
    (void)nx; (void)ny; (void)pht; (void)rf; (void)rh; (void)d1; (void)lam; (void)mu; (void)SX; \
    (void)u1; (void)v1; (void)w1; (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz;   \
    (void)SY; (void)SZ;                                                                        \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int k = r[4]; k <= r[5]; k++)                                                         \
        for (int j = r[2]; j <= r[3]; j++)                                                     \
            for (int i = r[0]; i <= r[1]; i++) {                                               \
                const long c = (long)IDX(h, i, j, k);                                          \
                const long pidx[5] = {                                                         \
                    ((long)(k - 1) * nd + (j - 1)) * nx + (i - 1),                             \
                    ((long)(k - 1) * nd + (ny - j)) * nx + (i - 1),                            \
                    ((long)(k - 1) * ny + (j - 1)) * nd + (i - 1),                             \
                    ((long)(k - 1) * ny + (j - 1)) * nd + (nx - i),                            \
                    ((long)(k - 1) * ny + (j - 1)) * nx + (i - 1)};                            \
                real d, dc, xl, xl2m, xm;                                                      \
                (void)d; (void)dc; (void)xl; (void)xl2m; (void)xm;
#define PML_END }

/* m_un: pml.f:267-300 */
static void orc_m_un(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*rf[ny-j+1]))/(R(2.) + dt*rf[ny-j+1]);
        PML(PN, H_, PU) = (R(2.)*dth*d* ((xx[c] - xx[c - SX]) + (xz[c] - xz[c - SZ])) + PML(PN, H_, PU)* (R(2.) - dt * pht * rf[ny-j+1]))/ (R(2.) + dt * pht * rf[ny-j+1]);
        u1[c] = PML(PN, T_, PU) + PML(PN, H_, PU);
    PML_END
}

/* m_vn: pml.f:304-337 */
static void orc_m_vn(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
        PML(PN, H_, PV) = (R(2.)*dth*d*((xy[c + SX] - xy[c]) + (yz[c] - yz[c - SZ])) + PML(PN, H_, PV) * (R(2.) - dt*pht*rh[ny-j+1]))/ (R(2.) + dt*pht*rh[ny-j+1]);
        v1[c] = PML(PN, T_, PV) + PML(PN, H_, PV);
    PML_END
}

/* m_wn: pml.f:341-374 */
static void orc_m_wn(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*rf[ny-j+1]))/(R(2.) + dt*rf[ny-j+1]);
        PML(PN, H_, PW_) = (R(2.)*dth*d*((xz[c + SX] - xz[c]) + (zz[c + SZ] - zz[c])) + PML(PN, H_, PW_) * (R(2.) - dt * pht*rf[ny-j+1])) / (R(2.) + dt * pht*rf[ny-j+1]);
        w1[c] = PML(PN, T_, PW_) + PML(PN, H_, PW_);
    PML_END
}

/* m_us: pml.f:378-409 */
static void orc_m_us(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*rh[j]))/(R(2.) + dt*rh[j]);
        PML(PS, H_, PU) = (R(2.)*d*dth*((xx[c] - xx[c - SX]) + (xz[c] - xz[c - SZ]))+ PML(PS, H_, PU)* (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
        u1[c] = PML(PS, T_, PU) + PML(PS, H_, PU);
    PML_END
}

/* m_vs: pml.f:413-444 */
static void orc_m_vs(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*rf[j]))/(R(2.) + dt*rf[j]);
        PML(PS, H_, PV) = (R(2.)*d*dth*((xy[c + SX] - xy[c]) + (yz[c] - yz[c - SZ])) + PML(PS, H_, PV)* (R(2.) - dt*pht*rf[j]))/(R(2.) + dt*pht*rf[j]);
        v1[c] = PML(PS, T_, PV) + PML(PS, H_, PV);
    PML_END
}

/* m_ws: pml.f:448-479 */
static void orc_m_ws(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*rh[j]))/(R(2.) + dt*rh[j]);
        PML(PS, H_, PW_) = (R(2.)*d*dth*((xz[c + SX] - xz[c]) + (zz[c + SZ] - zz[c]))+ PML(PS, H_, PW_) * (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
        w1[c] = PML(PS, T_, PW_) + PML(PS, H_, PW_);
    PML_END
}

/* m_uw: pml.f:483-514 */
static void orc_m_uw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*rh[i]))/(R(2.) + dt*rh[i]);
        PML(PW, H_, PU) = (R(2.)*d*dth*((xy[c] - xy[c - SY]) + (xz[c] - xz[c - SZ]))+ PML(PW, H_, PU)* (R(2.) - dt*pht*rh[i]))/(R(2.) + dt*pht*rh[i]);
        u1[c] = PML(PW, T_, PU) + PML(PW, H_, PU);
    PML_END
}

/* m_vw: pml.f:518-549 */
static void orc_m_vw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*rf[i]))/(R(2.) + dt*rf[i]);
        PML(PW, H_, PV) = (R(2.)*d*dth*((yy[c + SY] - yy[c]) + (yz[c] - yz[c - SZ])) + PML(PW, H_, PV) * (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
        v1[c] = PML(PW, T_, PV) + PML(PW, H_, PV);
    PML_END
}

/* m_ww: pml.f:553-584 */
static void orc_m_ww(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*rf[i]))/(R(2.) + dt*rf[i]);
        PML(PW, H_, PW_) = (R(2.)*d*dth*((yz[c] - yz[c - SY]) + (zz[c + SZ] - zz[c])) + PML(PW, H_, PW_)* (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
        w1[c] = PML(PW, T_, PW_) + PML(PW, H_, PW_);
    PML_END
}

/* m_ue: pml.f:588-619 */
static void orc_m_ue(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*rf[nx-i+1]))/(R(2.) + dt*rf[nx-i+1]);
        PML(PE, H_, PU) = (R(2.)*d*dth*((xy[c] - xy[c - SY]) + (xz[c] - xz[c - SZ])) + PML(PE, H_, PU)* (R(2.) - dt*pht*rf[nx-i+1]))/(R(2.) + dt*pht*rf[nx-i+1]);
        u1[c] = PML(PE, T_, PU) + PML(PE, H_, PU);
    PML_END
}

/* m_ve: pml.f:623-655 */
static void orc_m_ve(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*rh[nx-i+1]))/(R(2.) + dt*rh[nx-i+1]);
        PML(PE, H_, PV) = (R(2.)*d*dth*( (yy[c + SY] - yy[c]) + (yz[c] - yz[c - SZ])) + PML(PE, H_, PV) * (R(2.) - dt*pht*rh[nx-i+1]))/(R(2.) + dt*pht*rh[nx-i+1]);
        v1[c] = PML(PE, T_, PV) + PML(PE, H_, PV);
    PML_END
}

/* m_we: pml.f:659-691 */
static void orc_m_we(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*rh[nx-i+1]))/(R(2.) + dt*rh[nx-i+1]);
        PML(PE, H_, PW_) = (R(2.)*d*dth*( (yz[c] - yz[c - SY]) + (zz[c + SZ] - zz[c])) + PML(PE, H_, PW_) * (R(2.) - dt*pht*rh[nx-i+1]))/(R(2.) + dt*pht*rh[nx-i+1]);
        w1[c] = PML(PE, T_, PW_) + PML(PE, H_, PW_);
    PML_END
}

/* m_ub: pml.f:695-727 */
static void orc_m_ub(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*rh[k]))/(R(2.) + dt*rh[k]);
        PML(PB, H_, PU) = (R(2.)*d*dth*( (xy[c] - xy[c - SY]) + (xx[c] - xx[c - SX])) + PML(PB, H_, PU)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
        u1[c] = PML(PB, T_, PU) + PML(PB, H_, PU);
    PML_END
}

/* m_vb: pml.f:731-763 */
static void orc_m_vb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*rh[k]))/(R(2.) + dt*rh[k]);
        PML(PB, H_, PV) = (R(2.)*d*dth*( (xy[c + SX] - xy[c]) + (yy[c + SY] - yy[c])) + PML(PB, H_, PV)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
        v1[c] = PML(PB, T_, PV) + PML(PB, H_, PV);
    PML_END
}

/* m_wb: pml.f:767-799 */
static void orc_m_wb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
        PML(PB, H_, PW_) = (R(2.)*d*dth*( (yz[c] - yz[c - SY]) + (xz[c + SX] - xz[c])) + PML(PB, H_, PW_)* (R(2.) - dt*pht*rf[k]))/(R(2.) + dt*pht*rf[k]);
        w1[c] = PML(PB, T_, PW_) + PML(PB, H_, PW_);
    PML_END
}

/* m_usw: pml.f:806-843 */
static void orc_m_usw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rh[i];
        PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[i];
        PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[i]);
        PML(PS, H_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PS, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PS, T_, PU) + PML(PW, T_, PU) + PML(PS, H_, PU);
    PML_END
}

/* m_vsw: pml.f:847-884 */
static void orc_m_vsw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[j] + pht*rf[i];
        PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rf[i];
        PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rf[i]);
        PML(PS, H_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PS, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PS, T_, PV) + PML(PW, T_, PV) + PML(PS, H_, PV);
    PML_END
}

/* m_wsw: pml.f:888-925 */
static void orc_m_wsw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rf[i];
        PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i];
        PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[i]);
        PML(PS, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PS, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PS, T_, PW_) + PML(PW, T_, PW_) + PML(PS, H_, PW_);
    PML_END
}

/* m_use: pml.f:929-966 */
static void orc_m_use(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rf[nx-i+1];
        PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[nx-i+1];
        PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[nx-i+1]);
        PML(PS, H_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PS, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PS, T_, PU) + PML(PE, T_, PU) + PML(PS, H_, PU);
    PML_END
}

/* m_vse: pml.f:970-1007 */
static void orc_m_vse(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[j] + pht*rh[nx-i+1];
        PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[nx-i+1];
        PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rh[nx-i+1]);
        PML(PS, H_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ])+ PML(PS, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PS, T_, PV) + PML(PE, T_, PV) + PML(PS, H_, PV);
    PML_END
}

/* m_wse: pml.f:1011-1048 */
static void orc_m_wse(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht * rh[nx-i+1];
        PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1];
        PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[nx-i+1]);
        PML(PS, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PS, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PS, T_, PW_) + PML(PE, T_, PW_) + PML(PS, H_, PW_);
    PML_END
}

/* m_unw: pml.f:1052-1089 */
static void orc_m_unw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc = rf[ny-j+1] + pht*rh[i];
        PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc = pht*rf[ny-j+1] + rh[i];
        PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc = pht*(rf[ny-j+1] + rh[i]);
        PML(PN, H_, PU) =(R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PN, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PN, T_, PU) + PML(PW, T_, PU) + PML(PN, H_, PU);
    PML_END
}

/* m_vnw: pml.f:1093-1130 */
static void orc_m_vnw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc = rh[ny-j+1] + pht * rf[i];
        PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc = pht * rh[ny-j+1] + rf[i];
        PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc = pht * (rh[ny-j+1] + rf[i]);
        PML(PN, H_, PV) = (R(2.)* dth*d*(yz[c] - yz[c - SZ]) + PML(PN, H_, PV) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PN, T_, PV) + PML(PW, T_, PV) + PML(PN, H_, PV);
    PML_END
}

/* m_wnw: pml.f:1134-1171 */
static void orc_m_wnw(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht * rf[i];
        PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht * rf[ny-j+1] + rf[i];
        PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc = pht * (rf[ny-j+1] + rf[i]);
        PML(PN, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PN, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PN, T_, PW_) + PML(PW, T_, PW_) + PML(PN, H_, PW_);
    PML_END
}

/* m_une: pml.f:1175-1212 */
static void orc_m_une(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht*rf[nx-i+1];
        PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[nx-i+1];
        PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rf[nx-i+1]);
        PML(PN, H_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ])+ PML(PN, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PN, T_, PU) + PML(PE, T_, PU) + PML(PN, H_, PU);
    PML_END
}

/* m_vne: pml.f:1216-1253 */
static void orc_m_vne(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[ny-j+1] + pht*rh[nx-i+1];
        PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rh[nx-i+1];
        PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[ny-j+1] + rh[nx-i+1]);
        PML(PN, H_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PN, H_, PV) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PN, T_, PV) + PML(PE, T_, PV) + PML(PN, H_, PV);
    PML_END
}

/* m_wne: pml.f:1257-1294 */
static void orc_m_wne(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht * rh[nx-i+1];
        PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1];
        PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[nx-i+1]);
        PML(PN, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PN, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PN, T_, PW_) + PML(PE, T_, PW_) + PML(PN, H_, PW_);
    PML_END
}

/* m_usb: pml.f:1302-1339 */
static void orc_m_usb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rh[k];
        PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[k]);
        PML(PB, H_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PS, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
    PML_END
}

/* m_vsb: pml.f:1343-1380 */
static void orc_m_vsb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[j] + pht*rh[k];
        PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rh[k]);
        PML(PB, H_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PS, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
    PML_END
}

/* m_wsb: pml.f:1384-1421 */
static void orc_m_wsb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rf[k];
        PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[k]);
        PML(PB, H_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PB, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PS, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
    PML_END
}

/* m_unb: pml.f:1425-1462 */
static void orc_m_unb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht*rh[k];
        PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[k]);
        PML(PB, H_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PN, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
    PML_END
}

/* m_vnb: pml.f:1466-1503 */
static void orc_m_vnb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[ny-j+1] + pht*rh[k];
        PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[ny-j+1] + rh[k]);
        PML(PB, H_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PN, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
    PML_END
}

/* m_wnb: pml.f:1507-1544 */
static void orc_m_wnb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht*rf[k];
        PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rf[k]);
        PML(PB, H_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PB, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PN, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
    PML_END
}

/* m_uwb: pml.f:1548-1585 */
static void orc_m_uwb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[i] + pht*rh[k];
        PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[i] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[i] + rh[k]);
        PML(PB, H_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PW, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
    PML_END
}

/* m_vwb: pml.f:1589-1626 */
static void orc_m_vwb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[i] + pht*rh[k];
        PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[i] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[i] + rh[k]);
        PML(PB, H_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PW, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
    PML_END
}

/* m_wwb: pml.f:1630-1667 */
static void orc_m_wwb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[i] + pht*rf[k];
        PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[i] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[i] + rf[k]);
        PML(PB, H_, PW_) = (R(2.)* dth*d*(yz[c] - yz[c - SY]) + PML(PB, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PW, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
    PML_END
}

/* m_ueb: pml.f:1671-1708 */
static void orc_m_ueb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[nx-i+1] + pht*rh[k];
        PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[nx-i+1] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[nx-i+1] + rh[k]);
        PML(PB, H_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY])+ PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PE, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
    PML_END
}

/* m_veb: pml.f:1712-1749 */
static void orc_m_veb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[nx-i+1] + rh[k]);
        PML(PB, H_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PE, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
    PML_END
}

/* m_web: pml.f:1753-1790 */
static void orc_m_web(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[nx-i+1] + pht*rf[k];
        PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[nx-i+1] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[nx-i+1] + rf[k]);
        PML(PB, H_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PB, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PE, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
    PML_END
}

/* m_uswb: pml.f:1797-1834 */
static void orc_m_uswb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rh[i] + pht*rh[k];
        PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[i] + pht*rh[k];
        PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rh[i] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PS, T_, PU) + PML(PW, T_, PU) + PML(PB, T_, PU);
    PML_END
}

/* m_vswb: pml.f:1838-1875 */
static void orc_m_vswb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[j] + pht*rf[i] + pht*rh[k];
        PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rf[i] + pht*rh[k];
        PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + pht*rf[i] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PS, T_, PV) + PML(PW, T_, PV) + PML(PB, T_, PV);
    PML_END
}

/* m_wswb: pml.f:1879-1916 */
static void orc_m_wswb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rf[i] + pht*rf[k];
        PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i] + pht*rf[k];
        PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rf[i] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PS, T_, PW_) + PML(PW, T_, PW_) + PML(PB, T_, PW_);
    PML_END
}

/* m_unwb: pml.f:1920-1957 */
static void orc_m_unwb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht*rh[i] + pht*rh[k];
        PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[i] + pht*rh[k];
        PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rh[i] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PN, T_, PU) + PML(PW, T_, PU) + PML(PB, T_, PU);
    PML_END
}

/* m_vnwb: pml.f:1961-1998 */
static void orc_m_vnwb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[ny-j+1] + pht*rf[i] + pht*rh[k];
        PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rf[i] + pht*rh[k];
        PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + pht*rf[i] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PN, T_, PV) + PML(PW, T_, PV) + PML(PB, T_, PV);
    PML_END
}

/* m_wnwb: pml.f:2002-2039 */
static void orc_m_wnwb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht*rf[i] + pht*rf[k];
        PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[i] + pht*rf[k];
        PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rf[i] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PN, T_, PW_) + PML(PW, T_, PW_) + PML(PB, T_, PW_);
    PML_END
}

/* m_useb: pml.f:2043-2080 */
static void orc_m_useb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rf[nx-i+1] + pht*rh[k];
        PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[nx-i+1] + pht*rh[k];
        PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rf[nx-i+1] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PS, T_, PU) + PML(PE, T_, PU) + PML(PB, T_, PU);
    PML_END
}

/* m_vseb: pml.f:2084-2121 */
static void orc_m_vseb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[j] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PS, T_, PV) + PML(PE, T_, PV) + PML(PB, T_, PV);
    PML_END
}

/* m_wseb: pml.f:2125-2162 */
static void orc_m_wseb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[j] + pht*rh[nx-i+1] + pht*rf[k];
        PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1] + pht*rf[k];
        PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rh[nx-i+1] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PS, T_, PW_) + PML(PE, T_, PW_) + PML(PB, T_, PW_);
    PML_END
}

/* m_uneb: pml.f:2166-2203 */
static void orc_m_uneb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht*rf[nx-i+1] + pht*rh[k];
        PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[nx-i+1] + pht*rh[k];
        PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rf[nx-i+1] + rh[k];
        PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        u1[c] = PML(PN, T_, PU) + PML(PE, T_, PU) + PML(PB, T_, PU);
    PML_END
}

/* m_vneb: pml.f:2207-2244 */
static void orc_m_vneb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rh[ny-j+1] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        v1[c] = PML(PN, T_, PV) + PML(PE, T_, PV) + PML(PB, T_, PV);
    PML_END
}

/* m_wneb: pml.f:2248-2285 */
static void orc_m_wneb(orc_t *h, const int *r)
{
    PML_BEGIN
        d = R(1.)/d1[c];
        dc=rf[ny-j+1] + pht*rh[nx-i+1] + pht*rf[k];
        PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1] + pht*rf[k];
        PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rh[nx-i+1] + rf[k];
        PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        w1[c] = PML(PN, T_, PW_) + PML(PE, T_, PW_) + PML(PB, T_, PW_);
    PML_END
}

/* m_xyzn: pml.f:2292-2356 */
static void orc_m_xyzn(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        PML(PN, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PXX)* (R(2.) - dt*rf[ny-j+1]))/(R(2.) + dt*rf[ny-j+1]);
        PML(PN, H_, PXX) = (R(2.)*dth* (xl2m*(u1[c + SX] - u1[c]) + xl*(w1[c] - w1[c - SZ])) + PML(PN, H_, PXX) * (R(2.) - dt * pht * rf[ny-j+1]))/ (R(2.) + dt * pht * rf[ny-j+1]);
        xx[c] = PML(PN, T_, PXX) + PML(PN, H_, PXX);
        PML(PN, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PN, T_, PYY)* (R(2.) - dt*rf[ny-j+1]))/(R(2.) + dt*rf[ny-j+1]);
        PML(PN, H_, PYY) = (R(2.)*dth*xl*((u1[c + SX] - u1[c]) + (w1[c] - w1[c - SZ])) + PML(PN, H_, PYY)* (R(2.) - dt * pht * rf[ny-j+1]))/ (R(2.) + dt * pht * rf[ny-j+1]);
        yy[c] = PML(PN, T_, PYY) + PML(PN, H_, PYY);
        PML(PN, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PZZ)* (R(2.) - dt*rf[ny-j+1]))/(R(2.) + dt*rf[ny-j+1]);
        PML(PN, H_, PZZ) = (R(2.)*dth*(xl2m*(w1[c] - w1[c - SZ]) + xl*(u1[c + SX] - u1[c])) + PML(PN, H_, PZZ)* (R(2.) - dt * pht * rf[ny-j+1]))/ (R(2.) + dt * pht * rf[ny-j+1]);
        zz[c] = PML(PN, T_, PZZ) + PML(PN, H_, PZZ);
    PML_END
}

/* m_xzn: pml.f:2360-2392 */
static void orc_m_xzn(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*rf[ny-j+1])/(R(2.) + dt*rf[ny-j+1]);
        PML(PN, H_, PXZ) = (R(2.)*xm*dth*((u1[c + SZ] - u1[c]) + (w1[c] - w1[c - SX])) + PML(PN, H_, PXZ) * (R(2.) - dt * pht * rf[ny-j+1]))/ (R(2.) + dt * pht * rf[ny-j+1]);
        xz[c] = PML(PN, T_, PXZ) + PML(PN, H_, PXZ);
    PML_END
}

/* m_yzn: pml.f:2396-2429 */
static void orc_m_yzn(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
        PML(PN, H_, PYZ) = (R(2.) * dth * xm*(v1[c + SZ] - v1[c]) + PML(PN, H_, PYZ) * (R(2.) - dt * pht * rh[ny-j+1]))/ (R(2.) + dt * pht * rh[ny-j+1]);
        yz[c] = PML(PN, T_, PYZ) + PML(PN, H_, PYZ);
    PML_END
}

/* m_xyn: pml.f:2433-2466 */
static void orc_m_xyn(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PN, T_, PXY) = (R(2.)*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
        PML(PN, H_, PXY) = (R(2.)*xm*dth*(v1[c] - v1[c - SX]) + PML(PN, H_, PXY) * (R(2.) - dt * pht * rh[ny-j+1]))/ (R(2.) + dt * pht * rh[ny-j+1]);
        xy[c] = PML(PN, T_, PXY) + PML(PN, H_, PXY);
    PML_END
}

/* m_xyzs: pml.f:2470-2530 */
static void orc_m_xyzs(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        PML(PS, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PXX)* (R(2.) - dt*rh[j]))/(R(2.) + dt*rh[j]);
        PML(PS, H_, PXX) = (R(2.)*dth*(xl2m*(u1[c + SX] - u1[c]) + xl*(w1[c] - w1[c - SZ])) + PML(PS, H_, PXX)* (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
        xx[c] = PML(PS, T_, PXX) + PML(PS, H_, PXX);
        PML(PS, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PS, T_, PYY)* (R(2.) - dt*rh[j]))/(R(2.) + dt*rh[j]);
        PML(PS, H_, PYY) = (R(2.)*dth*xl*((u1[c + SX] - u1[c]) + (w1[c] - w1[c - SZ])) + PML(PS, H_, PYY)* (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
        yy[c] = PML(PS, T_, PYY) + PML(PS, H_, PYY);
        PML(PS, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PZZ)* (R(2.) - dt*rh[j]))/(R(2.) + dt*rh[j]);
        PML(PS, H_, PZZ) = (R(2.)*dth*(xl2m*(w1[c] - w1[c - SZ]) + xl*(u1[c + SX] - u1[c]))+ PML(PS, H_, PZZ)* (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
        zz[c] = PML(PS, T_, PZZ) + PML(PS, H_, PZZ);
    PML_END
}

/* m_xzs: pml.f:2534-2564 */
static void orc_m_xzs(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*rh[j])/(R(2.) + dt*rh[j]);
        PML(PS, H_, PXZ) = (R(2.)*xm*dth*((u1[c + SZ] - u1[c]) + (w1[c] - w1[c - SX])) + PML(PS, H_, PXZ)* (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
        xz[c] = PML(PS, T_, PXZ) + PML(PS, H_, PXZ);
    PML_END
}

/* m_yzs: pml.f:2568-2599 */
static void orc_m_yzs(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*rf[j]))/(R(2.) + dt*rf[j]);
        PML(PS, H_, PYZ) = (R(2.)*xm*dth*(v1[c + SZ] - v1[c]) + PML(PS, H_, PYZ)* (R(2.) - dt*pht*rf[j]))/(R(2.) + dt*pht*rf[j]);
        yz[c] = PML(PS, T_, PYZ) + PML(PS, H_, PYZ);
    PML_END
}

/* m_xys: pml.f:2603-2634 */
static void orc_m_xys(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*rf[j]))/(R(2.) + dt*rf[j]);
        PML(PS, H_, PXY) = (R(2.)* xm*dth*(v1[c] - v1[c - SX]) + PML(PS, H_, PXY) * (R(2.) - dt*pht*rf[j]))/(R(2.) + dt*pht*rf[j]);
        xy[c] = PML(PS, T_, PXY) + PML(PS, H_, PXY);
    PML_END
}

/* m_xyzw: pml.f:2638-2698 */
static void orc_m_xyzw(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        PML(PW, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PW, T_, PXX)* (R(2.) - dt*rf[i]))/(R(2.) + dt*rf[i]);
        PML(PW, H_, PXX) = (R(2.)*dth*xl*((v1[c] - v1[c - SY]) + (w1[c] - w1[c - SZ])) + PML(PW, H_, PXX) * (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
        xx[c] = PML(PW, T_, PXX) + PML(PW, H_, PXX);
        PML(PW, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PYY)* (R(2.) - dt*rf[i]))/(R(2.) + dt*rf[i]);
        PML(PW, H_, PYY) = (R(2.)*dth*(xl2m*(v1[c] - v1[c - SY]) + xl*(w1[c] - w1[c - SZ])) + PML(PW, H_, PYY) * (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
        yy[c] = PML(PW, T_, PYY) + PML(PW, H_, PYY);
        PML(PW, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PZZ)* (R(2.) - dt*rf[i]))/(R(2.) + dt*rf[i]);
        PML(PW, H_, PZZ) = (R(2.)*dth*(xl*(v1[c] - v1[c - SY]) + xl2m*(w1[c] - w1[c - SZ])) + PML(PW, H_, PZZ) * (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
        zz[c] = PML(PW, T_, PZZ) + PML(PW, H_, PZZ);
    PML_END
}

/* m_xzw: pml.f:2702-2733 */
static void orc_m_xzw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*rh[i]))/(R(2.) + dt*rh[i]);
        PML(PW, H_, PXZ) = (R(2.)*xm*dth*(u1[c + SZ] - u1[c]) + PML(PW, H_, PXZ) * (R(2.) - dt*pht*rh[i]))/(R(2.) + dt*pht*rh[i]);
        xz[c] = PML(PW, T_, PXZ) + PML(PW, H_, PXZ);
    PML_END
}

/* m_yzw: pml.f:2737-2767 */
static void orc_m_yzw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*rf[i])/(R(2.) + dt*rf[i]);
        PML(PW, H_, PYZ) = (R(2.)*xm*dth*((v1[c + SZ] - v1[c]) + (w1[c + SY] - w1[c]))+ PML(PW, H_, PYZ) * (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
        yz[c] = PML(PW, T_, PYZ) + PML(PW, H_, PYZ);
    PML_END
}

/* m_xyw: pml.f:2771-2802 */
static void orc_m_xyw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*rh[i]))/(R(2.) + dt*rh[i]);
        PML(PW, H_, PXY) = (R(2.)*xm*dth*(u1[c + SY] - u1[c]) + PML(PW, H_, PXY)* (R(2.) - dt*pht*rh[i]))/(R(2.) + dt*pht*rh[i]);
        xy[c] = PML(PW, T_, PXY) + PML(PW, H_, PXY);
    PML_END
}

/* m_xyze: pml.f:2806-2869 */
static void orc_m_xyze(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        PML(PE, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PE, T_, PXX)* (R(2.) - dt*rh[nx-i+1]))/(R(2.) + dt*rh[nx-i+1]);
        PML(PE, H_, PXX) = (R(2.)*dth*xl*((v1[c] - v1[c - SY]) + (w1[c] - w1[c - SZ])) + PML(PE, H_, PXX)* (R(2.) - dt*pht*rh[nx-i+1]))/ (R(2.) + dt*pht*rh[nx-i+1]);
        xx[c] = PML(PE, T_, PXX) + PML(PE, H_, PXX);
        PML(PE, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PYY)* (R(2.) - dt*rh[nx-i+1]))/(R(2.) + dt*rh[nx-i+1]);
        PML(PE, H_, PYY) = (R(2.)*dth*(xl2m*(v1[c] - v1[c - SY]) + xl*(w1[c] - w1[c - SZ]))+ PML(PE, H_, PYY)* (R(2.) - dt*pht*rh[nx-i+1]))/ (R(2.) + dt*pht*rh[nx-i+1]);
        yy[c] = PML(PE, T_, PYY) + PML(PE, H_, PYY);
        PML(PE, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PZZ)* (R(2.) - dt*rh[nx-i+1]))/(R(2.) + dt*rh[nx-i+1]);
        PML(PE, H_, PZZ) = (R(2.)*dth*(xl*(v1[c] - v1[c - SY]) + xl2m*(w1[c] - w1[c - SZ])) + PML(PE, H_, PZZ)* (R(2.) - dt*pht*rh[nx-i+1]))/ (R(2.) + dt*pht*rh[nx-i+1]);
        zz[c] = PML(PE, T_, PZZ) + PML(PE, H_, PZZ);
    PML_END
}

/* m_xze: pml.f:2873-2905 */
static void orc_m_xze(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*rf[nx-i+1]))/(R(2.) + dt*rf[nx-i+1]);
        PML(PE, H_, PXZ) = (R(2.)*xm*dth*(u1[c + SZ] - u1[c]) + PML(PE, H_, PXZ)* (R(2.) - dt*pht*rf[nx-i+1]))/ (R(2.) + dt*pht*rf[nx-i+1]);
        xz[c] = PML(PE, T_, PXZ) + PML(PE, H_, PXZ);
    PML_END
}

/* m_yze: pml.f:2909-2940 */
static void orc_m_yze(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*rh[nx-i+1])/(R(2.) + dt*rh[nx-i+1]);
        PML(PE, H_, PYZ) =(R(2.)*xm*dth*((v1[c + SZ] - v1[c]) + (w1[c + SY] - w1[c]))+ PML(PE, H_, PYZ)* (R(2.) - dt*pht*rh[nx-i+1]))/ (R(2.) + dt*pht*rh[nx-i+1]);
        yz[c] = PML(PE, T_, PYZ) + PML(PE, H_, PYZ);
    PML_END
}

/* m_xye: pml.f:2944-2976 */
static void orc_m_xye(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*rf[nx-i+1]))/(R(2.) + dt*rf[nx-i+1]);
        PML(PE, H_, PXY) = (R(2.)*xm*dth*(u1[c + SY] - u1[c]) + PML(PE, H_, PXY)* (R(2.) - dt*pht*rf[nx-i+1]))/ (R(2.) + dt*pht*rf[nx-i+1]);
        xy[c] = PML(PE, T_, PXY) + PML(PE, H_, PXY);
    PML_END
}

/* m_xyzb: pml.f:2980-3040 */
static void orc_m_xyzb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*rh[k]))/(R(2.) + dt*rh[k]);
        PML(PB, H_, PXX) = (R(2.)* dth*(xl2m*(u1[c + SX] - u1[c]) + xl*(v1[c] - v1[c - SY])) + PML(PB, H_, PXX)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
        xx[c] = PML(PB, T_, PXX) + PML(PB, H_, PXX);
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*rh[k]))/(R(2.) + dt*rh[k]);
        PML(PB, H_, PYY) = (R(2.)* dth*(xl*(u1[c + SX] - u1[c]) + xl2m*(v1[c] - v1[c - SY])) + PML(PB, H_, PYY)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
        yy[c] = PML(PB, T_, PYY) + PML(PB, H_, PYY);
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*rh[k]))/(R(2.) + dt*rh[k]);
        PML(PB, H_, PZZ) = (R(2.)*dth*(xl*(u1[c + SX] - u1[c]) + xl*(v1[c] - v1[c - SY])) + PML(PB, H_, PZZ)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
        zz[c] = PML(PB, T_, PZZ) + PML(PB, H_, PZZ);
    PML_END
}

/* m_xzb: pml.f:3044-3075 */
static void orc_m_xzb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
        PML(PB, H_, PXZ) = (R(2.)*xm*dth*(w1[c] - w1[c - SX]) + PML(PB, H_, PXZ)* (R(2.) - dt*pht*rf[k]))/(R(2.) + dt*pht*rf[k]);
        xz[c] = PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
    PML_END
}

/* m_yzb: pml.f:3079-3110 */
static void orc_m_yzb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
        PML(PB, H_, PYZ) = (R(2.)* xm*dth*(w1[c + SY] - w1[c])+ PML(PB, H_, PYZ)* (R(2.) - dt*pht*rf[k]))/(R(2.) + dt*pht*rf[k]);
        yz[c] = PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
    PML_END
}

/* m_xyb: pml.f:3114-3144 */
static void orc_m_xyb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*rh[k])/(R(2.) + dt*rh[k]);
        PML(PB, H_, PXY) = (R(2.)* xm*dth*((u1[c + SY] - u1[c]) + (v1[c] - v1[c - SX])) + PML(PB, H_, PXY)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
        xy[c] = PML(PB, T_, PXY) + PML(PB, H_, PXY);
    PML_END
}

/* m_xyzsw: pml.f:3151-3231 */
static void orc_m_xyzsw(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rh[j] + pht*rf[i];
        PML(PS, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i];
        PML(PW, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PW, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[i]);
        PML(PS, H_, PXX) = (R(2.)*dth*xl*(w1[c] - w1[c - SZ]) + PML(PS, H_, PXX) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PS, T_, PXX) + PML(PW, T_, PXX) + PML(PS, H_, PXX);
        dc=rh[j] + pht*rf[i];
        PML(PS, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PS, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i];
        PML(PW, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[i]);
        PML(PS, H_, PYY) = (R(2.)*dth*xl*(w1[c] - w1[c - SZ]) + PML(PS, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PS, T_, PYY) + PML(PW, T_, PYY) + PML(PS, H_, PYY);
        dc=rh[j] + pht*rf[i];
        PML(PS, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i];
        PML(PW, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[i]);
        PML(PS, H_, PZZ) = (R(2.)* dth*xl2m*(w1[c] - w1[c - SZ])+ PML(PS, H_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PS, T_, PZZ) + PML(PW, T_, PZZ) + PML(PS, H_, PZZ);
    PML_END
}

/* m_xzsw: pml.f:3235-3272 */
static void orc_m_xzsw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[j] + pht*rh[i];
        PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[i];
        PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[i]);
        PML(PS, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PS, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PS, T_, PXZ) + PML(PW, T_, PXZ) + PML(PS, H_, PXZ);
    PML_END
}

/* m_yzsw: pml.f:3276-3313 */
static void orc_m_yzsw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rf[i];
        PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rf[i];
        PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rf[i]);
        PML(PS, H_, PYZ) = (R(2.)*dth*xm*(v1[c + SZ] - v1[c]) + PML(PS, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PS, T_, PYZ) + PML(PW, T_, PYZ) + PML(PS, H_, PYZ);
    PML_END
}

/* m_xysw: pml.f:3317-3355 */
static void orc_m_xysw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rh[i];
        PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[i];
        PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rh[i]);
        PML(PS, H_, PXY) = PML(PS, H_, PXY) * (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PS, T_, PXY) + PML(PW, T_, PXY) + PML(PS, H_, PXY);
    PML_END
}

/* m_xyzse: pml.f:3359-3439 */
static void orc_m_xyzse(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rh[j] + pht*rh[nx-i+1];
        PML(PS, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1];
        PML(PE, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PE, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[nx-i+1]);
        PML(PS, H_, PXX) = (R(2.)*dth*xl*(w1[c] - w1[c - SZ])+ PML(PS, H_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PS, T_, PXX) + PML(PE, T_, PXX) + PML(PS, H_, PXX);
        dc=rh[j] + pht*rh[nx-i+1];
        PML(PS, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PS, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1];
        PML(PE, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[nx-i+1]);
        PML(PS, H_, PYY) = (R(2.)*dth*xl*(w1[c] - w1[c - SZ]) + PML(PS, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PS, T_, PYY) + PML(PE, T_, PYY) + PML(PS, H_, PYY);
        dc=rh[j] + pht*rh[nx-i+1];
        PML(PS, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1];
        PML(PE, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[nx-i+1]);
        PML(PS, H_, PZZ) = (R(2.)*dth*xl2m*(w1[c] - w1[c - SZ]) + PML(PS, H_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PS, T_, PZZ) + PML(PE, T_, PZZ) + PML(PS, H_, PZZ);
    PML_END
}

/* m_xzse: pml.f:3443-3480 */
static void orc_m_xzse(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[j] + pht*rf[nx-i+1];
        PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[nx-i+1];
        PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[nx-i+1]);
        PML(PS, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PS, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PS, T_, PXZ) + PML(PE, T_, PXZ) + PML(PS, H_, PXZ);
    PML_END
}

/* m_yzse: pml.f:3484-3521 */
static void orc_m_yzse(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rh[nx-i+1];
        PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[nx-i+1];
        PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rh[nx-i+1]);
        PML(PS, H_, PYZ) = (R(2.)* dth*xm*(v1[c + SZ] - v1[c])+ PML(PS, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PS, T_, PYZ) + PML(PE, T_, PYZ) + PML(PS, H_, PYZ);
    PML_END
}

/* m_xyse: pml.f:3525-3563 */
static void orc_m_xyse(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rf[nx-i+1];
        PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rf[nx-i+1];
        PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rf[nx-i+1]);
        PML(PS, H_, PXY) = R(2.)*PML(PS, H_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PS, T_, PXY) + PML(PE, T_, PXY) + PML(PS, H_, PXY);
    PML_END
}

/* m_xyznw: pml.f:3567-3648 */
static void orc_m_xyznw(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rf[ny-j+1] + rf[i] * pht;
        PML(PN, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht * rf[ny-j+1] + rf[i];
        PML(PW, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PW, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1]+rf[i]);
        PML(PN, H_, PXX) = (R(2.)* dth*xl*(w1[c] - w1[c - SZ]) + PML(PN, H_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PN, T_, PXX) + PML(PW, T_, PXX) + PML(PN, H_, PXX);
        dc=rf[ny-j+1] + pht*rf[i];
        PML(PN, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PN, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[i];
        PML(PW, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1]+rf[i]);
        PML(PN, H_, PYY) =(R(2.)* dth*xl*(w1[c] - w1[c - SZ]) + PML(PN, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PN, T_, PYY) + PML(PW, T_, PYY) + PML(PN, H_, PYY);
        dc=rf[ny-j+1] + pht*rf[i];
        PML(PN, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht * rf[ny-j+1] + rf[i];
        PML(PW, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht * (rf[ny-j+1] + rf[i]);
        PML(PN, H_, PZZ) = (R(2.)*dth*xl2m*(w1[c] - w1[c - SZ]) + PML(PN, H_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PN, T_, PZZ) + PML(PW, T_, PZZ) + PML(PN, H_, PZZ);
    PML_END
}

/* m_xznw: pml.f:3652-3689 */
static void orc_m_xznw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[ny-j+1] + pht*rh[i];
        PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[i];
        PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[i]);
        PML(PN, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PN, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PN, T_, PXZ) + PML(PW, T_, PXZ) + PML(PN, H_, PXZ);
    PML_END
}

/* m_yznw: pml.f:3693-3730 */
static void orc_m_yznw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht * rf[i];
        PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rf[i];
        PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rh[ny-j+1] + rf[i]);
        PML(PN, H_, PYZ) = (R(2.)*dth*xm*(v1[c + SZ] - v1[c])+ PML(PN, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PN, T_, PYZ) + PML(PW, T_, PYZ) + PML(PN, H_, PYZ);
    PML_END
}

/* m_xynw: pml.f:3734-3772 */
static void orc_m_xynw(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rh[i];
        PML(PN, T_, PXY) = (R(2.)*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rh[i];
        PML(PW, T_, PXY) = (R(2.)*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[ny-j+1] + rh[i]);
        PML(PN, H_, PXY) = PML(PN, H_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PN, T_, PXY) + PML(PW, T_, PXY) + PML(PN, H_, PXY);
    PML_END
}

/* m_xyzne: pml.f:3776-3856 */
static void orc_m_xyzne(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rf[ny-j+1] + pht * rh[nx-i+1];
        PML(PN, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1];
        PML(PE, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PE, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[nx-i+1]);
        PML(PN, H_, PXX) = (R(2.)*dth*xl*(w1[c] - w1[c - SZ])+ PML(PN, H_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PN, T_, PXX) + PML(PE, T_, PXX) + PML(PN, H_, PXX);
        dc=rf[ny-j+1] + pht * rh[nx-i+1];
        PML(PN, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PN, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1];
        PML(PE, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[nx-i+1]);
        PML(PN, H_, PYY) = (R(2.)*dth*xl*(w1[c] - w1[c - SZ])+ PML(PN, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PN, T_, PYY) + PML(PE, T_, PYY) +PML(PN, H_, PYY);
        dc=rf[ny-j+1] + pht * rh[nx-i+1];
        PML(PN, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1];
        PML(PE, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[nx-i+1]);
        PML(PN, H_, PZZ) = (R(2.)*dth*xl2m*(w1[c] - w1[c - SZ])+ PML(PN, H_, PZZ) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PN, T_, PZZ) + PML(PE, T_, PZZ) + PML(PN, H_, PZZ);
    PML_END
}

/* m_xzne: pml.f:3860-3897 */
static void orc_m_xzne(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[ny-j+1] + pht * rf[nx-i+1];
        PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[nx-i+1];
        PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rf[nx-i+1]);
        PML(PN, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PN, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PN, T_, PXZ) + PML(PE, T_, PXZ) + PML(PN, H_, PXZ);
    PML_END
}

/* m_yzne: pml.f:3901-3938 */
static void orc_m_yzne(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rh[nx-i+1];
        PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
        dc=pht*rh[ny-j+1] + rh[nx-i+1];
        PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rh[ny-j+1] + rh[nx-i+1]);
        PML(PN, H_, PYZ) = (R(2.)* dth*xm*(v1[c + SZ] - v1[c])+ PML(PN, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PN, T_, PYZ) + PML(PE, T_, PYZ) + PML(PN, H_, PYZ);
    PML_END
}

/* m_xyne: pml.f:3942-3979 */
static void orc_m_xyne(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rf[nx-i+1];
        PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rf[nx-i+1];
        PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        PML(PN, H_, PXY) = R(2.)*PML(PN, H_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PN, T_, PXY) + PML(PE, T_, PXY) + PML(PN, H_, PXY);
    PML_END
}

/* m_xyzsb: pml.f:3986-4066 */
static void orc_m_xyzsb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rh[j] + pht*rh[k];
        PML(PS, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[k]);
        PML(PB, H_, PXX) = (R(2.)* dth*xl2m*(u1[c + SX] - u1[c]) + PML(PB, H_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PS, T_, PXX) + PML(PB, T_, PXX) + PML(PB, H_, PXX);
        dc=rh[j] + pht*rh[k];
        PML(PS, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PS, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[k]);
        PML(PB, H_, PYY) = (R(2.)* dth*xl*(u1[c + SX] - u1[c])+ PML(PB, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PS, T_, PYY) + PML(PB, T_, PYY) + PML(PB, H_, PYY);
        dc=rh[j] + pht*rh[k];
        PML(PS, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rh[k]);
        PML(PB, H_, PZZ) = (R(2.)*dth*xl*(u1[c + SX] - u1[c]) + PML(PB, H_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PS, T_, PZZ) + PML(PB, T_, PZZ) + PML(PB, H_, PZZ);
    PML_END
}

/* m_xzsb: pml.f:4070-4107 */
static void orc_m_xzsb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[j] + pht*rf[k];
        PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[j] + rf[k]);
        PML(PB, H_, PXZ) = (R(2.)* dth*xm*(w1[c] - w1[c - SX])+ PML(PB, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PS, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
    PML_END
}

/* m_yzsb: pml.f:4111-4149 */
static void orc_m_yzsb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rf[k];
        PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rf[k]);
        PML(PB, H_, PYZ) = PML(PB, H_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        yz[c] = PML(PS, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
    PML_END
}

/* m_xysb: pml.f:4153-4190 */
static void orc_m_xysb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rh[k];
        PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rf[j] + rh[k]);
        PML(PB, H_, PXY) = (R(2.)*dth*xm*(v1[c] - v1[c - SX])+ PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xy[c] = PML(PS, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
    PML_END
}

/* m_xyznb: pml.f:4194-4274 */
static void orc_m_xyznb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rf[ny-j+1] + pht*rh[k];
        PML(PN, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[k]);
        PML(PB, H_, PXX) = (R(2.)*dth*xl2m*(u1[c + SX] - u1[c]) + PML(PB, H_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PN, T_, PXX) + PML(PB, T_, PXX) + PML(PB, H_, PXX);
        dc=rf[ny-j+1] + pht*rh[k];
        PML(PN, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PN, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[k]);
        PML(PB, H_, PYY) = (R(2.)*dth*xl*(u1[c + SX] - u1[c]) + PML(PB, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PN, T_, PYY) + PML(PB, T_, PYY) + PML(PB, H_, PYY);
        dc=rf[ny-j+1] + pht*rh[k];
        PML(PN, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rh[k]);
        PML(PB, H_, PZZ) = (R(2.)* dth*xl*(u1[c + SX] - u1[c]) + PML(PB, H_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PN, T_, PZZ) + PML(PB, T_, PZZ) + PML(PB, H_, PZZ);
    PML_END
}

/* m_xznb: pml.f:4278-4315 */
static void orc_m_xznb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[ny-j+1] + pht*rf[k];
        PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[ny-j+1] + rf[k]);
        PML(PB, H_, PXZ) = (R(2.)*dth*xm*(w1[c] - w1[c - SX]) + PML(PB, H_, PXZ) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PN, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
    PML_END
}

/* m_yznb: pml.f:4319-4357 */
static void orc_m_yznb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rf[k];
        PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[ny-j+1] + rf[k]);
        PML(PB, H_, PYZ) = PML(PB, H_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        yz[c] = PML(PN, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
    PML_END
}

/* m_xynb: pml.f:4361-4398 */
static void orc_m_xynb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rh[k];
        PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rh[ny-j+1] + rh[k]);
        PML(PB, H_, PXY) = (R(2.)* dth*xm*(v1[c] - v1[c - SX]) + PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xy[c] = PML(PN, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
    PML_END
}

/* m_xyzwb: pml.f:4402-4482 */
static void orc_m_xyzwb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rf[i] + pht*rh[k];
        PML(PW, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PW, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[i] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[i] + rh[k]);
        PML(PB, H_, PXX) = (R(2.)*dth*xl*(v1[c] - v1[c - SY]) + PML(PB, H_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PW, T_, PXX) + PML(PB, T_, PXX) + PML(PB, H_, PXX);
        dc=rf[i] + pht*rh[k];
        PML(PW, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[i] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[i] + rh[k]);
        PML(PB, H_, PYY) = (R(2.)*dth*xl2m*(v1[c] - v1[c - SY])+ PML(PB, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PW, T_, PYY) + PML(PB, T_, PYY) + PML(PB, H_, PYY);
        dc=rf[i] + pht*rh[k];
        PML(PW, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[i] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[i] + rh[k]);
        PML(PB, H_, PZZ) = (R(2.)*dth*xl*(v1[c] - v1[c - SY])+ PML(PB, H_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PW, T_, PZZ) + PML(PB, T_, PZZ) + PML(PB, H_, PZZ);
    PML_END
}

/* m_xzwb: pml.f:4486-4524 */
static void orc_m_xzwb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[i] + pht*rf[k];
        PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[i] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[i] + rf[k]);
        PML(PB, H_, PXZ) = PML(PB, H_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xz[c] = PML(PW, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
    PML_END
}

/* m_yzwb: pml.f:4528-4565 */
static void orc_m_yzwb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[i] + pht*rf[k];
        PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[i] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[i] + rf[k]);
        PML(PB, H_, PYZ) = (R(2.)*dth*xm*(w1[c + SY] - w1[c])+ PML(PB, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PW, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
    PML_END
}

/* m_xywb: pml.f:4569-4606 */
static void orc_m_xywb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[i] + pht*rh[k];
        PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[i] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rh[i] + rh[k]);
        PML(PB, H_, PXY) = (R(2.)*dth*xm*(u1[c + SY] - u1[c])+ PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xy[c] = PML(PW, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
    PML_END
}

/* m_xyzeb: pml.f:4610-4690 */
static void orc_m_xyzeb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PE, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[nx-i+1] + rh[k]);
        PML(PB, H_, PXX) = (R(2.)*dth*xl*(v1[c] - v1[c - SY])+ PML(PB, H_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PE, T_, PXX) + PML(PB, T_, PXX) + PML(PB, H_, PXX);
        dc=rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[nx-i+1] + rh[k]);
        PML(PB, H_, PYY) = (R(2.)*dth*xl2m*(v1[c] - v1[c - SY])+ PML(PB, H_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PE, T_, PYY) + PML(PB, T_, PYY) + PML(PB, H_, PYY);
        dc=rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[nx-i+1] + rh[k]);
        PML(PB, H_, PZZ) = (R(2.)*dth*xl*(v1[c] - v1[c - SY])+ PML(PB, H_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PE, T_, PZZ) + PML(PB, T_, PZZ) + PML(PB, H_, PZZ);
    PML_END
}

/* m_xzeb: pml.f:4694-4732 */
static void orc_m_xzeb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[nx-i+1] + pht*rf[k];
        PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[nx-i+1] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rf[nx-i+1] + rf[k]);
        PML(PB, H_, PXZ) = PML(PB, H_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xz[c] = PML(PE, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
    PML_END
}

/* m_yzeb: pml.f:4736-4773 */
static void orc_m_yzeb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[nx-i+1] + pht*rf[k];
        PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[nx-i+1] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*(rh[nx-i+1] + rf[k]);
        PML(PB, H_, PYZ) = (R(2.)* dth*xm*(w1[c + SY] - w1[c]) + PML(PB, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PE, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
    PML_END
}

/* m_xyeb: pml.f:4777-4814 */
static void orc_m_xyeb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[nx-i+1] + pht*rh[k];
        PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[nx-i+1] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*(rf[nx-i+1] + rh[k]);
        PML(PB, H_, PXY) = (R(2.)*dth*xm*(u1[c + SY] - u1[c]) + PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xy[c] = PML(PE, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
    PML_END
}

/* m_xyzswb: pml.f:4821-4904 */
static void orc_m_xyzswb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rh[j] + pht*rf[i] + pht*rh[k];
        PML(PS, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i] + pht*rh[k];
        PML(PW, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PW, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rf[i] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PS, T_, PXX) + PML(PW, T_, PXX) + PML(PB, T_, PXX);
        dc=rh[j] + pht*rf[i] + pht*rh[k];
        PML(PS, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PS, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i] + pht*rh[k];
        PML(PW, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rf[i] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PS, T_, PYY) + PML(PW, T_, PYY) + PML(PB, T_, PYY);
        dc=rh[j] + pht*rf[i] + pht*rh[k];
        PML(PS, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[i] + pht*rh[k];
        PML(PW, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rf[i] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PS, T_, PZZ) + PML(PW, T_, PZZ) + PML(PB, T_, PZZ);
    PML_END
}

/* m_xzswb: pml.f:4908-4946 */
static void orc_m_xzswb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[j] + pht*rh[i] + pht*rf[k];
        PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[i] + pht*rf[k];
        PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rh[i] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PS, T_, PXZ) + PML(PW, T_, PXZ) + PML(PB, T_, PXZ);
    PML_END
}

/* m_yzswb: pml.f:4950-4988 */
static void orc_m_yzswb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rf[i] + pht*rf[k];
        PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rf[i] + pht*rf[k];
        PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[j] + pht*rf[i] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PS, T_, PYZ) + PML(PW, T_, PYZ) + PML(PB, T_, PYZ);
    PML_END
}

/* m_xyswb: pml.f:4992-5030 */
static void orc_m_xyswb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rh[i] + pht*rh[k];
        PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[i] + pht*rh[k];
        PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + pht*rh[i] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PS, T_, PXY) + PML(PW, T_, PXY) + PML(PB, T_, PXY);
    PML_END
}

/* m_xyzseb: pml.f:5034-5117 */
static void orc_m_xyzseb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rh[j] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PS, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PE, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PS, T_, PXX) + PML(PE, T_, PXX) + PML(PB, T_, PXX);
        dc=rh[j] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PS, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PS, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PS, T_, PYY) + PML(PE, T_, PYY) + PML(PB, T_, PYY);
        dc=rh[j] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PS, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PS, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PS, T_, PZZ) + PML(PE, T_, PZZ) + PML(PB, T_, PZZ);
    PML_END
}

/* m_xzseb: pml.f:5121-5159 */
static void orc_m_xzseb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[j] + pht*rf[nx-i+1] + pht*rf[k];
        PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[j] + rf[nx-i+1] + pht*rf[k];
        PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[j] + pht*rf[nx-i+1] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PS, T_, PXZ) + PML(PE, T_, PXZ) + PML(PB, T_, PXZ);
    PML_END
}

/* m_yzseb: pml.f:5163-5201 */
static void orc_m_yzseb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rh[nx-i+1] + pht*rf[k];
        PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rh[nx-i+1] + pht*rf[k];
        PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[j] + pht*rh[nx-i+1] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PS, T_, PYZ) + PML(PE, T_, PYZ) + PML(PB, T_, PYZ);
    PML_END
}

/* m_xyseb: pml.f:5205-5243 */
static void orc_m_xyseb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[j] + pht*rf[nx-i+1] + pht*rh[k];
        PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + rf[nx-i+1] + pht*rh[k];
        PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[j] + pht*rf[nx-i+1] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PS, T_, PXY) + PML(PE, T_, PXY) + PML(PB, T_, PXY);
    PML_END
}

/* m_xyznwb: pml.f:5247-5330 */
static void orc_m_xyznwb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rf[ny-j+1] + pht*rf[i] + pht*rh[k];
        PML(PN, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[i] + pht*rh[k];
        PML(PW, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PW, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rf[i] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PN, T_, PXX) + PML(PW, T_, PXX) + PML(PB, T_, PXX);
        dc=rf[ny-j+1] + pht*rf[i] + pht*rh[k];
        PML(PN, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PN, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[i] + pht*rh[k];
        PML(PW, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rf[i] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PN, T_, PYY) + PML(PW, T_, PYY) + PML(PB, T_, PYY);
        dc=rf[ny-j+1] + pht*rf[i] + pht*rh[k];
        PML(PN, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[i] + pht*rh[k];
        PML(PW, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PW, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rf[i] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PN, T_, PZZ) + PML(PW, T_, PZZ) + PML(PB, T_, PZZ);
    PML_END
}

/* m_xznwb: pml.f:5334-5372 */
static void orc_m_xznwb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[ny-j+1] + pht*rh[i] + pht*rf[k];
        PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[i] + pht*rf[k];
        PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rh[i] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xz[c] = PML(PN, T_, PXZ) + PML(PW, T_, PXZ) + PML(PB, T_, PXZ);
    PML_END
}

/* m_yznwb: pml.f:5376-5414 */
static void orc_m_yznwb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rf[i] + pht*rf[k];
        PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rf[i] + pht*rf[k];
        PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + pht*rf[i] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PN, T_, PYZ) + PML(PW, T_, PYZ) + PML(PB, T_, PYZ);
    PML_END
}

/* m_xynwb: pml.f:5418-5456 */
static void orc_m_xynwb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rh[i] + pht*rh[k];
        PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rh[i] + pht*rh[k];
        PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + pht*rh[i] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PN, T_, PXY) + PML(PW, T_, PXY) + PML(PB, T_, PXY);
    PML_END
}

/* m_xyzneb: pml.f:5460-5543 */
static void orc_m_xyzneb(orc_t *h, const int *r)
{
    PML_BEGIN
        xl = R(1.)/lam[c];
        xl2m = R(2.)/mu[c] + xl;
        dc=rf[ny-j+1] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PN, T_, PXX) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PXX) = (R(2.)*dth*xl2m* (u1[c + SX] - u1[c]) + PML(PE, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PXX) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PXX)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        xx[c] = PML(PN, T_, PXX) + PML(PE, T_, PXX) + PML(PB, T_, PXX);
        dc=rf[ny-j+1] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PN, T_, PYY) = (R(2.)*dth*xl2m* (v1[c] - v1[c - SY]) + PML(PN, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PYY) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PYY) = (R(2.)*dth*xl* (w1[c] - w1[c - SZ]) + PML(PB, T_, PYY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yy[c] = PML(PN, T_, PYY) + PML(PE, T_, PYY) + PML(PB, T_, PYY);
        dc=rf[ny-j+1] + pht*rh[nx-i+1] + pht*rh[k];
        PML(PN, T_, PZZ) = (R(2.)*dth*xl* (v1[c] - v1[c - SY]) + PML(PN, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rh[nx-i+1] + pht*rh[k];
        PML(PE, T_, PZZ) = (R(2.)*dth*xl* (u1[c + SX] - u1[c]) + PML(PE, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rh[nx-i+1] + rh[k];
        PML(PB, T_, PZZ) = (R(2.)*dth*xl2m* (w1[c] - w1[c - SZ]) + PML(PB, T_, PZZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        zz[c] = PML(PN, T_, PZZ) + PML(PE, T_, PZZ) + PML(PB, T_, PZZ);
    PML_END
}

/* m_xzneb: pml.f:5547-5585 */
static void orc_m_xzneb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rf[ny-j+1] + pht*rf[nx-i+1] + pht*rf[k];
        PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + rf[nx-i+1] + pht*rf[k];
        PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rf[ny-j+1] + pht*rf[nx-i+1] + rf[k];
        PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
        xz[c] = PML(PN, T_, PXZ) + PML(PE, T_, PXZ) + PML(PB, T_, PXZ);
    PML_END
}

/* m_yzneb: pml.f:5589-5627 */
static void orc_m_yzneb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rh[nx-i+1] + pht*rf[k];
        PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rh[nx-i+1] + pht*rf[k];
        PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + pht*rh[nx-i+1] + rf[k];
        PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        yz[c] = PML(PN, T_, PYZ) + PML(PE, T_, PYZ) + PML(PB, T_, PYZ);
    PML_END
}

/* m_xyneb: pml.f:5631-5669 */
static void orc_m_xyneb(orc_t *h, const int *r)
{
    PML_BEGIN
        xm = R(1.)/mu[c];
        dc=rh[ny-j+1] + pht*rf[nx-i+1] + pht*rh[k];
        PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + rf[nx-i+1] + pht*rh[k];
        PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
        dc=pht*rh[ny-j+1] + pht*rf[nx-i+1] + rh[k];
        PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
        xy[c] = PML(PN, T_, PXY) + PML(PE, T_, PXY) + PML(PB, T_, PXY);
    PML_END
}

/* inipml (pml.f:4-44): damping series of the PML width nd from the
 * harmonic mean of the lowest and highest S velocity, full-node rf and
 * half-node rh, index 1 at the outer edge */
static void orc_inipml(orc_t *h)
{
    const orc_params *p = &h->p;
    const int ndt = p->nd;
    const real c0 = (real)0., c1 = (real)8. / (real)15., c2 = -((real)3. / (real)100.), c3 = (real)1. / (real)1500.;
    const real f = c0 + (real)ndt * c1 + (real)(ndt * ndt) * c2 + (real)(ndt * ndt * ndt) * c3;
    const real v = (real)1. / ((real)0.5 * ((real)1. / (real)h->vse[0] + (real)1. / (real)h->vse[1]));
    const real coef = (real)p->arbc * f * v / ((real)ndt * (real)p->dh);
    for (int i = 1; i <= ndt; i++) h->rf[ndt + 1 - i] = coef * (real)i * (real)i / (real)(ndt * ndt);
    h->rh[1] = h->rf[1] + (real)0.50 * (h->rf[1] - h->rf[2]);
    for (int i = 2; i <= ndt; i++) h->rh[i] = (real)0.5 * (h->rf[i - 1] + h->rf[i]);
}

/* zone bounds of a single rank (bound.f:837-893 with the ranges of
 * bound.f:14-238): x / y ranges 1 = 1..nd, 5 = n-nd+1..n, 6 = nd+1..n-nd;
 * z ranges 1 = 1..nd, 2 = nd+1..nz */
static void orc_pml_zone(const orc_params *p, int zone, int r[6])
{
    static const char xr[19] = {0, 6, 1, 6, 5, 6, 1, 1, 5, 5, 6, 1, 6, 5, 1, 1, 5, 5, 6};
    static const char yr[19] = {0, 1, 6, 5, 6, 6, 1, 5, 1, 5, 1, 6, 5, 6, 1, 5, 1, 5, 6};
    static const char zr[19] = {0, 2, 2, 2, 2, 1, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 2};
    const int nd = p->nd;
    const int n[2] = {p->nx, p->ny};
    const char rr[2] = {xr[zone], yr[zone]};
    for (int a = 0; a < 2; a++) {
        if (rr[a] == 1) { r[2 * a] = 1; r[2 * a + 1] = nd; }
        else if (rr[a] == 5) { r[2 * a] = n[a] - nd + 1; r[2 * a + 1] = n[a]; }
        else { r[2 * a] = nd + 1; r[2 * a + 1] = n[a] - nd; }
    }
    if (zr[zone] == 1) { r[4] = 1; r[5] = nd; }
    else { r[4] = nd + 1; r[5] = p->nz; }
}

typedef void (*orc_pml_fn)(orc_t *, const int *);

/* pmlvel (pml.f:49-146): planes, vertical edges, horizontal edges, corners */
static void orc_pmlvel(orc_t *h)
{
    static const struct { int zone; orc_pml_fn f[3]; } seq[] = {
        {1, {orc_m_us, orc_m_vs, orc_m_ws}}, {2, {orc_m_uw, orc_m_vw, orc_m_ww}},
        {3, {orc_m_un, orc_m_vn, orc_m_wn}}, {4, {orc_m_ue, orc_m_ve, orc_m_we}},
        {5, {orc_m_ub, orc_m_vb, orc_m_wb}},
        {6, {orc_m_usw, orc_m_vsw, orc_m_wsw}}, {8, {orc_m_use, orc_m_vse, orc_m_wse}},
        {7, {orc_m_unw, orc_m_vnw, orc_m_wnw}}, {9, {orc_m_une, orc_m_vne, orc_m_wne}},
        {10, {orc_m_usb, orc_m_vsb, orc_m_wsb}}, {12, {orc_m_unb, orc_m_vnb, orc_m_wnb}},
        {11, {orc_m_uwb, orc_m_vwb, orc_m_wwb}}, {13, {orc_m_ueb, orc_m_veb, orc_m_web}},
        {14, {orc_m_uswb, orc_m_vswb, orc_m_wswb}}, {15, {orc_m_unwb, orc_m_vnwb, orc_m_wnwb}},
        {16, {orc_m_useb, orc_m_vseb, orc_m_wseb}}, {17, {orc_m_uneb, orc_m_vneb, orc_m_wneb}},
    };
    for (size_t n = 0; n < sizeof seq / sizeof seq[0]; n++) {
        int r[6];
        orc_pml_zone(&h->p, seq[n].zone, r);
        for (int a = 0; a < 3; a++) seq[n].f[a](h, r);
    }
}

/* pmlstr (pml.f:148-263) */
static void orc_pmlstr(orc_t *h)
{
    static const struct { int zone; orc_pml_fn f[4]; } seq[] = {
        {3, {orc_m_xyzn, orc_m_xzn, orc_m_yzn, orc_m_xyn}}, {1, {orc_m_xyzs, orc_m_xzs, orc_m_yzs, orc_m_xys}},
        {2, {orc_m_xyzw, orc_m_xzw, orc_m_yzw, orc_m_xyw}}, {4, {orc_m_xyze, orc_m_xze, orc_m_yze, orc_m_xye}},
        {5, {orc_m_xyzb, orc_m_xzb, orc_m_yzb, orc_m_xyb}},
        {6, {orc_m_xyzsw, orc_m_xzsw, orc_m_yzsw, orc_m_xysw}}, {8, {orc_m_xyzse, orc_m_xzse, orc_m_yzse, orc_m_xyse}},
        {7, {orc_m_xyznw, orc_m_xznw, orc_m_yznw, orc_m_xynw}}, {9, {orc_m_xyzne, orc_m_xzne, orc_m_yzne, orc_m_xyne}},
        {10, {orc_m_xyzsb, orc_m_xzsb, orc_m_yzsb, orc_m_xysb}}, {12, {orc_m_xyznb, orc_m_xznb, orc_m_yznb, orc_m_xynb}},
        {11, {orc_m_xyzwb, orc_m_xzwb, orc_m_yzwb, orc_m_xywb}}, {13, {orc_m_xyzeb, orc_m_xzeb, orc_m_yzeb, orc_m_xyeb}},
        {14, {orc_m_xyzswb, orc_m_xzswb, orc_m_yzswb, orc_m_xyswb}},
        {15, {orc_m_xyznwb, orc_m_xznwb, orc_m_yznwb, orc_m_xynwb}},
        {16, {orc_m_xyzseb, orc_m_xzseb, orc_m_yzseb, orc_m_xyseb}},
        {17, {orc_m_xyzneb, orc_m_xzneb, orc_m_yzneb, orc_m_xyneb}},
    };
    for (size_t n = 0; n < sizeof seq / sizeof seq[0]; n++) {
        int r[6];
        orc_pml_zone(&h->p, seq[n].zone, r);
        for (int a = 0; a < 4; a++) seq[n].f[a](h, r);
    }
}
