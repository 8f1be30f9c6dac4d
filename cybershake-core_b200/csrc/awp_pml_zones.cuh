/*
 * awp_pml_zones.cuh -- per-cell arithmetic of the PML zones (NPC = 1), one
 * device routine per routine of AWP-ODC-SGT/src/pml.f, each restating that
 * routine's statements in their order and grouping (the oracle's FP32 build
 * evaluates the same statements, so the results are bit-identical).
 *
 * Vocabulary: PML(plane, split, field) is the split array of the routine at
 * the cell (planes PS PN PW PE PB, splits T_ H_, fields PU PV PW_ PXX PYY PZZ
 * PXY PXZ PYZ); the wavefield and media arrays are indexed from the cell c
 * with strides SX SY SZ; rf / rh are the full- and half-node damping
 * profiles (index 1 at the outer edge); R() marks an FP32 constant.
 */
#ifndef AWP_PML_ZONES_CUH
#define AWP_PML_ZONES_CUH

/* m_un (pml.f:267-300) */
__device__ __forceinline__ void m_un(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*rf[ny-j+1]))/(R(2.) + dt*rf[ny-j+1]);
    PML(PN, H_, PU) = (R(2.)*dth*d* ((xx[c] - xx[c - SX]) + (xz[c] - xz[c - SZ])) + PML(PN, H_, PU)* (R(2.) - dt * pht * rf[ny-j+1]))/ (R(2.) + dt * pht * rf[ny-j+1]);
    u1[c] = PML(PN, T_, PU) + PML(PN, H_, PU);
}

/* m_vn (pml.f:304-337) */
__device__ __forceinline__ void m_vn(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
    PML(PN, H_, PV) = (R(2.)*dth*d*((xy[c + SX] - xy[c]) + (yz[c] - yz[c - SZ])) + PML(PN, H_, PV) * (R(2.) - dt*pht*rh[ny-j+1]))/ (R(2.) + dt*pht*rh[ny-j+1]);
    v1[c] = PML(PN, T_, PV) + PML(PN, H_, PV);
}

/* m_wn (pml.f:341-374) */
__device__ __forceinline__ void m_wn(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*rf[ny-j+1]))/(R(2.) + dt*rf[ny-j+1]);
    PML(PN, H_, PW_) = (R(2.)*dth*d*((xz[c + SX] - xz[c]) + (zz[c + SZ] - zz[c])) + PML(PN, H_, PW_) * (R(2.) - dt * pht*rf[ny-j+1])) / (R(2.) + dt * pht*rf[ny-j+1]);
    w1[c] = PML(PN, T_, PW_) + PML(PN, H_, PW_);
}

/* m_us (pml.f:378-409) */
__device__ __forceinline__ void m_us(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*rh[j]))/(R(2.) + dt*rh[j]);
    PML(PS, H_, PU) = (R(2.)*d*dth*((xx[c] - xx[c - SX]) + (xz[c] - xz[c - SZ]))+ PML(PS, H_, PU)* (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
    u1[c] = PML(PS, T_, PU) + PML(PS, H_, PU);
}

/* m_vs (pml.f:413-444) */
__device__ __forceinline__ void m_vs(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*rf[j]))/(R(2.) + dt*rf[j]);
    PML(PS, H_, PV) = (R(2.)*d*dth*((xy[c + SX] - xy[c]) + (yz[c] - yz[c - SZ])) + PML(PS, H_, PV)* (R(2.) - dt*pht*rf[j]))/(R(2.) + dt*pht*rf[j]);
    v1[c] = PML(PS, T_, PV) + PML(PS, H_, PV);
}

/* m_ws (pml.f:448-479) */
__device__ __forceinline__ void m_ws(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*rh[j]))/(R(2.) + dt*rh[j]);
    PML(PS, H_, PW_) = (R(2.)*d*dth*((xz[c + SX] - xz[c]) + (zz[c + SZ] - zz[c]))+ PML(PS, H_, PW_) * (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
    w1[c] = PML(PS, T_, PW_) + PML(PS, H_, PW_);
}

/* m_uw (pml.f:483-514) */
__device__ __forceinline__ void m_uw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*rh[i]))/(R(2.) + dt*rh[i]);
    PML(PW, H_, PU) = (R(2.)*d*dth*((xy[c] - xy[c - SY]) + (xz[c] - xz[c - SZ]))+ PML(PW, H_, PU)* (R(2.) - dt*pht*rh[i]))/(R(2.) + dt*pht*rh[i]);
    u1[c] = PML(PW, T_, PU) + PML(PW, H_, PU);
}

/* m_vw (pml.f:518-549) */
__device__ __forceinline__ void m_vw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*rf[i]))/(R(2.) + dt*rf[i]);
    PML(PW, H_, PV) = (R(2.)*d*dth*((yy[c + SY] - yy[c]) + (yz[c] - yz[c - SZ])) + PML(PW, H_, PV) * (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
    v1[c] = PML(PW, T_, PV) + PML(PW, H_, PV);
}

/* m_ww (pml.f:553-584) */
__device__ __forceinline__ void m_ww(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*rf[i]))/(R(2.) + dt*rf[i]);
    PML(PW, H_, PW_) = (R(2.)*d*dth*((yz[c] - yz[c - SY]) + (zz[c + SZ] - zz[c])) + PML(PW, H_, PW_)* (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
    w1[c] = PML(PW, T_, PW_) + PML(PW, H_, PW_);
}

/* m_ue (pml.f:588-619) */
__device__ __forceinline__ void m_ue(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*rf[nx-i+1]))/(R(2.) + dt*rf[nx-i+1]);
    PML(PE, H_, PU) = (R(2.)*d*dth*((xy[c] - xy[c - SY]) + (xz[c] - xz[c - SZ])) + PML(PE, H_, PU)* (R(2.) - dt*pht*rf[nx-i+1]))/(R(2.) + dt*pht*rf[nx-i+1]);
    u1[c] = PML(PE, T_, PU) + PML(PE, H_, PU);
}

/* m_ve (pml.f:623-655) */
__device__ __forceinline__ void m_ve(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*rh[nx-i+1]))/(R(2.) + dt*rh[nx-i+1]);
    PML(PE, H_, PV) = (R(2.)*d*dth*( (yy[c + SY] - yy[c]) + (yz[c] - yz[c - SZ])) + PML(PE, H_, PV) * (R(2.) - dt*pht*rh[nx-i+1]))/(R(2.) + dt*pht*rh[nx-i+1]);
    v1[c] = PML(PE, T_, PV) + PML(PE, H_, PV);
}

/* m_we (pml.f:659-691) */
__device__ __forceinline__ void m_we(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*rh[nx-i+1]))/(R(2.) + dt*rh[nx-i+1]);
    PML(PE, H_, PW_) = (R(2.)*d*dth*( (yz[c] - yz[c - SY]) + (zz[c + SZ] - zz[c])) + PML(PE, H_, PW_) * (R(2.) - dt*pht*rh[nx-i+1]))/(R(2.) + dt*pht*rh[nx-i+1]);
    w1[c] = PML(PE, T_, PW_) + PML(PE, H_, PW_);
}

/* m_ub (pml.f:695-727) */
__device__ __forceinline__ void m_ub(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*rh[k]))/(R(2.) + dt*rh[k]);
    PML(PB, H_, PU) = (R(2.)*d*dth*( (xy[c] - xy[c - SY]) + (xx[c] - xx[c - SX])) + PML(PB, H_, PU)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
    u1[c] = PML(PB, T_, PU) + PML(PB, H_, PU);
}

/* m_vb (pml.f:731-763) */
__device__ __forceinline__ void m_vb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*rh[k]))/(R(2.) + dt*rh[k]);
    PML(PB, H_, PV) = (R(2.)*d*dth*( (xy[c + SX] - xy[c]) + (yy[c + SY] - yy[c])) + PML(PB, H_, PV)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
    v1[c] = PML(PB, T_, PV) + PML(PB, H_, PV);
}

/* m_wb (pml.f:767-799) */
__device__ __forceinline__ void m_wb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
    PML(PB, H_, PW_) = (R(2.)*d*dth*( (yz[c] - yz[c - SY]) + (xz[c + SX] - xz[c])) + PML(PB, H_, PW_)* (R(2.) - dt*pht*rf[k]))/(R(2.) + dt*pht*rf[k]);
    w1[c] = PML(PB, T_, PW_) + PML(PB, H_, PW_);
}

/* m_usw (pml.f:806-843) */
__device__ __forceinline__ void m_usw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rh[i];
    PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rh[i];
    PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rh[i]);
    PML(PS, H_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PS, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PS, T_, PU) + PML(PW, T_, PU) + PML(PS, H_, PU);
}

/* m_vsw (pml.f:847-884) */
__device__ __forceinline__ void m_vsw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[j] + pht*rf[i];
    PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rf[i];
    PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rf[i]);
    PML(PS, H_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PS, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PS, T_, PV) + PML(PW, T_, PV) + PML(PS, H_, PV);
}

/* m_wsw (pml.f:888-925) */
__device__ __forceinline__ void m_wsw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rf[i];
    PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[i];
    PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rf[i]);
    PML(PS, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PS, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PS, T_, PW_) + PML(PW, T_, PW_) + PML(PS, H_, PW_);
}

/* m_use (pml.f:929-966) */
__device__ __forceinline__ void m_use(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rf[nx-i+1];
    PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[nx-i+1];
    PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rf[nx-i+1]);
    PML(PS, H_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PS, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PS, T_, PU) + PML(PE, T_, PU) + PML(PS, H_, PU);
}

/* m_vse (pml.f:970-1007) */
__device__ __forceinline__ void m_vse(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[j] + pht*rh[nx-i+1];
    PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[nx-i+1];
    PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rh[nx-i+1]);
    PML(PS, H_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ])+ PML(PS, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PS, T_, PV) + PML(PE, T_, PV) + PML(PS, H_, PV);
}

/* m_wse (pml.f:1011-1048) */
__device__ __forceinline__ void m_wse(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht * rh[nx-i+1];
    PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rh[nx-i+1];
    PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rh[nx-i+1]);
    PML(PS, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PS, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PS, T_, PW_) + PML(PE, T_, PW_) + PML(PS, H_, PW_);
}

/* m_unw (pml.f:1052-1089) */
__device__ __forceinline__ void m_unw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc = rf[ny-j+1] + pht*rh[i];
    PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc = pht*rf[ny-j+1] + rh[i];
    PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc = pht*(rf[ny-j+1] + rh[i]);
    PML(PN, H_, PU) =(R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PN, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PN, T_, PU) + PML(PW, T_, PU) + PML(PN, H_, PU);
}

/* m_vnw (pml.f:1093-1130) */
__device__ __forceinline__ void m_vnw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc = rh[ny-j+1] + pht * rf[i];
    PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc = pht * rh[ny-j+1] + rf[i];
    PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc = pht * (rh[ny-j+1] + rf[i]);
    PML(PN, H_, PV) = (R(2.)* dth*d*(yz[c] - yz[c - SZ]) + PML(PN, H_, PV) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PN, T_, PV) + PML(PW, T_, PV) + PML(PN, H_, PV);
}

/* m_wnw (pml.f:1134-1171) */
__device__ __forceinline__ void m_wnw(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht * rf[i];
    PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht * rf[ny-j+1] + rf[i];
    PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc = pht * (rf[ny-j+1] + rf[i]);
    PML(PN, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PN, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PN, T_, PW_) + PML(PW, T_, PW_) + PML(PN, H_, PW_);
}

/* m_une (pml.f:1175-1212) */
__device__ __forceinline__ void m_une(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht*rf[nx-i+1];
    PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rf[nx-i+1];
    PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[ny-j+1] + rf[nx-i+1]);
    PML(PN, H_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ])+ PML(PN, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PN, T_, PU) + PML(PE, T_, PU) + PML(PN, H_, PU);
}

/* m_vne (pml.f:1216-1253) */
__device__ __forceinline__ void m_vne(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[ny-j+1] + pht*rh[nx-i+1];
    PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rh[nx-i+1];
    PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[ny-j+1] + rh[nx-i+1]);
    PML(PN, H_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PN, H_, PV) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PN, T_, PV) + PML(PE, T_, PV) + PML(PN, H_, PV);
}

/* m_wne (pml.f:1257-1294) */
__device__ __forceinline__ void m_wne(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht * rh[nx-i+1];
    PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rh[nx-i+1];
    PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[ny-j+1] + rh[nx-i+1]);
    PML(PN, H_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PN, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PN, T_, PW_) + PML(PE, T_, PW_) + PML(PN, H_, PW_);
}

/* m_usb (pml.f:1302-1339) */
__device__ __forceinline__ void m_usb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rh[k];
    PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rh[k]);
    PML(PB, H_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PS, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
}

/* m_vsb (pml.f:1343-1380) */
__device__ __forceinline__ void m_vsb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[j] + pht*rh[k];
    PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rh[k]);
    PML(PB, H_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PS, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
}

/* m_wsb (pml.f:1384-1421) */
__device__ __forceinline__ void m_wsb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rf[k];
    PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rf[k]);
    PML(PB, H_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PB, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PS, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
}

/* m_unb (pml.f:1425-1462) */
__device__ __forceinline__ void m_unb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht*rh[k];
    PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[ny-j+1] + rh[k]);
    PML(PB, H_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PN, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
}

/* m_vnb (pml.f:1466-1503) */
__device__ __forceinline__ void m_vnb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[ny-j+1] + pht*rh[k];
    PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[ny-j+1] + rh[k]);
    PML(PB, H_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PN, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
}

/* m_wnb (pml.f:1507-1544) */
__device__ __forceinline__ void m_wnb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht*rf[k];
    PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[ny-j+1] + rf[k]);
    PML(PB, H_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PB, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PN, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
}

/* m_uwb (pml.f:1548-1585) */
__device__ __forceinline__ void m_uwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[i] + pht*rh[k];
    PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[i] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[i] + rh[k]);
    PML(PB, H_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PW, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
}

/* m_vwb (pml.f:1589-1626) */
__device__ __forceinline__ void m_vwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[i] + pht*rh[k];
    PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[i] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[i] + rh[k]);
    PML(PB, H_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PW, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
}

/* m_wwb (pml.f:1630-1667) */
__device__ __forceinline__ void m_wwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[i] + pht*rf[k];
    PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[i] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[i] + rf[k]);
    PML(PB, H_, PW_) = (R(2.)* dth*d*(yz[c] - yz[c - SY]) + PML(PB, H_, PW_) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PW, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
}

/* m_ueb (pml.f:1671-1708) */
__device__ __forceinline__ void m_ueb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[nx-i+1] + pht*rh[k];
    PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[nx-i+1] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[nx-i+1] + rh[k]);
    PML(PB, H_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY])+ PML(PB, H_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PE, T_, PU) + PML(PB, T_, PU) + PML(PB, H_, PU);
}

/* m_veb (pml.f:1712-1749) */
__device__ __forceinline__ void m_veb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[nx-i+1] + pht*rh[k];
    PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[nx-i+1] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[nx-i+1] + rh[k]);
    PML(PB, H_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PB, H_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PE, T_, PV) + PML(PB, T_, PV) + PML(PB, H_, PV);
}

/* m_web (pml.f:1753-1790) */
__device__ __forceinline__ void m_web(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[nx-i+1] + pht*rf[k];
    PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[nx-i+1] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[nx-i+1] + rf[k]);
    PML(PB, H_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PB, H_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PE, T_, PW_) + PML(PB, T_, PW_) + PML(PB, H_, PW_);
}

/* m_uswb (pml.f:1797-1834) */
__device__ __forceinline__ void m_uswb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rh[i] + pht*rh[k];
    PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rh[i] + pht*rh[k];
    PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + pht*rh[i] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PS, T_, PU) + PML(PW, T_, PU) + PML(PB, T_, PU);
}

/* m_vswb (pml.f:1838-1875) */
__device__ __forceinline__ void m_vswb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[j] + pht*rf[i] + pht*rh[k];
    PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rf[i] + pht*rh[k];
    PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + pht*rf[i] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PS, T_, PV) + PML(PW, T_, PV) + PML(PB, T_, PV);
}

/* m_wswb (pml.f:1879-1916) */
__device__ __forceinline__ void m_wswb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rf[i] + pht*rf[k];
    PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[i] + pht*rf[k];
    PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + pht*rf[i] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PS, T_, PW_) + PML(PW, T_, PW_) + PML(PB, T_, PW_);
}

/* m_unwb (pml.f:1920-1957) */
__device__ __forceinline__ void m_unwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht*rh[i] + pht*rh[k];
    PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rh[i] + pht*rh[k];
    PML(PW, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PW, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + pht*rh[i] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PN, T_, PU) + PML(PW, T_, PU) + PML(PB, T_, PU);
}

/* m_vnwb (pml.f:1961-1998) */
__device__ __forceinline__ void m_vnwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[ny-j+1] + pht*rf[i] + pht*rh[k];
    PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rf[i] + pht*rh[k];
    PML(PW, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PW, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + pht*rf[i] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PN, T_, PV) + PML(PW, T_, PV) + PML(PB, T_, PV);
}

/* m_wnwb (pml.f:2002-2039) */
__device__ __forceinline__ void m_wnwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht*rf[i] + pht*rf[k];
    PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rf[i] + pht*rf[k];
    PML(PW, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PW, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + pht*rf[i] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PN, T_, PW_) + PML(PW, T_, PW_) + PML(PB, T_, PW_);
}

/* m_useb (pml.f:2043-2080) */
__device__ __forceinline__ void m_useb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rf[nx-i+1] + pht*rh[k];
    PML(PS, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PS, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[nx-i+1] + pht*rh[k];
    PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + pht*rf[nx-i+1] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PS, T_, PU) + PML(PE, T_, PU) + PML(PB, T_, PU);
}

/* m_vseb (pml.f:2084-2121) */
__device__ __forceinline__ void m_vseb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[j] + pht*rh[nx-i+1] + pht*rh[k];
    PML(PS, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PS, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[nx-i+1] + pht*rh[k];
    PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + pht*rh[nx-i+1] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PS, T_, PV) + PML(PE, T_, PV) + PML(PB, T_, PV);
}

/* m_wseb (pml.f:2125-2162) */
__device__ __forceinline__ void m_wseb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[j] + pht*rh[nx-i+1] + pht*rf[k];
    PML(PS, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PS, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + rh[nx-i+1] + pht*rf[k];
    PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + pht*rh[nx-i+1] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PS, T_, PW_) + PML(PE, T_, PW_) + PML(PB, T_, PW_);
}

/* m_uneb (pml.f:2166-2203) */
__device__ __forceinline__ void m_uneb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht*rf[nx-i+1] + pht*rh[k];
    PML(PN, T_, PU) = (R(2.)*dth*d*(xy[c] - xy[c - SY]) + PML(PN, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rf[nx-i+1] + pht*rh[k];
    PML(PE, T_, PU) = (R(2.)*dth*d*(xx[c] - xx[c - SX]) + PML(PE, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + pht*rf[nx-i+1] + rh[k];
    PML(PB, T_, PU) = (R(2.)*dth*d*(xz[c] - xz[c - SZ]) + PML(PB, T_, PU)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    u1[c] = PML(PN, T_, PU) + PML(PE, T_, PU) + PML(PB, T_, PU);
}

/* m_vneb (pml.f:2207-2244) */
__device__ __forceinline__ void m_vneb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rh[ny-j+1] + pht*rh[nx-i+1] + pht*rh[k];
    PML(PN, T_, PV) = (R(2.)*dth*d*(yy[c + SY] - yy[c]) + PML(PN, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rh[nx-i+1] + pht*rh[k];
    PML(PE, T_, PV) = (R(2.)*dth*d*(xy[c + SX] - xy[c]) + PML(PE, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + pht*rh[nx-i+1] + rh[k];
    PML(PB, T_, PV) = (R(2.)*dth*d*(yz[c] - yz[c - SZ]) + PML(PB, T_, PV)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    v1[c] = PML(PN, T_, PV) + PML(PE, T_, PV) + PML(PB, T_, PV);
}

/* m_wneb (pml.f:2248-2285) */
__device__ __forceinline__ void m_wneb(const PmlCell &x)
{
    PML_CELL_LOCALS
    d = R(1.)/d1[c];
    dc=rf[ny-j+1] + pht*rh[nx-i+1] + pht*rf[k];
    PML(PN, T_, PW_) = (R(2.)*dth*d*(yz[c] - yz[c - SY]) + PML(PN, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rh[nx-i+1] + pht*rf[k];
    PML(PE, T_, PW_) = (R(2.)*dth*d*(xz[c + SX] - xz[c]) + PML(PE, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + pht*rh[nx-i+1] + rf[k];
    PML(PB, T_, PW_) = (R(2.)*dth*d*(zz[c + SZ] - zz[c]) + PML(PB, T_, PW_)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    w1[c] = PML(PN, T_, PW_) + PML(PE, T_, PW_) + PML(PB, T_, PW_);
}

/* m_xyzn (pml.f:2292-2356) */
__device__ __forceinline__ void m_xyzn(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzn (pml.f:2360-2392) */
__device__ __forceinline__ void m_xzn(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*rf[ny-j+1])/(R(2.) + dt*rf[ny-j+1]);
    PML(PN, H_, PXZ) = (R(2.)*xm*dth*((u1[c + SZ] - u1[c]) + (w1[c] - w1[c - SX])) + PML(PN, H_, PXZ) * (R(2.) - dt * pht * rf[ny-j+1]))/ (R(2.) + dt * pht * rf[ny-j+1]);
    xz[c] = PML(PN, T_, PXZ) + PML(PN, H_, PXZ);
}

/* m_yzn (pml.f:2396-2429) */
__device__ __forceinline__ void m_yzn(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
    PML(PN, H_, PYZ) = (R(2.) * dth * xm*(v1[c + SZ] - v1[c]) + PML(PN, H_, PYZ) * (R(2.) - dt * pht * rh[ny-j+1]))/ (R(2.) + dt * pht * rh[ny-j+1]);
    yz[c] = PML(PN, T_, PYZ) + PML(PN, H_, PYZ);
}

/* m_xyn (pml.f:2433-2466) */
__device__ __forceinline__ void m_xyn(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PN, T_, PXY) = (R(2.)*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
    PML(PN, H_, PXY) = (R(2.)*xm*dth*(v1[c] - v1[c - SX]) + PML(PN, H_, PXY) * (R(2.) - dt * pht * rh[ny-j+1]))/ (R(2.) + dt * pht * rh[ny-j+1]);
    xy[c] = PML(PN, T_, PXY) + PML(PN, H_, PXY);
}

/* m_xyzs (pml.f:2470-2530) */
__device__ __forceinline__ void m_xyzs(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzs (pml.f:2534-2564) */
__device__ __forceinline__ void m_xzs(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*rh[j])/(R(2.) + dt*rh[j]);
    PML(PS, H_, PXZ) = (R(2.)*xm*dth*((u1[c + SZ] - u1[c]) + (w1[c] - w1[c - SX])) + PML(PS, H_, PXZ)* (R(2.) - dt*pht*rh[j]))/(R(2.) + dt*pht*rh[j]);
    xz[c] = PML(PS, T_, PXZ) + PML(PS, H_, PXZ);
}

/* m_yzs (pml.f:2568-2599) */
__device__ __forceinline__ void m_yzs(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*rf[j]))/(R(2.) + dt*rf[j]);
    PML(PS, H_, PYZ) = (R(2.)*xm*dth*(v1[c + SZ] - v1[c]) + PML(PS, H_, PYZ)* (R(2.) - dt*pht*rf[j]))/(R(2.) + dt*pht*rf[j]);
    yz[c] = PML(PS, T_, PYZ) + PML(PS, H_, PYZ);
}

/* m_xys (pml.f:2603-2634) */
__device__ __forceinline__ void m_xys(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*rf[j]))/(R(2.) + dt*rf[j]);
    PML(PS, H_, PXY) = (R(2.)* xm*dth*(v1[c] - v1[c - SX]) + PML(PS, H_, PXY) * (R(2.) - dt*pht*rf[j]))/(R(2.) + dt*pht*rf[j]);
    xy[c] = PML(PS, T_, PXY) + PML(PS, H_, PXY);
}

/* m_xyzw (pml.f:2638-2698) */
__device__ __forceinline__ void m_xyzw(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzw (pml.f:2702-2733) */
__device__ __forceinline__ void m_xzw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*rh[i]))/(R(2.) + dt*rh[i]);
    PML(PW, H_, PXZ) = (R(2.)*xm*dth*(u1[c + SZ] - u1[c]) + PML(PW, H_, PXZ) * (R(2.) - dt*pht*rh[i]))/(R(2.) + dt*pht*rh[i]);
    xz[c] = PML(PW, T_, PXZ) + PML(PW, H_, PXZ);
}

/* m_yzw (pml.f:2737-2767) */
__device__ __forceinline__ void m_yzw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*rf[i])/(R(2.) + dt*rf[i]);
    PML(PW, H_, PYZ) = (R(2.)*xm*dth*((v1[c + SZ] - v1[c]) + (w1[c + SY] - w1[c]))+ PML(PW, H_, PYZ) * (R(2.) - dt*pht*rf[i]))/(R(2.) + dt*pht*rf[i]);
    yz[c] = PML(PW, T_, PYZ) + PML(PW, H_, PYZ);
}

/* m_xyw (pml.f:2771-2802) */
__device__ __forceinline__ void m_xyw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*rh[i]))/(R(2.) + dt*rh[i]);
    PML(PW, H_, PXY) = (R(2.)*xm*dth*(u1[c + SY] - u1[c]) + PML(PW, H_, PXY)* (R(2.) - dt*pht*rh[i]))/(R(2.) + dt*pht*rh[i]);
    xy[c] = PML(PW, T_, PXY) + PML(PW, H_, PXY);
}

/* m_xyze (pml.f:2806-2869) */
__device__ __forceinline__ void m_xyze(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xze (pml.f:2873-2905) */
__device__ __forceinline__ void m_xze(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*rf[nx-i+1]))/(R(2.) + dt*rf[nx-i+1]);
    PML(PE, H_, PXZ) = (R(2.)*xm*dth*(u1[c + SZ] - u1[c]) + PML(PE, H_, PXZ)* (R(2.) - dt*pht*rf[nx-i+1]))/ (R(2.) + dt*pht*rf[nx-i+1]);
    xz[c] = PML(PE, T_, PXZ) + PML(PE, H_, PXZ);
}

/* m_yze (pml.f:2909-2940) */
__device__ __forceinline__ void m_yze(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*rh[nx-i+1])/(R(2.) + dt*rh[nx-i+1]);
    PML(PE, H_, PYZ) =(R(2.)*xm*dth*((v1[c + SZ] - v1[c]) + (w1[c + SY] - w1[c]))+ PML(PE, H_, PYZ)* (R(2.) - dt*pht*rh[nx-i+1]))/ (R(2.) + dt*pht*rh[nx-i+1]);
    yz[c] = PML(PE, T_, PYZ) + PML(PE, H_, PYZ);
}

/* m_xye (pml.f:2944-2976) */
__device__ __forceinline__ void m_xye(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*rf[nx-i+1]))/(R(2.) + dt*rf[nx-i+1]);
    PML(PE, H_, PXY) = (R(2.)*xm*dth*(u1[c + SY] - u1[c]) + PML(PE, H_, PXY)* (R(2.) - dt*pht*rf[nx-i+1]))/ (R(2.) + dt*pht*rf[nx-i+1]);
    xy[c] = PML(PE, T_, PXY) + PML(PE, H_, PXY);
}

/* m_xyzb (pml.f:2980-3040) */
__device__ __forceinline__ void m_xyzb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzb (pml.f:3044-3075) */
__device__ __forceinline__ void m_xzb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
    PML(PB, H_, PXZ) = (R(2.)*xm*dth*(w1[c] - w1[c - SX]) + PML(PB, H_, PXZ)* (R(2.) - dt*pht*rf[k]))/(R(2.) + dt*pht*rf[k]);
    xz[c] = PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
}

/* m_yzb (pml.f:3079-3110) */
__device__ __forceinline__ void m_yzb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
    PML(PB, H_, PYZ) = (R(2.)* xm*dth*(w1[c + SY] - w1[c])+ PML(PB, H_, PYZ)* (R(2.) - dt*pht*rf[k]))/(R(2.) + dt*pht*rf[k]);
    yz[c] = PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
}

/* m_xyb (pml.f:3114-3144) */
__device__ __forceinline__ void m_xyb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*rh[k])/(R(2.) + dt*rh[k]);
    PML(PB, H_, PXY) = (R(2.)* xm*dth*((u1[c + SY] - u1[c]) + (v1[c] - v1[c - SX])) + PML(PB, H_, PXY)* (R(2.) - dt*pht*rh[k]))/(R(2.) + dt*pht*rh[k]);
    xy[c] = PML(PB, T_, PXY) + PML(PB, H_, PXY);
}

/* m_xyzsw (pml.f:3151-3231) */
__device__ __forceinline__ void m_xyzsw(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzsw (pml.f:3235-3272) */
__device__ __forceinline__ void m_xzsw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[j] + pht*rh[i];
    PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[j] + rh[i];
    PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rh[i]);
    PML(PS, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PS, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PS, T_, PXZ) + PML(PW, T_, PXZ) + PML(PS, H_, PXZ);
}

/* m_yzsw (pml.f:3276-3313) */
__device__ __forceinline__ void m_yzsw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rf[i];
    PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rf[i];
    PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rf[i]);
    PML(PS, H_, PYZ) = (R(2.)*dth*xm*(v1[c + SZ] - v1[c]) + PML(PS, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PS, T_, PYZ) + PML(PW, T_, PYZ) + PML(PS, H_, PYZ);
}

/* m_xysw (pml.f:3317-3355) */
__device__ __forceinline__ void m_xysw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rh[i];
    PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[i];
    PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rh[i]);
    PML(PS, H_, PXY) = PML(PS, H_, PXY) * (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PS, T_, PXY) + PML(PW, T_, PXY) + PML(PS, H_, PXY);
}

/* m_xyzse (pml.f:3359-3439) */
__device__ __forceinline__ void m_xyzse(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzse (pml.f:3443-3480) */
__device__ __forceinline__ void m_xzse(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[j] + pht*rf[nx-i+1];
    PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[nx-i+1];
    PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rf[nx-i+1]);
    PML(PS, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PS, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PS, T_, PXZ) + PML(PE, T_, PXZ) + PML(PS, H_, PXZ);
}

/* m_yzse (pml.f:3484-3521) */
__device__ __forceinline__ void m_yzse(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rh[nx-i+1];
    PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[nx-i+1];
    PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rh[nx-i+1]);
    PML(PS, H_, PYZ) = (R(2.)* dth*xm*(v1[c + SZ] - v1[c])+ PML(PS, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PS, T_, PYZ) + PML(PE, T_, PYZ) + PML(PS, H_, PYZ);
}

/* m_xyse (pml.f:3525-3563) */
__device__ __forceinline__ void m_xyse(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rf[nx-i+1];
    PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rf[nx-i+1];
    PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rf[nx-i+1]);
    PML(PS, H_, PXY) = R(2.)*PML(PS, H_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PS, T_, PXY) + PML(PE, T_, PXY) + PML(PS, H_, PXY);
}

/* m_xyznw (pml.f:3567-3648) */
__device__ __forceinline__ void m_xyznw(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xznw (pml.f:3652-3689) */
__device__ __forceinline__ void m_xznw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[ny-j+1] + pht*rh[i];
    PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rh[i];
    PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[ny-j+1] + rh[i]);
    PML(PN, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PN, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PN, T_, PXZ) + PML(PW, T_, PXZ) + PML(PN, H_, PXZ);
}

/* m_yznw (pml.f:3693-3730) */
__device__ __forceinline__ void m_yznw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht * rf[i];
    PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rf[i];
    PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rh[ny-j+1] + rf[i]);
    PML(PN, H_, PYZ) = (R(2.)*dth*xm*(v1[c + SZ] - v1[c])+ PML(PN, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PN, T_, PYZ) + PML(PW, T_, PYZ) + PML(PN, H_, PYZ);
}

/* m_xynw (pml.f:3734-3772) */
__device__ __forceinline__ void m_xynw(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rh[i];
    PML(PN, T_, PXY) = (R(2.)*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rh[i];
    PML(PW, T_, PXY) = (R(2.)*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[ny-j+1] + rh[i]);
    PML(PN, H_, PXY) = PML(PN, H_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PN, T_, PXY) + PML(PW, T_, PXY) + PML(PN, H_, PXY);
}

/* m_xyzne (pml.f:3776-3856) */
__device__ __forceinline__ void m_xyzne(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzne (pml.f:3860-3897) */
__device__ __forceinline__ void m_xzne(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[ny-j+1] + pht * rf[nx-i+1];
    PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rf[nx-i+1];
    PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[ny-j+1] + rf[nx-i+1]);
    PML(PN, H_, PXZ) = (R(2.)*dth*xm*(u1[c + SZ] - u1[c]) + PML(PN, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PN, T_, PXZ) + PML(PE, T_, PXZ) + PML(PN, H_, PXZ);
}

/* m_yzne (pml.f:3901-3938) */
__device__ __forceinline__ void m_yzne(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rh[nx-i+1];
    PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*rh[ny-j+1]))/(R(2.) + dt*rh[ny-j+1]);
    dc=pht*rh[ny-j+1] + rh[nx-i+1];
    PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rh[ny-j+1] + rh[nx-i+1]);
    PML(PN, H_, PYZ) = (R(2.)* dth*xm*(v1[c + SZ] - v1[c])+ PML(PN, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PN, T_, PYZ) + PML(PE, T_, PYZ) + PML(PN, H_, PYZ);
}

/* m_xyne (pml.f:3942-3979) */
__device__ __forceinline__ void m_xyne(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rf[nx-i+1];
    PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rf[nx-i+1];
    PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    PML(PN, H_, PXY) = R(2.)*PML(PN, H_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PN, T_, PXY) + PML(PE, T_, PXY) + PML(PN, H_, PXY);
}

/* m_xyzsb (pml.f:3986-4066) */
__device__ __forceinline__ void m_xyzsb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzsb (pml.f:4070-4107) */
__device__ __forceinline__ void m_xzsb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[j] + pht*rf[k];
    PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[j] + rf[k]);
    PML(PB, H_, PXZ) = (R(2.)* dth*xm*(w1[c] - w1[c - SX])+ PML(PB, H_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PS, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
}

/* m_yzsb (pml.f:4111-4149) */
__device__ __forceinline__ void m_yzsb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rf[k];
    PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rf[k]);
    PML(PB, H_, PYZ) = PML(PB, H_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    yz[c] = PML(PS, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
}

/* m_xysb (pml.f:4153-4190) */
__device__ __forceinline__ void m_xysb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rh[k];
    PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rf[j] + rh[k]);
    PML(PB, H_, PXY) = (R(2.)*dth*xm*(v1[c] - v1[c - SX])+ PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xy[c] = PML(PS, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
}

/* m_xyznb (pml.f:4194-4274) */
__device__ __forceinline__ void m_xyznb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xznb (pml.f:4278-4315) */
__device__ __forceinline__ void m_xznb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[ny-j+1] + pht*rf[k];
    PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[ny-j+1] + rf[k]);
    PML(PB, H_, PXZ) = (R(2.)*dth*xm*(w1[c] - w1[c - SX]) + PML(PB, H_, PXZ) * (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PN, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
}

/* m_yznb (pml.f:4319-4357) */
__device__ __forceinline__ void m_yznb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rf[k];
    PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[ny-j+1] + rf[k]);
    PML(PB, H_, PYZ) = PML(PB, H_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    yz[c] = PML(PN, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
}

/* m_xynb (pml.f:4361-4398) */
__device__ __forceinline__ void m_xynb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rh[k];
    PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rh[ny-j+1] + rh[k]);
    PML(PB, H_, PXY) = (R(2.)* dth*xm*(v1[c] - v1[c - SX]) + PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xy[c] = PML(PN, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
}

/* m_xyzwb (pml.f:4402-4482) */
__device__ __forceinline__ void m_xyzwb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzwb (pml.f:4486-4524) */
__device__ __forceinline__ void m_xzwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[i] + pht*rf[k];
    PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[i] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[i] + rf[k]);
    PML(PB, H_, PXZ) = PML(PB, H_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xz[c] = PML(PW, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
}

/* m_yzwb (pml.f:4528-4565) */
__device__ __forceinline__ void m_yzwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[i] + pht*rf[k];
    PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[i] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[i] + rf[k]);
    PML(PB, H_, PYZ) = (R(2.)*dth*xm*(w1[c + SY] - w1[c])+ PML(PB, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PW, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
}

/* m_xywb (pml.f:4569-4606) */
__device__ __forceinline__ void m_xywb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[i] + pht*rh[k];
    PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[i] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rh[i] + rh[k]);
    PML(PB, H_, PXY) = (R(2.)*dth*xm*(u1[c + SY] - u1[c])+ PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xy[c] = PML(PW, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
}

/* m_xyzeb (pml.f:4610-4690) */
__device__ __forceinline__ void m_xyzeb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzeb (pml.f:4694-4732) */
__device__ __forceinline__ void m_xzeb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[nx-i+1] + pht*rf[k];
    PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[nx-i+1] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rf[nx-i+1] + rf[k]);
    PML(PB, H_, PXZ) = PML(PB, H_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xz[c] = PML(PE, T_, PXZ) + PML(PB, T_, PXZ) + PML(PB, H_, PXZ);
}

/* m_yzeb (pml.f:4736-4773) */
__device__ __forceinline__ void m_yzeb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[nx-i+1] + pht*rf[k];
    PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[nx-i+1] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*(rh[nx-i+1] + rf[k]);
    PML(PB, H_, PYZ) = (R(2.)* dth*xm*(w1[c + SY] - w1[c]) + PML(PB, H_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PE, T_, PYZ) + PML(PB, T_, PYZ) + PML(PB, H_, PYZ);
}

/* m_xyeb (pml.f:4777-4814) */
__device__ __forceinline__ void m_xyeb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[nx-i+1] + pht*rh[k];
    PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[nx-i+1] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*(rf[nx-i+1] + rh[k]);
    PML(PB, H_, PXY) = (R(2.)*dth*xm*(u1[c + SY] - u1[c]) + PML(PB, H_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xy[c] = PML(PE, T_, PXY) + PML(PB, T_, PXY) + PML(PB, H_, PXY);
}

/* m_xyzswb (pml.f:4821-4904) */
__device__ __forceinline__ void m_xyzswb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzswb (pml.f:4908-4946) */
__device__ __forceinline__ void m_xzswb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[j] + pht*rh[i] + pht*rf[k];
    PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[j] + rh[i] + pht*rf[k];
    PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + pht*rh[i] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PS, T_, PXZ) + PML(PW, T_, PXZ) + PML(PB, T_, PXZ);
}

/* m_yzswb (pml.f:4950-4988) */
__device__ __forceinline__ void m_yzswb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rf[i] + pht*rf[k];
    PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rf[i] + pht*rf[k];
    PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[j] + pht*rf[i] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PS, T_, PYZ) + PML(PW, T_, PYZ) + PML(PB, T_, PYZ);
}

/* m_xyswb (pml.f:4992-5030) */
__device__ __forceinline__ void m_xyswb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rh[i] + pht*rh[k];
    PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[i] + pht*rh[k];
    PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + pht*rh[i] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PS, T_, PXY) + PML(PW, T_, PXY) + PML(PB, T_, PXY);
}

/* m_xyzseb (pml.f:5034-5117) */
__device__ __forceinline__ void m_xyzseb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzseb (pml.f:5121-5159) */
__device__ __forceinline__ void m_xzseb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[j] + pht*rf[nx-i+1] + pht*rf[k];
    PML(PS, T_, PXZ) = PML(PS, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[j] + rf[nx-i+1] + pht*rf[k];
    PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[j] + pht*rf[nx-i+1] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PS, T_, PXZ) + PML(PE, T_, PXZ) + PML(PB, T_, PXZ);
}

/* m_yzseb (pml.f:5163-5201) */
__device__ __forceinline__ void m_yzseb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rh[nx-i+1] + pht*rf[k];
    PML(PS, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PS, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rh[nx-i+1] + pht*rf[k];
    PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[j] + pht*rh[nx-i+1] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PS, T_, PYZ) + PML(PE, T_, PYZ) + PML(PB, T_, PYZ);
}

/* m_xyseb (pml.f:5205-5243) */
__device__ __forceinline__ void m_xyseb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[j] + pht*rf[nx-i+1] + pht*rh[k];
    PML(PS, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PS, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + rf[nx-i+1] + pht*rh[k];
    PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[j] + pht*rf[nx-i+1] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PS, T_, PXY) + PML(PE, T_, PXY) + PML(PB, T_, PXY);
}

/* m_xyznwb (pml.f:5247-5330) */
__device__ __forceinline__ void m_xyznwb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xznwb (pml.f:5334-5372) */
__device__ __forceinline__ void m_xznwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[ny-j+1] + pht*rh[i] + pht*rf[k];
    PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rh[i] + pht*rf[k];
    PML(PW, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PW, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + pht*rh[i] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    xz[c] = PML(PN, T_, PXZ) + PML(PW, T_, PXZ) + PML(PB, T_, PXZ);
}

/* m_yznwb (pml.f:5376-5414) */
__device__ __forceinline__ void m_yznwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rf[i] + pht*rf[k];
    PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rf[i] + pht*rf[k];
    PML(PW, T_, PYZ) = PML(PW, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + pht*rf[i] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PN, T_, PYZ) + PML(PW, T_, PYZ) + PML(PB, T_, PYZ);
}

/* m_xynwb (pml.f:5418-5456) */
__device__ __forceinline__ void m_xynwb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rh[i] + pht*rh[k];
    PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rh[i] + pht*rh[k];
    PML(PW, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PW, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + pht*rh[i] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PN, T_, PXY) + PML(PW, T_, PXY) + PML(PB, T_, PXY);
}

/* m_xyzneb (pml.f:5460-5543) */
__device__ __forceinline__ void m_xyzneb(const PmlCell &x)
{
    PML_CELL_LOCALS
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
}

/* m_xzneb (pml.f:5547-5585) */
__device__ __forceinline__ void m_xzneb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rf[ny-j+1] + pht*rf[nx-i+1] + pht*rf[k];
    PML(PN, T_, PXZ) = PML(PN, T_, PXZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + rf[nx-i+1] + pht*rf[k];
    PML(PE, T_, PXZ) = (R(2.)*dth*xm* (w1[c] - w1[c - SX]) + PML(PE, T_, PXZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rf[ny-j+1] + pht*rf[nx-i+1] + rf[k];
    PML(PB, T_, PXZ) = (R(2.)*dth*xm* (u1[c + SZ] - u1[c]) + PML(PB, T_, PXZ)* (R(2.) - dt*rf[k]))/(R(2.) + dt*rf[k]);
    xz[c] = PML(PN, T_, PXZ) + PML(PE, T_, PXZ) + PML(PB, T_, PXZ);
}

/* m_yzneb (pml.f:5589-5627) */
__device__ __forceinline__ void m_yzneb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rh[nx-i+1] + pht*rf[k];
    PML(PN, T_, PYZ) = (R(2.)*dth*xm* (w1[c + SY] - w1[c]) + PML(PN, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rh[nx-i+1] + pht*rf[k];
    PML(PE, T_, PYZ) = PML(PE, T_, PYZ)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + pht*rh[nx-i+1] + rf[k];
    PML(PB, T_, PYZ) = (R(2.)*dth*xm* (v1[c + SZ] - v1[c]) + PML(PB, T_, PYZ)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    yz[c] = PML(PN, T_, PYZ) + PML(PE, T_, PYZ) + PML(PB, T_, PYZ);
}

/* m_xyneb (pml.f:5631-5669) */
__device__ __forceinline__ void m_xyneb(const PmlCell &x)
{
    PML_CELL_LOCALS
    xm = R(1.)/mu[c];
    dc=rh[ny-j+1] + pht*rf[nx-i+1] + pht*rh[k];
    PML(PN, T_, PXY) = (2*dth*xm* (u1[c + SY] - u1[c]) + PML(PN, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + rf[nx-i+1] + pht*rh[k];
    PML(PE, T_, PXY) = (2*dth*xm* (v1[c] - v1[c - SX]) + PML(PE, T_, PXY)* (R(2.) - dt*dc))/(R(2.) + dt*dc);
    dc=pht*rh[ny-j+1] + pht*rf[nx-i+1] + rh[k];
    PML(PB, T_, PXY) = PML(PB, T_, PXY)* (R(2.) - dt*dc)/(R(2.) + dt*dc);
    xy[c] = PML(PN, T_, PXY) + PML(PE, T_, PXY) + PML(PB, T_, PXY);
}

#endif
