// fd3d_common.cuh -- device data layout and launch-wide constants of the B200 path.
//
// Layout in HBM (one model):
//   * 9 wave fields (u,v,w,xx,yy,zz,xy,yz,xz) and 3 media (lam1,mu1,d1), each a
//     separate array of nzt x nyt rows of `px` elements.  Element (i,j,k) of the
//     reference (1-based, x fastest) lives at  off + (i-1) + px*((j-1) + nyt*(k-1)).
//     `off` shifts the row so that i = nabc+1, the first interior column, starts on a
//     128-byte boundary (fp32) and px (a multiple of 32) keeps every row aligned.
//   * fault-plane arrays (i,k) at (i-1) + nxt*(k-1), the reference's own layout.
//   * PML auxiliary arrays per strip: (ni x nj1 x nk), i fastest, as allocated by
//     init_pml (src/fd3d_deriv.f90:1319-1410), one array per split component.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fd3d {

struct Grid {
    int nxt, nyt, nzt, nabc, nfs;
    int px;          // row pitch (elements)
    int off;         // x offset of i=1 inside a row
    long long plane; // px*nyt
    long long n3;    // plane*nzt + tail pad

    __host__ __device__ __forceinline__ long long at(int i, int j, int k) const {
        return (long long)off + (i - 1) + (long long)px * (j - 1) + plane * (k - 1);
    }
    __host__ __device__ __forceinline__ int at2(int i, int k) const { return (i - 1) + nxt * (k - 1); }
    __host__ __device__ __forceinline__ int ks() const { return nzt - nfs; }  // free-surface row
};

// Split-field PML strip (strip s = 1 x-low, 2 x-high, 3 y-low, 4 z-low).
struct Strip {
    int nxb, nxe, nyb, nye, nzb, nze;  // reference box (v/xy/yz loops end at nye)
    int ni, nj1, nk;                   // aux dims, nj1 = nye-nyb+2
    int jend_uw;                       // last j of the u/w and normal/xz loops
    long long base;                    // offset of this strip in each aux pool
    long long ncells;                  // ni*nj1*nk
    int ox_off, oxS_off, oy_off, oyS_off, oz_off, ozS_off;  // offsets into the profile table
};

// 24 split components per strip: u(3) v(3) w(3) xx(3) yy(3) zz(3) xy(2) xz(2) yz(2)
enum AuxId {
    AX_U0 = 0, AX_U1, AX_U2, AX_V0, AX_V1, AX_V2, AX_W0, AX_W1, AX_W2,
    AX_XX0, AX_XX1, AX_XX2, AX_YY0, AX_YY1, AX_YY2, AX_ZZ0, AX_ZZ1, AX_ZZ2,
    AX_XY0, AX_XY1, AX_XZ0, AX_XZ1, AX_YZ0, AX_YZ1, AX_N
};

template <class T>
struct Fields {
    T *u, *v, *w, *xx, *yy, *zz, *xy, *yz, *xz;
    const T *lam, *mu, *d;
};

// Fault-plane state.  F = field type, double = accumulators (slip, slip path,
// rupture time, rise, slip time, psi).
template <class T>
struct Fault {
    // traction_com
    T *tx, *tz;           // traction after friction (read by next step's fault velocity)
    T *txt, *tzt;         // trial traction (before friction)
    T *RFx, *RFz, *avdx, *avdz, *v1t, *au1, *av1, *aw1;
    // friction_com
    T *uZ, *wX, *tabsX, *tabsZ, *T0X, *T0Z, *T0Xb, *Dc;
    T *peakX, *dynX, *DcX, *peakZ, *dynZ, *DcZ, *coh;
    T *aX, *bX, *vwX, *fwX, *aZ, *bZ, *vwZ, *fwZ;
    double *psiX, *psiZ;
    // source_com
    double *distX, *distZ, *slipX, *slipZ, *ruptime, *rise, *sliptime;
    T *schangeX, *schangeZ;  // last step's shear traction / strength planes
};

struct FvwScalars {
    double Sn, v0, f0, fw, uini, wini;
    int nucleation;
    double hx0, hz0, perturb, RR2, TT2, strinixI;
};

// Scalars of one time step in the field type T, computed on the host exactly as the
// reference computes them in `real` (dth = dt/dh, ...).
template <class T>
struct StepConst {
    T dt, dh, dth, dth2, dht, damp_s, c1, c2;
    double dtA, dhA, dthA;   // FP64 copies for the FP64 parts
};

// Device-side status word bits.
enum { ST_NEWTON = 1, ST_NONFINITE = 2 };

#ifndef FD3D_NEWTON_MAXIT
#define FD3D_NEWTON_MAXIT 200
#endif

}  // namespace fd3d
