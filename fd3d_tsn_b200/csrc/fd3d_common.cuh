// fd3d_common.cuh -- device data layout and launch-wide constants of the B200 path.
//
// Layout in HBM (one model):
//   * 9 wave fields (u,v,w,xx,yy,zz,xy,yz,xz) and 3 media (lam1,mu1,d1), each a
//     separate array of nzt x nyt rows of `px` elements.  Element (i,j,k) of the
//     reference (1-based, x fastest) lives at  off + (i-1) + px*((j-1) + nyt*(k-1)).
//     `off` shifts the row so that i = nabc+1, the first interior column, starts on a
//     128-byte boundary (fp32) and px (a multiple of 32) keeps every row aligned.
//   * fault-plane arrays (i,k) at (i-1) + nxt*(k-1), the reference's own layout.
//   * PML auxiliary (split) components of init_pml (src/fd3d_deriv.f90:1319-1410): one
//     pool indexed by the compact cell index of the strips (4, or 5 under FSPACE), in 32-cell blocks per
//     group of components (PmlAux, fd3d_kernels.cuh).
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace fd3d {

struct Grid {
    int nxt, nyt, nzt, nabc, nfs;
    int fspace;      // FSPACE build: a PML strip above k = ks() instead of the free surface
    int px;          // row pitch (elements)
    int off;         // x offset of i=1 inside a row
    long long plane; // px*nyt
    long long n3;    // plane*nzl + tail pad: the elements of one stored 3-D array
    // z-slab of a model decomposed over several contexts: the context updates planes
    // klo..khi and stores planes kofs+1 .. kofs+nzl (its own and the halo planes of its
    // neighbours).  Field pointers are offset by -kofs planes, so at() takes the global k
    // everywhere.  A whole model: klo = 1, khi = nzt, kofs = 0, nzl = nzt.
    int klo, khi, kofs, nzl;

    __host__ __device__ __forceinline__ long long at(int i, int j, int k) const {
        return (long long)off + (i - 1) + (long long)px * (j - 1) + plane * (k - 1);
    }
    __host__ __device__ __forceinline__ int at2(int i, int k) const { return (i - 1) + nxt * (k - 1); }
    __host__ __device__ __forceinline__ int ks() const { return nzt - nfs; }  // free-surface row (top row of the
                                                                              // interior box under FSPACE)
    __host__ __device__ __forceinline__ bool owns(int k) const { return k >= klo && k <= khi; }
    // the planes of the interior box (and fault rows) this context updates
    __host__ __device__ __forceinline__ int kin_lo() const { return klo > nabc + 1 ? klo : nabc + 1; }
    __host__ __device__ __forceinline__ int kin_hi() const { return khi < ks() ? khi : ks(); }
};

// Split-field PML strip (strip s = 1 x-low, 2 x-high, 3 y-low, 4 z-low, 5 z-high under FSPACE).
struct Strip {
    int nxb, nxe, nyb, nye, nzb, nze;  // reference box (v/xy/yz loops end at nye)
    int ni, nj1, nk;                   // aux dims, nj1 = nye-nyb+2
    int jend_uw;                       // last j of the u/w and normal/xz loops
    long long base;                    // offset of this strip in each aux pool
    long long ncells;                  // ni*nj1*nk
    int ox_off, oxS_off, oy_off, oyS_off, oz_off, ozS_off;  // offsets into the profile table
    float rni, rnj;                    // 1/ni, 1/(jend_uw-nyb+1) for the index split (udiv_small)
    int fastdiv;                       // the strip's u/w range has fewer than 2^24 cells
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
    // The same medium as a 1-D profile when it varies with k only (the layered medium
    // of readcrustalmodel): lam at lay[k-1], mu at lay[nzt+k-1], d at lay[2*nzt+k-1],
    // dth/d (the IEEE quotient the interior velocity sweep forms per cell) at
    // lay[3*nzt+k-1] and dt/d (the PML velocity sweep's) at lay[4*nzt+k-1]; null
    // otherwise.  The interior and PML sweeps then read values per plane instead of
    // arrays per cell.
    const T* lay;
};
constexpr int LAY_N = 5;  // profile entries per plane

// Fault-plane state.  F = field type, double = accumulators (slip, slip path,
// rupture time, rise, slip time, psi).
//
// avdx, avdz (the damping memory of the trial traction) and distX (the slip path of the
// X nodes) hold two planes each: step it reads plane (it+1)&1 and writes plane it&1, so
// the fault boundary condition, which recomputes the trial and post-friction tractions of
// a tile's neighbouring nodes, never reads a value another CTA is updating.  After n steps
// the current plane is n&1 (pp_rd / pp_wr below).
template <class T>
struct Fault {
    // traction_com
    T *tx, *tz;           // traction after friction (read by next step's fault velocity)
    T *txt, *tzt;         // trial traction (scratch of the separate-launch fault BC only)
    T *RFx, *RFz, *avdx, *avdz, *v1t, *au1, *av1, *aw1;
    // friction_com
    T *uZ, *wX, *tabsX, *tabsZ, *T0X, *T0Z, *T0Xb, *Dc;
    T *peakX, *dynX, *DcX, *peakZ, *dynZ, *DcZ, *coh;
    T *aX, *bX, *vwX, *fwX, *aZ, *bZ, *vwZ, *fwZ;
    double *psiX, *psiZ;
    // source_com
    double *distX, *distZ, *slipX, *slipZ, *ruptime, *rise, *sliptime;
    T *schangeX, *schangeZ;  // last step's shear traction / strength planes
    int n2;                  // nxt*nzt, the size of one plane
};

// plane of a two-plane state array that step `it` reads / writes
template <class U>
__host__ __device__ __forceinline__ U* pp_rd(U* base, int it, int n2) { return base + (size_t)((it + 1) & 1) * n2; }
template <class U>
__host__ __device__ __forceinline__ U* pp_wr(U* base, int it, int n2) { return base + (size_t)(it & 1) * n2; }

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
    T rdh;                   // RN(1/dh) for div_pre (NaN: divide directly)
    double dtA, dhA, dthA;   // FP64 copies for the FP64 parts
};

// x / b rounded to nearest for a divisor b > 0 known before the launch, given
// y = RN(1/b) formed on the host by an IEEE division.
//
// Method: Markstein's theorem (P. W. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; also in
// J.-M. Muller et al., "Handbook of Floating-Point Arithmetic", the chapter on
// FMA-based division): if y is within half an ulp of 1/b and q within one ulp of
// x/b, the remainder r = x - b*q is exact and RN(q + r*y) = RN(x/b).  q0 = RN(x*y)
// can be 1.5 ulp off, so one correction step first brings it within one ulp; the
// second step is the theorem's.  Five FP32 operations, no reciprocal
// approximation and no branch on the common path.
//
// The theorem assumes that nothing under- or overflows.  For |x| outside
// [2^-98, 2^98] (zero aside), NaN, infinities and a divisor outside the range checked
// on the host (y is NaN then) the quotient is formed in FP64 and rounded to FP32: both
// operands are exact in FP64, and rounding a quotient first to 53 bits and then to 24
// (or fewer, for a subnormal result) gives the directly rounded quotient because
// 53 >= 2*24 + 2 (S. A. Figueroa, "When is double rounding innocuous?", SIGNUM
// Newsletter 30(3), 1995).  A zero dividend stays on the common path: every step then
// yields a zero, and the sign of x put on the result makes it the signed zero x/b is
// (for any other x in range the quotient already has the sign of x, since b > 0).  Zero
// is the value of every cell ahead of the wavefront, so it must cost no more than a
// normal value.  The result is therefore the IEEE FP32 quotient for every input; an
// exhaustive GPU test over all 2^32 dividends (fd3d_check_division) holds it to that.
// (The wave field's leading edge carries long runs of tiny values, so the fallback must
// not be the slow path of a single-precision division.)
__device__ __forceinline__ float div_pre(float x, float b, float y) {
    float q = __fmul_rn(x, y);
    float r = __fmaf_rn(-q, b, x);
    q = __fmaf_rn(r, y, q);
    r = __fmaf_rn(-q, b, x);
    float q2 = copysignf(__fmaf_rn(r, y, q), x);
    const float a = fabsf(x);
    if (!((a >= 0x1p-98f || a == 0.0f) && a <= 0x1p98f && q2 == q2))
        q2 = __double2float_rn(__ddiv_rn((double)x, (double)b));
    return q2;
}
// the FP64 build divides directly (parity build, not the fast path)
__device__ __forceinline__ double div_pre(double x, double b, double) { return x / b; }

// y = RN(1/b) for div_pre, or NaN when b is outside [2^-20, 2^20] (FP64 fallback)
template <class T>
inline T div_pre_recip(T b) {
    const double ab = (double)b;
    if (!(ab >= 0x1p-20 && ab <= 0x1p20)) return (T)NAN;
    return (T)1 / b;
}

// n / d for n < 2^24 and 1 <= d < 2^24 with rd = RN(1/d): the float product is within
// one of the quotient, and one remainder test each way makes it exact (a few integer
// operations instead of a 32-bit division, which the GPU runs as a long sequence).
__host__ __device__ __forceinline__ unsigned udiv_small(unsigned n, unsigned d, float rd, unsigned& rem) {
    unsigned q = (unsigned)((float)n * rd);
    int r = (int)(n - q * d);
    if (r < 0) { --q; r += (int)d; }
    else if (r >= (int)d) { ++q; r -= (int)d; }
    rem = (unsigned)r;
    return q;
}

// Device-side status word bits.
enum { ST_NEWTON = 1, ST_NONFINITE = 2, ST_TIMEOUT = 4 };

#ifndef FD3D_NEWTON_MAXIT
#define FD3D_NEWTON_MAXIT 200
#endif

}  // namespace fd3d
