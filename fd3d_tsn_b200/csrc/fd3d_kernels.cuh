// fd3d_kernels.cuh -- sm_100a kernels of one FD3D_TSN time step (templated on the
// field type T: float for the production build, double for the FP64 build).
//
// The step is eight launches, each a set of reference regions whose write sets are
// disjoint and which read nothing another thread of the same launch writes (the fused
// fault boundary condition forms what its fres CTAs write from what they read):
//   1 vel_interior  uxx1/vyy1/wzz1 (fd3d_deriv.f90:50-193)
//   2 vel_fault     uxx0a/vyy0a/wzz0a at j=nyt-1 + v mirror (fd3d_deriv.f90:198-508),
//                   tasu1/tasw1 at j=nyt (fd3d_deriv.f90:1109-1234)
//   3 vel_pml       pml_uvw, 4 strips, 5 under FSPACE (fd3d_deriv.f90:1927-2299)
//   4 vel_fs        fuvw (fd3d_deriv.f90:1018-1062)
//   5 str_interior  dstres (fd3d_deriv.f90:513-622)
//   6 str_fault     sxx/sxy0/sxz0/syz0 at j=nyt-1 + xy/yz mirror, sxz1, tasii
//                   (fd3d_deriv.f90:677-1012,1239-1314)
//   7 str_pml       pml_xyz (fd3d_deriv.f90:2304-2992)
//   8 fault_bc      fres (fd3d_deriv.f90:1067-1104) and the fault boundary condition
//                   (fd3d_theo.f90:225-467): trial traction, |T| at the staggered nodes,
//                   friction law with slip and rupture time, output planes, fused per
//                   tile (fault_bc_body)
// and, for rate-and-state runs with a nucleation ramp, the ramp (fd3d_theo.f90:487-542).
// The fault boundary condition also exists as separate launches (str_fs, traction,
// friction, output), which fd3d_run_noalloc uses.
//
// Operation order inside every expression follows the reference so that, with
// contraction of multiply-add switched off (--fmad=false), the FP32 and FP64
// builds reproduce the CPU restatement's arithmetic exactly for slip weakening.
#pragma once
#include "fd3d_async.cuh"
#include "fd3d_common.cuh"

namespace fd3d {

// ---------------------------------------------------------------- velocity
// Interior 4th-order velocity: one thread per (i,j), marching a chunk of k.
template <class T>
__global__ void __launch_bounds__(256) k_vel_interior(Grid g, Fields<T> f, StepConst<T> c, int kchunk) {
    const int i = g.nabc + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = g.nabc + 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nxt - g.nabc || j > g.nyt - 2) return;
    const int kb = g.kin_lo() + blockIdx.z * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const long long sy = g.px, sz = g.plane;
    const T c1 = c.c1, c2 = c.c2;
    const T* __restrict__ xx = f.xx; const T* __restrict__ yy = f.yy; const T* __restrict__ zz = f.zz;
    const T* __restrict__ xy = f.xy; const T* __restrict__ yz = f.yz; const T* __restrict__ xz = f.xz;
    for (int k = kb; k <= ke; ++k) {
        const long long p = g.at(i, j, k);
        const T r = c.dth / f.d[p];
        f.u[p] = f.u[p] + r * (c1 * (xx[p] - xx[p - 1]) + c2 * (xx[p + 1] - xx[p - 2]) +
                               c1 * (xy[p] - xy[p - sy]) + c2 * (xy[p + sy] - xy[p - 2 * sy]) +
                               c1 * (xz[p] - xz[p - sz]) + c2 * (xz[p + sz] - xz[p - 2 * sz]));
        f.v[p] = f.v[p] + r * (c1 * (xy[p + 1] - xy[p]) + c2 * (xy[p + 2] - xy[p - 1]) +
                               c1 * (yy[p + sy] - yy[p]) + c2 * (yy[p + 2 * sy] - yy[p - sy]) +
                               c1 * (yz[p] - yz[p - sz]) + c2 * (yz[p + sz] - yz[p - 2 * sz]));
        f.w[p] = f.w[p] + r * (c1 * (xz[p + 1] - xz[p]) + c2 * (xz[p + 2] - xz[p - 1]) +
                               c1 * (yz[p] - yz[p - sy]) + c2 * (yz[p + sy] - yz[p - 2 * sy]) +
                               c1 * (zz[p + sz] - zz[p]) + c2 * (zz[p + 2 * sz] - zz[p - sz]));
    }
}

// FVW Newton solve of one node (fd3d_deriv.f90:1148-1161), FP64, bounded.
__device__ __forceinline__ double fvw_newton(double vtilde, double cdelta, double uw, double psi, double a,
                                             double v0, int* status) {
    const double e = v0 * exp(-psi / a);
    double ferr = 10.0;
    int it = 0;
    while (fabs(ferr) > 1e-10) {
        ++it;
        const double fwv = vtilde + cdelta * uw + sinh(uw) * e;
        const double dfw = cdelta + cosh(uw) * e;
        ferr = fwv / dfw;
        uw = uw - ferr;
        if (it > FD3D_NEWTON_MAXIT) { atomicOr(status, ST_NEWTON); break; }
    }
    return uw;
}

// Band j=nyt-1 (2nd order + damping, v mirror) and split-node fault velocity at j=nyt.
template <class T>
__device__ __forceinline__ void vel_fault_body(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, int law, FvwScalars s,
                            int* it_dev, int* status, int bx_, int by_, int bz_) {
    const int ii = bx_ * blockDim.x + threadIdx.x;
    const int kk = by_ * blockDim.y + threadIdx.y;
    if (ii == 0 && kk == 0) atomicAdd(it_dev, 1);  // step counter read by the fault BC launches
    const int ks = g.ks();
    const long long sy = g.px, sz = g.plane;
    // ghost row k=ks+1: v(:,nyt,ks+1) = v(:,nyt-1,ks+1)  (bnd2d mirror, fd3d_deriv.f90:225-232);
    // under FSPACE that row belongs to the top PML strip, whose tiles mirror it
    if (!g.fspace && kk == 0 && ii < g.nxt && g.owns(ks + 1)) {
        const long long p = g.at(ii + 1, g.nyt - 1, ks + 1);
        f.v[p + sy] = f.v[p];
    }
    const int i = g.nabc + 1 + ii, k = g.kin_lo() + kk;
    if (i > g.nxt - g.nabc || k > g.kin_hi()) return;
    const int n2 = g.at2(i, k);
    {   // uxx0a / vyy0a / wzz0a  (fd3d_deriv.f90:284-508)
        const long long p = g.at(i, g.nyt - 1, k);
        const T r = c.dth / f.d[p];
        const T pdx = (f.xx[p] - f.xx[p - 1]) + (f.xy[p] - f.xy[p - sy]) + (f.xz[p] - f.xz[p - sz]);
        const T au = pdx - q.au1[n2];
        f.u[p] = f.u[p] + r * (pdx + c.damp_s * au);
        q.au1[n2] = pdx;
        const T pdy = (f.xy[p + 1] - f.xy[p]) + (f.yy[p + sy] - f.yy[p]) + (f.yz[p] - f.yz[p - sz]);
        const T av = pdy - q.av1[n2];
        const T vn = f.v[p] + r * (pdy + c.damp_s * av);
        f.v[p] = vn;
        f.v[p + sy] = vn;  // mirror into the fault plane
        q.av1[n2] = pdy;
        const T pdz = (f.xz[p + 1] - f.xz[p]) + (f.yz[p] - f.yz[p - sy]) + (f.zz[p + sz] - f.zz[p]);
        const T aw = pdz - q.aw1[n2];
        f.w[p] = f.w[p] + r * (pdz + c.damp_s * aw);
        q.aw1[n2] = pdz;
    }
    const long long pf = g.at(i, g.nyt, k);
    if (law == 0) {  // tasu1/tasw1 slip weakening
        const T r = c.dth / f.d[pf];
        f.u[pf] = f.u[pf] + r * (T)2 * (q.tx[n2] + q.RFx[n2]);
        f.w[pf] = f.w[pf] + r * ((T)2 * (q.tz[n2] + q.RFz[n2]));
        return;
    }
    // FVW (fd3d_deriv.f90:1141-1162, 1204-1226), FP64
    const double d = (double)f.d[pf];
    const double rr = c.dthA / d;
    {
        const double u = (double)f.u[pf];
        const double a = (double)q.aX[n2];
        const double s1 = 2.0 * (fabs((double)q.wX[n2]) + fabs(s.wini)), s2 = 2.0 * (fabs(u) + fabs(s.uini));
        const double sr = sqrt(s1 * s1 + s2 * s2);
        const double cdelta = 2.0 * rr * s.Sn * a;
        double uw = asinh(exp(q.psiX[n2] / a) * sr / (2.0 * s.v0));
        const double rfz = ((double)q.RFz[n2] + (double)q.RFz[g.at2(i - 1, k)] + (double)q.RFz[g.at2(i, k - 1)] +
                            (double)q.RFz[g.at2(i - 1, k - 1)]) / 4.0;
        const double q1 = (double)q.wX[n2] + 2.0 * rr * (rfz - (double)q.T0Z[n2]);
        const double q2 = u + 2.0 * rr * ((double)q.RFx[n2] - (double)q.T0X[n2]);
        const double vt = -sqrt(q1 * q1 + q2 * q2);
        uw = fvw_newton(vt, cdelta, uw, q.psiX[n2], a, s.v0, status);
        f.u[pf] = (T)(((double)q.tx[n2] + (double)q.T0X[n2]) * (-sinh(uw)) * s.v0 * exp(-q.psiX[n2] / a) /
                      (double)q.tabsX[n2] + s.uini);
    }
    {
        const double w = (double)f.w[pf];
        const double a = (double)q.aZ[n2];
        const double s1 = 2.0 * (w - s.wini), s2 = 2.0 * ((double)q.uZ[n2] - s.uini);
        const double sr = sqrt(s1 * s1 + s2 * s2);
        const double cdelta = 2.0 * rr * s.Sn * a;
        double uw = asinh(exp(q.psiZ[n2] / a) * sr / (2.0 * s.v0));
        const int e1 = g.at2(i + 1, k), e2 = g.at2(i, k + 1), e3 = g.at2(i + 1, k + 1);
        const double rfx = ((double)q.RFx[n2] + (double)q.RFx[e1] + (double)q.RFx[e2] + (double)q.RFx[e3]) / 4.0;
        const double t0x = ((double)q.T0X[n2] + (double)q.T0X[e1] + (double)q.T0X[e2] + (double)q.T0X[e3]) / 4.0;
        const double q1 = w + 2.0 * rr * ((double)q.RFz[n2] - (double)q.T0Z[n2]);
        const double q2 = (double)q.uZ[n2] + 2.0 * rr * (rfx - t0x);
        const double vt = -sqrt(q1 * q1 + q2 * q2);
        uw = fvw_newton(vt, cdelta, uw, q.psiZ[n2], a, s.v0, status);
        f.w[pf] = (T)(((double)q.tz[n2] + (double)q.T0Z[n2]) * (-sinh(uw) * s.v0 * exp(-q.psiZ[n2] / a)) /
                      (double)q.tabsZ[n2] + s.wini);
    }
}

constexpr int PML_MAXS = 5;  // strips 1-4, and 5 (the top) under FSPACE
struct PmlDesc {
    Strip s[PML_MAXS];
    long long cum[PML_MAXS + 1];  // first compact index of each strip (a multiple of PML_TILE); cum[PML_MAXS] = end
    long long cnt[PML_MAXS];      // cells of each strip's u/w loop range (0 for an absent strip)
    int ns;                       // strips present: 4, or 5 under FSPACE
    int klo, khi;                 // planes updated (Grid::klo, khi)
};

// PML auxiliary components (the 24 split fields that init_pml allocates per strip,
// fd3d_deriv.f90:1330-1406, 1413-1437) are indexed by the compact cell index t of the
// u/w loop ranges of the strips (strip s holds t in [cum[s], cum[s] + cnt[s]); each strip
// starts on a PML_TILE boundary, so every tile lies in one strip) and stored in blocks of
// 32 cells: inside a block the 32 values of one component are contiguous and the
// components of a group follow each other.  The velocity group (u,v,w splits, 9
// components) and the stress group (xx,yy,zz,xy,xz,yz splits, 15) are separate spans,
// so the auxiliaries of PML_TILE consecutive cells are one contiguous range per group:
// one bulk copy brings a tile's range into shared memory.
constexpr int AUX_NV = 9, AUX_NS = 15;
constexpr int PML_TILE = 256;
inline long long pml_aux_cells(const PmlDesc& D) { return (D.cum[PML_MAXS] + PML_TILE - 1) / PML_TILE * PML_TILE; }
inline size_t pml_aux_elems(const PmlDesc& D) { return (size_t)pml_aux_cells(D) * (AUX_NV + AUX_NS); }

// One entry of a damping profile (init_pml's omega at one index): the factors
// 1 - omega and 1 + omega of the split-field update and y = RN(1/(1 + omega)) for
// div_pre, formed on the host with the same IEEE operations the reference performs.
template <class T>
struct alignas(4 * sizeof(T)) Damp {
    T m, p, r, o;  // 1 - omega, 1 + omega, RN(1/(1 + omega)), omega
};

// Damping of one split direction over a strip, from where init_pml leaves the profiles
// zero (fd3d_deriv.f90:1436-1490): the x strips are damped in x only, the y strip in y
// and, in its corners, in x; the z strips in z and, in their corners and edges, in x and
// y.  SPLIT_NEVER: omega = 0 over the whole strip, the update is p + inc.  SPLIT_ALWAYS:
// the general form (p*(1-omega) + inc)/(1+omega), which is also exact where omega = 0
// (a*1 = a, x/1 = x).  SPLIT_MAYBE: the general form where any lane of the warp is
// damped, p + inc where none is (a warp-uniform branch, so no lane forms a quotient it
// discards).  The host checks the SPLIT_NEVER directions against the profiles
// (pml_modes_hold).
enum { SPLIT_NEVER = 0, SPLIT_MAYBE = 1, SPLIT_ALWAYS = 2 };
// strip class: 0 the x strips (1, 2), 1 the y strip (3), 2 the z strips (4, and 5 under FSPACE)
__host__ __device__ constexpr int pml_class(int s) { return s <= 1 ? 0 : (s == 2 ? 1 : 2); }
// mode of direction DIR (0 x, 1 y, 2 z) in strip class C
__host__ __device__ constexpr int split_mode(int C, int DIR) {
    return DIR == C ? SPLIT_ALWAYS : (DIR < C ? SPLIT_MAYBE : SPLIT_NEVER);
}

template <class T, int MODE>
__device__ __forceinline__ T pml_split(T p, T inc, const Damp<T>& o, bool warp_damped) {
    if (MODE == SPLIT_NEVER || (MODE == SPLIT_MAYBE && !warp_damped)) return p + inc;
    return div_pre(p * o.m + inc, o.p, o.r);
}

template <class T>
struct PmlAux {
    T* vel;              // velocity group, pml_aux_cells * AUX_NV elements
    T* str;              // stress group, pml_aux_cells * AUX_NS elements
    const Damp<T>* prof; // damping profiles
};

// carve the two groups out of one pool of pml_aux_elems(D) elements
template <class T>
inline void pml_aux_bind(PmlAux<T>& X, T* pool, const PmlDesc& D) {
    X.vel = pool;
    X.str = pool + pml_aux_cells(D) * AUX_NV;
}

// shared-memory slot of component c of the cell that thread l of a tile owns
__device__ __forceinline__ int aux_sm(int l, int ncomp, int c) { return (l >> 5) * 32 * ncomp + 32 * c + (l & 31); }

// strip of the tile that starts at compact index t0
__device__ __forceinline__ int pml_tile_strip(const PmlDesc& D, long long t0) {
    return (t0 >= D.cum[1]) + (t0 >= D.cum[2]) + (t0 >= D.cum[3]) + (t0 >= D.cum[4]);
}

// (i,j,k) of compact cell index t of strip s; false past the strip's last cell and, for
// a z-slab (SLAB), outside its planes
template <bool SLAB>
__device__ __forceinline__ bool pml_cell(const PmlDesc& D, int s, long long t, int& i, int& j, int& k) {
    const long long r0 = t - D.cum[s];
    if (r0 >= D.cnt[s]) return false;
    const Strip& S = D.s[s];
    // strip-local index fits 32 bits (a strip is ni*nj*nk cells)
    const unsigned r = (unsigned)r0;
    const unsigned ni = (unsigned)S.ni, nj = (unsigned)(S.jend_uw - S.nyb + 1);
    unsigned q1, k2, ri, rj;
    if (S.fastdiv) {
        q1 = udiv_small(r, ni, S.rni, ri);
        k2 = udiv_small(q1, nj, S.rnj, rj);
    } else {
        q1 = r / ni; ri = r - q1 * ni;
        k2 = q1 / nj; rj = q1 - k2 * nj;
    }
    i = S.nxb + (int)ri; j = S.nyb + (int)rj; k = S.nzb + (int)k2;
    return !SLAB || (k >= D.klo && k <= D.khi);
}

// Start of a tile: every thread orders its earlier generic accesses of the staging
// buffer before the async copy, then one thread issues the bulk load of the tile's
// range of the group (ncomp components).
template <class T>
__device__ __forceinline__ void pml_tile_begin(T* sm, const T* src, int ncomp, uint32_t bar) {
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        fence_proxy_async_global();
        const uint32_t bytes = PML_TILE * ncomp * (uint32_t)sizeof(T);
        mbar_expect_tx(bar, bytes);
        bulk_load(smem_addr(sm), src, bytes, bar);
    }
}
// Wait (bounded) for the tile's load; false on every thread if any thread gave up
// (ST_TIMEOUT recorded after one more bounded wait for the copy in flight).  Every
// thread of the CTA leaves it converged.
__device__ __forceinline__ bool pml_tile_wait(uint32_t bar, uint32_t parity, int* status) {
    const bool ok = mbar_wait(bar, parity);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0 && threadIdx.y == 0) atomicOr(status, ST_TIMEOUT);
        mbar_wait(bar, parity);
        return false;
    }
    return true;
}

// pml_uvw in one tile of strip class C (fd3d_deriv.f90:1927-2293): one cell per thread.
template <class T, int C, bool SLAB>
__device__ __forceinline__ bool vel_pml_tile_c(const Grid& g, const Fields<T>& f, const PmlDesc& D,
                                               const PmlAux<T>& X, const StepConst<T>& c, int s, long long t0, T* sm,
                                               uint32_t bar, uint32_t parity, int* status) {
    constexpr int MX = split_mode(C, 0), MY = split_mode(C, 1), MZ = split_mode(C, 2);
    const int l = threadIdx.y * blockDim.x + threadIdx.x;
    T* gaux = X.vel + t0 * AUX_NV;
    pml_tile_begin(sm, gaux, AUX_NV, bar);
    int i = 0, j = 0, k = 0;
    const bool act = pml_cell<SLAB>(D, s, t0 + l, i, j, k);
    T d = 1, rl = 0, xx0 = 0, xx1 = 0, xy0 = 0, xy1 = 0, xz0 = 0, xz1 = 0, xz2 = 0, yz0 = 0, yz1 = 0, zz0 = 0, zz1 = 0;
    T xy2 = 0, yy0 = 0, yy1 = 0, yz2 = 0, vold = 0;
    Damp<T> ox{}, oxS{}, oy{}, oz{};
    long long p = 0;
    bool dov = false;
    const long long sy = g.px, sz = g.plane;
    if (act) {  // field loads overlap the staging copy
        const Strip& S = D.s[s];
        if (MX != SPLIT_NEVER) { ox = X.prof[S.ox_off + i - S.nxb]; oxS = X.prof[S.oxS_off + i - S.nxb]; }
        if (MY != SPLIT_NEVER) oy = X.prof[S.oy_off + j - S.nyb];
        if (MZ != SPLIT_NEVER) oz = X.prof[S.oz_off + k - S.nzb];
        p = g.at(i, j, k);
        dov = (j <= S.nye);
        if (f.lay) rl = f.lay[4 * g.nzt + k - 1];  // dt/d of the plane (1-D medium)
        else d = f.d[p];
        xx0 = f.xx[p]; xx1 = f.xx[p - 1]; xy0 = f.xy[p]; xy1 = f.xy[p - sy]; xz0 = f.xz[p]; xz1 = f.xz[p - sz];
        xz2 = f.xz[p + 1]; yz0 = f.yz[p]; yz1 = f.yz[p - sy]; zz0 = f.zz[p]; zz1 = f.zz[p + sz];
        if (dov) {
            xy2 = f.xy[p + 1]; yy0 = f.yy[p + sy]; yy1 = f.yy[p]; yz2 = f.yz[p - sz];
            if (j == g.nyt - 1) vold = f.v[p];
        }
    }
    if (!pml_tile_wait(bar, parity, status)) return false;
    // warp-uniform: does any cell of this warp lie where the direction is damped?
    const bool wx = MX == SPLIT_MAYBE && __any_sync(0xffffffffu, ox.o != (T)0 || oxS.o != (T)0);
    const bool wy = MY == SPLIT_MAYBE && __any_sync(0xffffffffu, oy.o != (T)0);
    if (act) {
        const T dt = c.dt, dh = c.dh, rdh = c.rdh;
        const T r = f.lay ? rl : dt / d;
        // p = (p*(1 - omega) + (dt/d)*diff/dh) / (1 + omega), every division rounded as IEEE.
        // The result goes straight back to the component's global slot (one coalesced
        // 128-byte row per warp and component), so no bulk store has to drain.
        auto inc = [&](T diff) { return div_pre(r * diff, dh, rdh); };
        auto put = [&](int comp, T a) { gaux[aux_sm(l, AUX_NV, comp)] = a; return a; };
        auto aux = [&](int comp) { return sm[aux_sm(l, AUX_NV, comp)]; };
        const T u0 = put(AX_U0, pml_split<T, MX>(aux(AX_U0), inc(xx0 - xx1), ox, wx));
        const T u1 = put(AX_U1, pml_split<T, MY>(aux(AX_U1), inc(xy0 - xy1), oy, wy));
        const T u2 = put(AX_U2, pml_split<T, MZ>(aux(AX_U2), inc(xz0 - xz1), oz, false));
        const T w0 = put(AX_W0, pml_split<T, MX>(aux(AX_W0), inc(xz2 - xz0), oxS, wx));
        const T w1 = put(AX_W1, pml_split<T, MY>(aux(AX_W1), inc(yz0 - yz1), oy, wy));
        const T w2 = put(AX_W2, pml_split<T, MZ>(aux(AX_W2), inc(zz1 - zz0), oz, false));
        f.u[p] = u0 + u1 + u2;
        f.w[p] = w0 + w1 + w2;
        if (dov) {
            const T v0 = put(AX_V0, pml_split<T, MX>(aux(AX_V0), inc(xy2 - xy0), oxS, wx));
            const T v1 = put(AX_V1, pml_split<T, MY>(aux(AX_V1), inc(yy0 - yy1), oy, wy));
            const T v2 = put(AX_V2, pml_split<T, MZ>(aux(AX_V2), inc(yz0 - yz2), oz, false));
            if (j == g.nyt - 1) f.v[p + sy] = vold;  // bnd2d mirror of the value before this update
            f.v[p] = v0 + v1 + v2;
        }
    }
    return true;
}

// pml_uvw: split-field PML velocity in the strips (fd3d_deriv.f90:1927-2293), one
// tile of PML_TILE consecutive cells per CTA of PML_TILE threads.  Returns false if the
// staging copy timed out.
template <class T, bool SLAB = false>
__device__ __forceinline__ bool vel_pml_tile(const Grid& g, const Fields<T>& f, const PmlDesc& D, const PmlAux<T>& X,
                                             const StepConst<T>& c, int tile, T* sm, uint32_t bar, uint32_t parity,
                                             int* status) {
    const long long t0 = (long long)tile * PML_TILE;
    const int s = pml_tile_strip(D, t0);
    switch (pml_class(s)) {
        case 0: return vel_pml_tile_c<T, 0, SLAB>(g, f, D, X, c, s, t0, sm, bar, parity, status);
        case 1: return vel_pml_tile_c<T, 1, SLAB>(g, f, D, X, c, s, t0, sm, bar, parity, status);
        default: return vel_pml_tile_c<T, 2, SLAB>(g, f, D, X, c, s, t0, sm, bar, parity, status);
    }
}

// fuvw at the ghost row k=ks+1 (fd3d_deriv.f90:1018-1062).  w needs u and v of the
// ghost row at (i+1,j) and (i,j-1); they are recomputed with the same formula
// (identical operands and order), so no second launch is needed.
template <class T>
__device__ __forceinline__ void vel_fs_body(Grid g, Fields<T> f, int bx_, int by_, int bz_) {
    const int i = 1 + bx_ * blockDim.x + threadIdx.x;
    const int j = 1 + by_ * blockDim.y + threadIdx.y;
    if (i > g.nxt || j > g.nyt) return;
    const int n = g.ks();
    const long long sy = g.px, sz = g.plane;
    auto ug = [&](int ii, int jj) -> T {  // loop 1: j=1..nyt, i=2..nxt-1
        const long long p = g.at(ii, jj, n);
        return f.u[p] - (f.w[p] - f.w[p - 1]);
    };
    auto vg = [&](int ii, int jj) -> T {  // loop 2: j=2..nyt-1, i=2..nxt-1; else existing value
        const long long p = g.at(ii, jj, n);
        if (jj >= 2 && jj <= g.nyt - 1 && ii >= 2 && ii <= g.nxt - 1) return f.v[p] - (f.w[p + sy] - f.w[p]);
        return f.v[p + sz];
    };
    T un = (T)0, vn = (T)0, wn = (T)0;
    const bool du = (i >= 2 && i <= g.nxt - 1);
    const bool dv = (j >= 2 && j <= g.nyt - 1 && du);
    const bool dw = (j >= 2 && i >= 2 && i <= g.nxt - 2);
    if (du) un = ug(i, j);
    if (dv) vn = vg(i, j);
    if (dw) {
        const long long p = g.at(i, j, n);
        const T xl = f.lam[p + sz], xm = f.mu[p + sz];
        const T a = (T)2 * xl, b = xl + (T)2 * xm;
        const T u_i1 = ug(i + 1, j);
        const T u_i = du ? un : f.u[p + sz];
        const T v_j = vg(i, j);
        const T v_jm = vg(i, j - 1);
        wn = +(f.w[p - sz] - (a / b) * (f.u[p + 1] - f.u[p] + u_i1 - u_i + f.v[p] - f.v[p - sy] + v_j - v_jm));
    }
    // The ghost-row values read above (v at j=1 and j=nyt) are never written by this
    // launch, so the writes below cannot race with them.
    const long long pg = g.at(i, j, n + 1);
    if (du) f.u[pg] = un;
    if (dv) f.v[pg] = vn;
    if (dw) f.w[pg] = wn;
}

// ---------------------------------------------------------------- stress
template <class T>
__global__ void __launch_bounds__(256) k_str_interior(Grid g, Fields<T> f, StepConst<T> c, int kchunk) {
    const int i = g.nabc + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = g.nabc + 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nxt - g.nabc || j > g.nyt - 2) return;
    const int kb = g.kin_lo() + blockIdx.z * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const long long sy = g.px, sz = g.plane;
    const T c1 = c.c1, c2 = c.c2, dth = c.dth;
    const T* __restrict__ u = f.u; const T* __restrict__ v = f.v; const T* __restrict__ w = f.w;
    const T* __restrict__ mu = f.mu;
    for (int k = kb; k <= ke; ++k) {
        const long long p = g.at(i, j, k);
        const T xl = f.lam[p], xm = mu[p];
        const T a = xl + (T)2 * xm, b = xl;
        const T dxu1 = c1 * (u[p + 1] - u[p]), dxu2 = c2 * (u[p + 2] - u[p - 1]);
        const T dyv1 = c1 * (v[p] - v[p - sy]), dyv2 = c2 * (v[p + sy] - v[p - 2 * sy]);
        const T dzw1 = c1 * (w[p] - w[p - sz]), dzw2 = c2 * (w[p + sz] - w[p - 2 * sz]);
        f.xx[p] = f.xx[p] + dth * a * (dxu1 + dxu2) + dth * b * (dyv1 + dyv2 + dzw1 + dzw2);
        f.yy[p] = f.yy[p] + dth * a * (dyv1 + dyv2) + dth * b * (dxu1 + dxu2 + dzw1 + dzw2);
        f.zz[p] = f.zz[p] + dth * a * (dzw1 + dzw2) + dth * b * (dxu1 + dxu2 + dyv1 + dyv2);
        T xmu = (T)0.5 * (xm + mu[p + sy]);
        f.xy[p] = f.xy[p] + dth * xmu * (c1 * (u[p + sy] - u[p]) + c2 * (u[p + 2 * sy] - u[p - sy]) +
                                         c1 * (v[p] - v[p - 1]) + c2 * (v[p + 1] - v[p - 2]));
        xmu = (T)0.5 * (xm + mu[p + sz]);
        f.xz[p] = f.xz[p] + dth * xmu * (c1 * (u[p + sz] - u[p]) + c2 * (u[p + 2 * sz] - u[p - sz]) +
                                         c1 * (w[p] - w[p - 1]) + c2 * (w[p + 1] - w[p - 2]));
        xmu = (T)0.5 * (xm + mu[p + 1 + sy + sz]);
        f.yz[p] = f.yz[p] + dth * xmu * (c1 * (v[p + sz] - v[p]) + c2 * (v[p + 2 * sz] - v[p - sz]) +
                                         c1 * (w[p + sy] - w[p]) + c2 * (w[p + 2 * sy] - w[p - sy]));
    }
}

// Band j=nyt-1 stresses (2nd order) + xy/yz mirror; sxz1 and tasii at j=nyt.
template <class T>
__device__ __forceinline__ void str_fault_body(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, int bx_, int by_, int bz_) {
    const int i = g.nabc + 1 + bx_ * blockDim.x + threadIdx.x;
    const int k = g.kin_lo() + by_ * blockDim.y + threadIdx.y;
    if (i > g.nxt - g.nabc || k > g.kin_hi()) return;
    const long long sy = g.px, sz = g.plane;
    const T dth = c.dth, dth2 = c.dth2, c1 = c.c1, c2 = c.c2;
    {   // sxx, sxy0, sxz0, syz0 at j=nyt-1 (fd3d_deriv.f90:818-1012)
        const long long p = g.at(i, g.nyt - 1, k);
        const T xl = f.lam[p], xm = f.mu[p];
        const T a = xl + (T)2 * xm, b = xl;
        const T up = f.u[p], vp = f.v[p], wp = f.w[p];
        const T ux = f.u[p + 1], vy = f.v[p - sy], wz = f.w[p - sz];
        f.xx[p] = f.xx[p] + dth * a * (ux - up) + dth * b * (vp - vy + wp - wz);
        f.yy[p] = f.yy[p] + dth * a * (vp - vy) + dth * b * (ux - up + wp - wz);
        f.zz[p] = f.zz[p] + dth * a * (wp - wz) + dth * b * (ux - up + vp - vy);
        T xmu = xm + f.mu[p + sy];
        const T xyn = f.xy[p] + dth2 * xmu * (f.u[p + sy] - up + vp - f.v[p - 1]);
        f.xy[p] = xyn; f.xy[p + sy] = xyn;
        xmu = xm + f.mu[p + sz];
        f.xz[p] = f.xz[p] + dth2 * xmu * (f.u[p + sz] - up + wp - f.w[p - 1]);
        xmu = xm + f.mu[p + 1 + sy + sz];
        const T yzn = f.yz[p] + dth2 * xmu * (f.v[p + sz] - vp + f.w[p + sy] - wp);
        f.yz[p] = yzn; f.yz[p + sy] = yzn;
    }
    {   // sxz1 (tasxz) and tasii at j=nyt (fd3d_deriv.f90:677-722, 1263-1314)
        const long long p = g.at(i, g.nyt, k);
        const T* u = f.u; const T* w = f.w;
        T xmu = f.mu[p] + f.mu[p + sz];
        f.xz[p] = f.xz[p] + dth2 * xmu * (c1 * (u[p + sz] - u[p]) + c2 * (u[p + 2 * sz] - u[p - sz]) +
                                          c1 * (w[p] - w[p - 1]) + c2 * (w[p + 1] - w[p - 2]));
        const T xl = f.lam[p], xm = f.mu[p];
        const T a = xl + (T)2 * xm, b = xl;
        const T diff1 = c1 * (u[p + 1] - u[p]) + c2 * (u[p + 2] - u[p - 1]);
        const T diff3 = c1 * (w[p] - w[p - sz]) + c2 * (w[p + sz] - w[p - 2 * sz]);
        const T vb = f.v[p - sy];
        const T v1t = vb - b * (diff1 + diff3) / ((T)2 * a);
        q.v1t[g.at2(i, k)] = v1t;
        const T dv = v1t - vb;
        f.xx[p] = f.xx[p] + dth * a * (diff1) + dth * b * ((T)2 * dv + diff3);
        f.yy[p] = f.yy[p] + dth * a * (T)2 * dv + dth * b * (diff1 + diff3);
        f.zz[p] = f.zz[p] + dth * a * (diff3) + dth * b * (diff1 + (T)2 * dv);
    }
}

// pml_xyz in one tile of strip class C (fd3d_deriv.f90:2304-3143), as vel_pml_tile_c
template <class T, int C, bool SLAB>
__device__ __forceinline__ bool str_pml_tile_c(const Grid& g, const Fields<T>& f, const PmlDesc& D,
                                               const PmlAux<T>& X, const StepConst<T>& c, int s, long long t0, T* sm,
                                               uint32_t bar, uint32_t parity, int* status) {
    constexpr int MX = split_mode(C, 0), MY = split_mode(C, 1), MZ = split_mode(C, 2);
    const int l = threadIdx.y * blockDim.x + threadIdx.x;
    T* gaux = X.str + t0 * AUX_NS;
    pml_tile_begin(sm, gaux, AUX_NS, bar);
    int i = 0, j = 0, k = 0;
    const bool act = pml_cell<SLAB>(D, s, t0 + l, i, j, k);
    long long p = 0;
    bool dxy = false, top = false;
    const long long sy = g.px, sz = g.plane;
    T xl = 0, xm = 0, mz = 0, up = 0, ux = 0, uz = 0, vp = 0, vy = 0, wp = 0, wz = 0, wx = 0;
    T my = 0, md = 0, uy = 0, vx = 0, vz = 0, wy = 0, xyo = 0, yzo = 0;
    // xy and yz take omegayS in strips 3-5 and xz, yz omegazS in strips 4-5; in the other
    // strips those directions are undamped (SPLIT_NEVER), so oyS / ozS serve every class
    Damp<T> ox{}, oxS{}, oy{}, oyS{}, oz{}, ozS{};
    if (act) {  // field loads overlap the staging copy
        const Strip& S = D.s[s];
        const int i2 = i - S.nxb, j2 = j - S.nyb, k2 = k - S.nzb;
        if (MX != SPLIT_NEVER) { ox = X.prof[S.ox_off + i2]; oxS = X.prof[S.oxS_off + i2]; }
        if (MY != SPLIT_NEVER) { oy = X.prof[S.oy_off + j2]; oyS = X.prof[S.oyS_off + j2]; }
        if (MZ != SPLIT_NEVER) { oz = X.prof[S.oz_off + k2]; ozS = X.prof[S.ozS_off + k2]; }
        p = g.at(i, j, k);
        dxy = (j <= S.nye);
        top = !g.fspace && (C <= 1) && (k == S.nze);  // xz/yz aux zeroed at the top row, strips 1-3 (not FSPACE)
        if (f.lay) {  // 1-D medium: mu(i,j+1,k) = mu(i,j,k), mu(i+1,j+1,k+1) = mu(i,j,k+1)
            xl = f.lay[k - 1]; xm = f.lay[g.nzt + k - 1]; mz = f.lay[g.nzt + k];
        } else {
            xl = f.lam[p]; xm = f.mu[p]; mz = f.mu[p + sz];
        }
        up = f.u[p]; ux = f.u[p + 1]; uz = f.u[p + sz];
        vp = f.v[p]; vy = f.v[p - sy];
        wp = f.w[p]; wz = f.w[p - sz]; wx = f.w[p - 1];
        if (dxy) {
            if (f.lay) { my = xm; md = mz; }
            else { my = f.mu[p + sy]; md = f.mu[p + 1 + sy + sz]; }
            uy = f.u[p + sy]; vx = f.v[p - 1]; vz = f.v[p + sz]; wy = f.w[p + sy];
        }
    }
    if (!pml_tile_wait(bar, parity, status)) return false;
    const bool dx = MX == SPLIT_MAYBE && __any_sync(0xffffffffu, ox.o != (T)0 || oxS.o != (T)0);
    const bool dy = MY == SPLIT_MAYBE && __any_sync(0xffffffffu, oy.o != (T)0 || oyS.o != (T)0);
    if (act) {
        const T dt = c.dt, dh = c.dh, rdh = c.rdh;
        const T a = xl + (T)2 * xm, b = xl;
        const T diff1 = ux - up, diff2 = vp - vy, diff3 = wp - wz;
        // p = (p*(1 - omega) + dt*modulus*diff/dh) / (1 + omega), every division rounded as IEEE
        auto inc = [&](T mod, T diff) { return div_pre(dt * mod * diff, dh, rdh); };
        auto aux = [&](int comp) { return sm[aux_sm(l, AUX_NS, comp - AUX_NV)]; };
        auto put = [&](int comp, T v) { gaux[aux_sm(l, AUX_NS, comp - AUX_NV)] = v; return v; };
        const T x0 = put(AX_XX0, pml_split<T, MX>(aux(AX_XX0), inc(a, diff1), oxS, dx));
        const T x1 = put(AX_XX1, pml_split<T, MY>(aux(AX_XX1), inc(b, diff2), oy, dy));
        const T x2 = put(AX_XX2, pml_split<T, MZ>(aux(AX_XX2), inc(b, diff3), oz, false));
        f.xx[p] = x0 + x1 + x2;
        const T y0 = put(AX_YY0, pml_split<T, MX>(aux(AX_YY0), inc(b, diff1), oxS, dx));
        const T y1 = put(AX_YY1, pml_split<T, MY>(aux(AX_YY1), inc(a, diff2), oy, dy));
        const T y2 = put(AX_YY2, pml_split<T, MZ>(aux(AX_YY2), inc(b, diff3), oz, false));
        f.yy[p] = y0 + y1 + y2;
        const T z0 = put(AX_ZZ0, pml_split<T, MX>(aux(AX_ZZ0), inc(b, diff1), oxS, dx));
        const T z1 = put(AX_ZZ1, pml_split<T, MY>(aux(AX_ZZ1), inc(b, diff2), oy, dy));
        const T z2 = put(AX_ZZ2, pml_split<T, MZ>(aux(AX_ZZ2), inc(a, diff3), oz, false));
        f.zz[p] = z0 + z1 + z2;
        {   // xz (j up to jend_uw)
            const T xmu = (xm + mz) / (T)2;
            const T q0 = put(AX_XZ0, pml_split<T, MZ>(aux(AX_XZ0), inc(xmu, uz - up), ozS, false));
            const T q1 = put(AX_XZ1, pml_split<T, MX>(aux(AX_XZ1), inc(xmu, wp - wx), ox, dx));
            f.xz[p] = q0 + q1;
            if (top) { put(AX_XZ0, (T)0); put(AX_XZ1, (T)0); }
        }
        if (dxy) {
            T xmu = (xm + my) / (T)2;
            const T e0 = put(AX_XY0, pml_split<T, MY>(aux(AX_XY0), inc(xmu, uy - up), oyS, dy));
            const T e1 = put(AX_XY1, pml_split<T, MX>(aux(AX_XY1), inc(xmu, vp - vx), ox, dx));
            xmu = (xm + md) / (T)2;
            const T h0 = put(AX_YZ0, pml_split<T, MZ>(aux(AX_YZ0), inc(xmu, vz - vp), ozS, false));
            const T h1 = put(AX_YZ1, pml_split<T, MY>(aux(AX_YZ1), inc(xmu, wy - wp), oyS, dy));
            if (j == g.nyt - 1) {  // strbnd mirror of the values before this update (read here, not
                xyo = f.xy[p];     // held across the staging wait: four fewer live registers)
                yzo = f.yz[p];
                f.xy[p + sy] = xyo;
                f.yz[p + sy] = yzo;
            }
            f.xy[p] = e0 + e1;
            f.yz[p] = h0 + h1;
            if (top) { put(AX_YZ0, (T)0); put(AX_YZ1, (T)0); }
        }
    }
    return true;
}

// pml_xyz in the strips (fd3d_deriv.f90:2304-3143), one tile per CTA as vel_pml_tile
template <class T, bool SLAB = false>
__device__ __forceinline__ bool str_pml_tile(const Grid& g, const Fields<T>& f, const PmlDesc& D, const PmlAux<T>& X,
                                             const StepConst<T>& c, int tile, T* sm, uint32_t bar, uint32_t parity,
                                             int* status) {
    const long long t0 = (long long)tile * PML_TILE;
    const int s = pml_tile_strip(D, t0);
    switch (pml_class(s)) {
        case 0: return str_pml_tile_c<T, 0, SLAB>(g, f, D, X, c, s, t0, sm, bar, parity, status);
        case 1: return str_pml_tile_c<T, 1, SLAB>(g, f, D, X, c, s, t0, sm, bar, parity, status);
        default: return str_pml_tile_c<T, 2, SLAB>(g, f, D, X, c, s, t0, sm, bar, parity, status);
    }
}

// fres (fd3d_deriv.f90:1067-1104)
template <class T>
__device__ __forceinline__ void str_fs_body(Grid g, Fields<T> f, int bx_, int by_, int bz_) {
    const int i = 1 + bx_ * blockDim.x + threadIdx.x;
    const int j = 1 + by_ * blockDim.y + threadIdx.y;
    if (i > g.nxt || j > g.nyt) return;
    const long long p = g.at(i, j, g.ks()), sz = g.plane;
    f.zz[p + sz] = -f.zz[p];
    f.zz[p + 2 * sz] = -f.zz[p - sz];
    f.xz[p + sz] = -f.xz[p - sz];
    f.xz[p + 2 * sz] = -f.xz[p - 2 * sz];
    f.yz[p + sz] = -f.yz[p - sz];
    f.yz[p + 2 * sz] = -f.yz[p - 2 * sz];
    f.xz[p] = (T)0;
    f.yz[p] = (T)0;
}

// ---------------------------------------------------------------- fault BC
// trial traction, damping, RF (fd3d_theo.f90:233-308).  Under FSPACE the top row k = ks
// takes the interior formula and no ghost row is written (fd3d_theo.f90:260-283).
template <class T>
__device__ __forceinline__ void traction_body(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, const int* it_dev,
                                              int bx_, int by_, int bz_) {
    const int i = g.nabc + 1 + bx_ * blockDim.x + threadIdx.x;
    const int k = g.kin_lo() + by_ * blockDim.y + threadIdx.y;
    const int ks = g.ks();
    if (i > g.nxt - g.nabc || k > g.kin_hi()) return;
    const long long sy = g.px, sz = g.plane;
    const long long p = g.at(i, g.nyt, k);
    const int n2 = g.at2(i, k);
    const T c1 = c.c1, c2 = c.c2, dht = c.dht, ds = c.damp_s;
    const T* xx = f.xx; const T* xz = f.xz; const T* zz = f.zz;
    const int it = *it_dev;
    const T* avdz_rd = pp_rd(q.avdz, it, q.n2); T* avdz_wr = pp_wr(q.avdz, it, q.n2);
    const T* avdx_rd = pp_rd(q.avdx, it, q.n2); T* avdx_wr = pp_wr(q.avdx, it, q.n2);
    const bool inner = (k < ks) || g.fspace;
    T pdz;
    if (inner)
        pdz = (c1 * (xz[p + 1] - xz[p]) + c2 * (xz[p + 2] - xz[p - 1])) / (T)2 +
              (c1 * (zz[p + sz] - zz[p]) + c2 * (zz[p + 2 * sz] - zz[p - sz])) / (T)2 - f.yz[p - sy];
    else
        pdz = ((xz[p + 1 - sz] - xz[p - sz]) / ((T)2 * (T)4) + (zz[p + sz] - zz[p]) / ((T)2 * (T)2) -
               f.yz[p - sy - sz] / (T)4);
    T av = ds * (pdz - avdz_rd[n2]);
    T rf = pdz + av;
    q.RFz[n2] = rf;
    T tzv;
    if (inner) tzv = -rf - (T)0.5 * f.d[p] * dht * f.w[p];
    else        tzv = -rf - (T)0.5 * f.d[p] * dht * f.w[p] / (T)2;
    q.tzt[n2] = tzv;
    avdz_wr[n2] = pdz;
    const T pdx = (c1 * (xx[p] - xx[p - 1]) + c2 * (xx[p + 1] - xx[p - 2])) / (T)2 +
                  (c1 * (xz[p] - xz[p - sz]) + c2 * (xz[p + sz] - xz[p - 2 * sz])) / (T)2 - f.xy[p - sy];
    av = ds * (pdx - avdx_rd[n2]);
    rf = pdx + av;
    q.RFx[n2] = rf;
    const T txv = -rf - (T)0.5 * f.d[p] * dht * f.u[p];
    q.txt[n2] = txv;
    avdx_wr[n2] = pdx;
    // ghost row nzt-1 (fd3d_theo.f90:304-307); with nfs=2: nzt-1 = ks+1, nzt-2 = ks, nzt-3 = ks-1
    if (!g.fspace && k == ks) q.txt[g.at2(i, ks + 1)] = +txv;
    if (!g.fspace && k == ks - 1) q.tzt[g.at2(i, ks + 1)] = -tzv;
}

// |T| at staggered nodes, friction law, slip, rupture time (fd3d_theo.f90:313-410)
template <class T>
__device__ __forceinline__ void friction_body(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, int law, FvwScalars s,
                           const int* it_dev, int bx_, int by_, int bz_) {
    const int i = g.nabc + 1 + bx_ * blockDim.x + threadIdx.x;
    const int k = g.kin_lo() + by_ * blockDim.y + threadIdx.y;
    if (i > g.nxt - g.nabc || k > g.kin_hi()) return;
    const int it = *it_dev;
    const double time = (double)it * c.dtA;
    const double* distX_rd = pp_rd(q.distX, it, q.n2);
    double* distX_wr = pp_wr(q.distX, it, q.n2);
    const double dtA = c.dtA, rup = 1.e-3;
    const long long sy = g.px, sz = g.plane;
    (void)sy;
    const int n2 = g.at2(i, k);
    const int e1 = g.at2(i + 1, k), e2 = g.at2(i, k + 1), e3 = g.at2(i + 1, k + 1);
    const int w1i = g.at2(i - 1, k), w2i = g.at2(i, k - 1), w3i = g.at2(i - 1, k - 1);
    const T* txt = q.txt; const T* tzt = q.tzt; const T* T0X = q.T0X; const T* T0Z = q.T0Z;
    T tint = (txt[n2] + T0X[n2] + txt[e1] + T0X[e1] + txt[e2] + T0X[e2] + txt[e3] + T0X[e3]) / (T)4;
    const T szv = tzt[n2] + T0Z[n2];
    const T tabsZ = sqrt(tint * tint + szv * szv);
    tint = (tzt[n2] + T0Z[n2] + tzt[w1i] + T0Z[w1i] + tzt[w2i] + T0Z[w2i] + tzt[w3i] + T0Z[w3i]) / (T)4;
    const T sxv = txt[n2] + T0X[n2];
    const T tabsX = sqrt(sxv * sxv + tint * tint);
    q.tabsZ[n2] = tabsZ;
    q.tabsX[n2] = tabsX;
    const long long p = g.at(i, g.nyt, k);
    const T U = f.u[p], W = f.w[p];
    // Z nodes (fd3d_theo.f90:326-373)
    {
        const T uZ = (U + f.u[p + 1] + f.u[p + sz] + f.u[p + 1 + sz]) / (T)4;
        q.uZ[n2] = uZ;
        const T u1out = -sqrt(W * W + uZ * uZ);
        T tzn = tzt[n2];
        if (law == 1) {
            const double a = (double)q.aZ[n2];
            const double s1 = 2.0 * (fabs((double)W) + fabs(s.wini)), s2 = 2.0 * (fabs((double)uZ) + fabs(s.uini));
            const double sr = sqrt(s1 * s1 + s2 * s2);
            const double flv = s.f0 - ((double)q.bZ[n2] - a) * log(sr / s.v0);
            const double fw = (double)q.fwZ[n2];
            const double fss = fw + (flv - fw) / pow(1.0 + pow(sr / (double)q.vwZ[n2], 8.0), 1.0 / 8.0);
            const double psiss = a * (log(sinh(fss / a)) + log(2.0 * s.v0 / sr));
            const double psi = (q.psiZ[n2] - psiss) * exp(-sr * dtA / (double)q.Dc[n2]) + psiss;
            q.psiZ[n2] = psi;
            const double fric = s.Sn * a * asinh(sr * exp(psi / a) / (2.0 * s.v0));
            q.distZ[n2] = q.distZ[n2] - 2.0 * (double)u1out * dtA;
            q.schangeZ[n2] = (T)fric;
            if (fabs(2.0 * (double)u1out) > rup) {
                if (q.ruptime[n2] != 1.e4) q.rise[n2] = time;
                if (q.ruptime[n2] == 1.e4) q.ruptime[n2] = time;
            }
        } else {
            const double dz = q.distZ[n2], dcz = (double)q.DcZ[n2];
            double fric;
            if (dz <= dcz) fric = (double)q.peakZ[n2] * (1.0 - dz / dcz) + (double)q.dynZ[n2] * dz / dcz + (double)q.coh[n2];
            else           fric = (double)q.dynZ[n2] + (double)q.coh[n2];
            if ((double)tabsZ >= fric) {
                q.distZ[n2] = dz - 2.0 * (double)u1out * dtA;
                tzn = (T)(((double)tzn + (double)T0Z[n2]) * fric / (double)tabsZ - (double)T0Z[n2]);
                if (-2.0 * (double)u1out > rup) {
                    if (q.ruptime[n2] != 1.e4) q.rise[n2] = time;
                    if (q.ruptime[n2] == 1.e4) q.ruptime[n2] = time;
                }
            }
        }
        q.tz[n2] = tzn;
        q.slipZ[n2] = q.slipZ[n2] - 2.0 * (double)W * dtA;
        q.slipX[n2] = q.slipX[n2] - 2.0 * (double)uZ * dtA;
        if (q.sliptime[n2] == 1.e4 && q.distZ[n2] > (double)q.Dc[n2]) q.sliptime[n2] = time;
    }
    // X nodes (fd3d_theo.f90:375-410)
    {
        const T wX = (W + f.w[p - 1] + f.w[p - sz] + f.w[p - 1 - sz]) / (T)4;
        q.wX[n2] = wX;
        const T u1out = -sqrt(wX * wX + U * U);
        T txn = txt[n2];
        if (law == 1) {
            const double a = (double)q.aX[n2];
            const double s1 = 2.0 * (fabs((double)wX) + fabs(s.wini)), s2 = 2.0 * (fabs((double)U) + fabs(s.uini));
            const double sr = sqrt(s1 * s1 + s2 * s2);
            const double flv = s.f0 - ((double)q.bX[n2] - a) * log(sr / s.v0);
            const double fw = (double)q.fwX[n2];
            const double fss = fw + (flv - fw) / pow(1.0 + pow(sr / (double)q.vwX[n2], 8.0), 1.0 / 8.0);
            const double psiss = a * (log(sinh(fss / a)) + log(2.0 * s.v0 / sr));
            const double psi = (q.psiX[n2] - psiss) * exp(-sr * dtA / (double)q.Dc[n2]) + psiss;
            q.psiX[n2] = psi;
            const double fric = s.Sn * a * asinh(sr * exp(psi / a) / (2.0 * s.v0));
            distX_wr[n2] = distX_rd[n2] - 2.0 * (double)u1out * dtA;
            q.schangeX[n2] = (T)fric;
        } else {
            const double dx = distX_rd[n2], dcx = (double)q.DcX[n2];
            double fric;
            if (dx <= (double)q.Dc[n2]) fric = (double)q.peakX[n2] * (1.0 - dx / dcx) + (double)q.dynX[n2] * dx / dcx + (double)q.coh[n2];
            else                        fric = (double)q.dynX[n2] + (double)q.coh[n2];
            if ((double)tabsX >= fric) {
                distX_wr[n2] = dx - 2.0 * (double)u1out * dtA;
                txn = (T)(((double)txn + (double)T0X[n2]) * fric / (double)tabsX - (double)T0X[n2]);
            } else {
                distX_wr[n2] = dx;  // carried into this step's plane
            }
        }
        q.tx[n2] = txn;
    }
    if (k == g.ks()) {  // the reference's tx/tz arrays also carry the ghost row nzt-1
        const int gh = g.at2(i, k + 1);
        q.tx[gh] = txt[gh];
        q.tz[gh] = tzt[gh];
    }
}

struct HistDesc {
    void* ring;         // [cap][nf][nzT][nxT] of T
    int cap, stride, nf;
    int nst;
    int sta[3 * 10];    // station (i,j,k)
    void* seis;         // [cap][nst*3] of T
};

// output planes, stations, history ring (fd3d_theo.f90:413-467); non-finite check
template <class T>
__device__ __forceinline__ void output_body(Grid g, Fields<T> f, Fault<T> q, int law, const int* it_dev, const HistDesc& h, int* status, int bx_, int by_, int bz_) {
    const int ii = bx_ * blockDim.x + threadIdx.x;
    const int kk = by_ * blockDim.y + threadIdx.y;
    const int it = *it_dev;
    const bool rec = (it % h.stride) == 0;
    const long long slot = (long long)((it / h.stride - 1) % h.cap);
    const int nxT = g.nxt - 2 * g.nabc, nzT = g.ks() - g.nabc;
    if (rec && ii < h.nst && kk == 0 && g.owns(h.sta[3 * ii + 2])) {
        const long long p = g.at(h.sta[3 * ii], h.sta[3 * ii + 1], h.sta[3 * ii + 2]);
        T* sp = (T*)h.seis + slot * (3 * h.nst) + 3 * ii;
        sp[0] = f.u[p]; sp[1] = f.v[p]; sp[2] = f.w[p];
    }
    const int i = g.nabc + 1 + ii, k = g.kin_lo() + kk;
    if (ii >= nxT || k > g.kin_hi()) return;
    const bool top = (k == g.ks());
    const long long p = g.at(i, g.nyt, k), sz = g.plane;
    const int n2 = g.at2(i, k), e1 = g.at2(i + 1, k), e2 = g.at2(i, k + 1), e3 = g.at2(i + 1, k + 1);
    const T U = f.u[p], U2 = f.u[p + 1], W = f.w[p];
    T srx, srz, scx, scz;
    srz = (T)-2 * W;
    if (!top) {
        const T U3 = f.u[p + sz], U4 = f.u[p + 1 + sz];
        srx = ((T)-2 * U - (T)2 * U2 - (T)2 * U3 - (T)2 * U4) / (T)4;
        if (law == 0) {
            scz = q.tz[n2] + q.T0Z[n2];
            scx = (q.tx[n2] + q.T0X[n2] + q.tx[e1] + q.T0X[e1] + q.tx[e2] + q.T0X[e2] + q.tx[e3] + q.T0X[e3]) / (T)4;
        }
    } else {
        if (law == 1) {
            srx = ((T)-2 * U - (T)2 * U2) / (T)4;
        } else {
            scz = q.tz[n2] + q.T0Z[n2];
            scx = (q.tx[n2] + q.T0X[n2] + q.tx[e1] + q.T0X[e1]) / (T)2;
            srx = ((T)-2 * U - (T)2 * U2) / (T)2;
        }
    }
    if (law == 1) { scx = q.schangeX[n2]; scz = q.schangeZ[n2]; }
    else { q.schangeX[n2] = scx; q.schangeZ[n2] = scz; }
    if (!(isfinite((double)srx) && isfinite((double)srz) && isfinite((double)scx) && isfinite((double)scz)))
        atomicOr(status, ST_NONFINITE);
    if (rec) {
        const long long plane = (long long)nxT * nzT;
        T* r = (T*)h.ring + slot * h.nf * plane + (long long)(k - g.nabc - 1) * nxT + ii;
        r[0] = srx;
        r[plane] = srz;
        r[2 * plane] = scx;
        r[3 * plane] = scz;
        if (h.nf > 4) r[4 * plane] = (T)q.psiZ[n2];
    }
}

// ---------------------------------------------------------------- fused fault BC
// The fault boundary condition of one step in one launch (fd3d_theo.f90:225-467): fres, the
// trial traction, |T| at the staggered nodes, the friction law with slip and rupture time,
// and the output planes.  A CTA owns a FBC_TX x FBC_TZ tile of fault nodes and computes the
// trial tractions of the tile and a one-node ring around it, and the post-friction
// tractions of the X nodes of the tile plus one column and one row beyond, into shared
// memory; the ring values it only reads, so the state it needs from neighbouring nodes is
// the state before this step (the two-plane avdx, avdz and distX of Fault) and nothing
// another CTA writes in the same launch.  fres runs in separate CTAs of the same launch:
// the three stresses it writes that the trial traction reads (zz at ks+1, xz at ks and
// ks+1, fd3d_deriv.f90:1087-1102) are formed from the values fres reads, with the same
// operation (a negation, or the zero it stores).
constexpr int FBC_TX = 32, FBC_TZ = 8;                   // owned nodes of a tile (CTA of 32 x 8 threads)
constexpr int FBC_HX = FBC_TX + 2, FBC_HZ = FBC_TZ + 2;  // trial tractions: the tile and a one-node ring
constexpr int FBC_PX = FBC_TX + 1, FBC_PZ = FBC_TZ + 1;  // post-friction X-node tractions: tile + 1 in +i, +k
constexpr int FBC_SMEM = 2 * FBC_HX * FBC_HZ + FBC_PX * FBC_PZ;  // elements of T

template <class T>
struct TrialTraction { T pdz, pdx, rfz, rfx, tzv, txv; };

// trial traction at fault node (i,k) (fd3d_theo.f90:233-308), in the operation order of
// traction_body; VIRT: fres has not run yet, its stores are formed here
template <class T, bool VIRT>
__device__ __forceinline__ TrialTraction<T> trial_traction(const Grid& g, const Fields<T>& f, const StepConst<T>& c,
                                                           const T* avdz_rd, const T* avdx_rd, int i, int k) {
    const int ks = g.ks();
    const bool virt = VIRT && !g.fspace;
    const long long sy = g.px;
    auto XZ = [&](int ii, int kk) -> T {
        if (virt && kk == ks) return (T)0;                                 // xz(i,nyt,nzt-nfs) = 0
        if (virt && kk == ks + 1) return -f.xz[g.at(ii, g.nyt, ks - 1)];   // xz(ks+1) = -xz(ks-1)
        return f.xz[g.at(ii, g.nyt, kk)];
    };
    auto ZZ = [&](int kk) -> T {
        if (virt && kk == ks + 1) return -f.zz[g.at(i, g.nyt, ks)];        // zz(ks+1) = -zz(ks)
        return f.zz[g.at(i, g.nyt, kk)];
    };
    const long long p = g.at(i, g.nyt, k);
    const int n2 = g.at2(i, k);
    const T c1 = c.c1, c2 = c.c2, dht = c.dht, ds = c.damp_s;
    const T* xx = f.xx;
    const bool inner = (k < ks) || g.fspace;
    TrialTraction<T> t;
    if (inner)
        t.pdz = (c1 * (XZ(i + 1, k) - XZ(i, k)) + c2 * (XZ(i + 2, k) - XZ(i - 1, k))) / (T)2 +
                (c1 * (ZZ(k + 1) - ZZ(k)) + c2 * (ZZ(k + 2) - ZZ(k - 1))) / (T)2 - f.yz[p - sy];
    else
        t.pdz = ((XZ(i + 1, k - 1) - XZ(i, k - 1)) / ((T)2 * (T)4) + (ZZ(k + 1) - ZZ(k)) / ((T)2 * (T)2) -
                 f.yz[p - sy - g.plane] / (T)4);
    T av = ds * (t.pdz - avdz_rd[n2]);
    t.rfz = t.pdz + av;
    if (inner) t.tzv = -t.rfz - (T)0.5 * f.d[p] * dht * f.w[p];
    else       t.tzv = -t.rfz - (T)0.5 * f.d[p] * dht * f.w[p] / (T)2;
    t.pdx = (c1 * (xx[p] - xx[p - 1]) + c2 * (xx[p + 1] - xx[p - 2])) / (T)2 +
            (c1 * (XZ(i, k) - XZ(i, k - 1)) + c2 * (XZ(i, k + 1) - XZ(i, k - 2))) / (T)2 - f.xy[p - sy];
    av = ds * (t.pdx - avdx_rd[n2]);
    t.rfx = t.pdx + av;
    t.txv = -t.rfx - (T)0.5 * f.d[p] * dht * f.u[p];
    return t;
}

// Friction at the X node (i,k) (fd3d_theo.f90:375-410) from trial tractions in shared
// memory: returns the traction after friction; OWN: also the node's state (tabsX, wX,
// slip path, psi, strength).
template <class T, bool OWN>
__device__ __forceinline__ T friction_x(const Grid& g, const Fields<T>& f, const Fault<T>& q, const StepConst<T>& c,
                                        int law, const FvwScalars& s, const double* distX_rd, double* distX_wr,
                                        T txt0, T tint, int i, int k) {
    const int n2 = g.at2(i, k);
    const double dtA = c.dtA;
    const long long sz = g.plane;
    const T sxv = txt0 + q.T0X[n2];
    const T tabsX = sqrt(sxv * sxv + tint * tint);
    const long long p = g.at(i, g.nyt, k);
    const T U = f.u[p], W = f.w[p];
    const T wX = (W + f.w[p - 1] + f.w[p - sz] + f.w[p - 1 - sz]) / (T)4;
    const T u1out = -sqrt(wX * wX + U * U);
    T txn = txt0;
    if (OWN) { q.tabsX[n2] = tabsX; q.wX[n2] = wX; }
    if (law == 1) {
        if (OWN) {
            const double a = (double)q.aX[n2];
            const double s1 = 2.0 * (fabs((double)wX) + fabs(s.wini)), s2 = 2.0 * (fabs((double)U) + fabs(s.uini));
            const double sr = sqrt(s1 * s1 + s2 * s2);
            const double flv = s.f0 - ((double)q.bX[n2] - a) * log(sr / s.v0);
            const double fw = (double)q.fwX[n2];
            const double fss = fw + (flv - fw) / pow(1.0 + pow(sr / (double)q.vwX[n2], 8.0), 1.0 / 8.0);
            const double psiss = a * (log(sinh(fss / a)) + log(2.0 * s.v0 / sr));
            const double psi = (q.psiX[n2] - psiss) * exp(-sr * dtA / (double)q.Dc[n2]) + psiss;
            q.psiX[n2] = psi;
            const double fric = s.Sn * a * asinh(sr * exp(psi / a) / (2.0 * s.v0));
            distX_wr[n2] = distX_rd[n2] - 2.0 * (double)u1out * dtA;
            q.schangeX[n2] = (T)fric;
        }
    } else {
        const double dx = distX_rd[n2], dcx = (double)q.DcX[n2];
        double fric;
        if (dx <= (double)q.Dc[n2]) fric = (double)q.peakX[n2] * (1.0 - dx / dcx) + (double)q.dynX[n2] * dx / dcx + (double)q.coh[n2];
        else                        fric = (double)q.dynX[n2] + (double)q.coh[n2];
        double dnew = dx;
        if ((double)tabsX >= fric) {
            dnew = dx - 2.0 * (double)u1out * dtA;
            txn = (T)(((double)txn + (double)q.T0X[n2]) * fric / (double)tabsX - (double)q.T0X[n2]);
        }
        if (OWN) distX_wr[n2] = dnew;
    }
    if (OWN) q.tx[n2] = txn;
    return txn;
}

// Friction at the Z node (i,k) (fd3d_theo.f90:326-373): state, slip, rupture time; returns tz.
template <class T>
__device__ __forceinline__ T friction_z(const Grid& g, const Fields<T>& f, const Fault<T>& q, const StepConst<T>& c,
                                        int law, const FvwScalars& s, double time, T tzt0, T tint, int i, int k) {
    const int n2 = g.at2(i, k);
    const double dtA = c.dtA, rup = 1.e-3;
    const long long sz = g.plane;
    const T* T0Z = q.T0Z;
    const T szv = tzt0 + T0Z[n2];
    const T tabsZ = sqrt(tint * tint + szv * szv);
    q.tabsZ[n2] = tabsZ;
    const long long p = g.at(i, g.nyt, k);
    const T U = f.u[p], W = f.w[p];
    const T uZ = (U + f.u[p + 1] + f.u[p + sz] + f.u[p + 1 + sz]) / (T)4;
    q.uZ[n2] = uZ;
    const T u1out = -sqrt(W * W + uZ * uZ);
    T tzn = tzt0;
    if (law == 1) {
        const double a = (double)q.aZ[n2];
        const double s1 = 2.0 * (fabs((double)W) + fabs(s.wini)), s2 = 2.0 * (fabs((double)uZ) + fabs(s.uini));
        const double sr = sqrt(s1 * s1 + s2 * s2);
        const double flv = s.f0 - ((double)q.bZ[n2] - a) * log(sr / s.v0);
        const double fw = (double)q.fwZ[n2];
        const double fss = fw + (flv - fw) / pow(1.0 + pow(sr / (double)q.vwZ[n2], 8.0), 1.0 / 8.0);
        const double psiss = a * (log(sinh(fss / a)) + log(2.0 * s.v0 / sr));
        const double psi = (q.psiZ[n2] - psiss) * exp(-sr * dtA / (double)q.Dc[n2]) + psiss;
        q.psiZ[n2] = psi;
        const double fric = s.Sn * a * asinh(sr * exp(psi / a) / (2.0 * s.v0));
        q.distZ[n2] = q.distZ[n2] - 2.0 * (double)u1out * dtA;
        q.schangeZ[n2] = (T)fric;
        if (fabs(2.0 * (double)u1out) > rup) {
            if (q.ruptime[n2] != 1.e4) q.rise[n2] = time;
            if (q.ruptime[n2] == 1.e4) q.ruptime[n2] = time;
        }
    } else {
        const double dz = q.distZ[n2], dcz = (double)q.DcZ[n2];
        double fric;
        if (dz <= dcz) fric = (double)q.peakZ[n2] * (1.0 - dz / dcz) + (double)q.dynZ[n2] * dz / dcz + (double)q.coh[n2];
        else           fric = (double)q.dynZ[n2] + (double)q.coh[n2];
        if ((double)tabsZ >= fric) {
            q.distZ[n2] = dz - 2.0 * (double)u1out * dtA;
            tzn = (T)(((double)tzn + (double)T0Z[n2]) * fric / (double)tabsZ - (double)T0Z[n2]);
            if (-2.0 * (double)u1out > rup) {
                if (q.ruptime[n2] != 1.e4) q.rise[n2] = time;
                if (q.ruptime[n2] == 1.e4) q.ruptime[n2] = time;
            }
        }
    }
    q.tz[n2] = tzn;
    q.slipZ[n2] = q.slipZ[n2] - 2.0 * (double)W * dtA;
    q.slipX[n2] = q.slipX[n2] - 2.0 * (double)uZ * dtA;
    if (q.sliptime[n2] == 1.e4 && q.distZ[n2] > (double)q.Dc[n2]) q.sliptime[n2] = time;
    return tzn;
}

// One tile of the fused fault boundary condition (without fres).  A CTA of 32 x 8 threads;
// sm holds FBC_SMEM elements.
template <class T>
__device__ __forceinline__ void fault_bc_body(const Grid& g, const Fields<T>& f, const Fault<T>& q,
                                              const StepConst<T>& c, int law, const FvwScalars& s, const int* it_dev,
                                              const HistDesc& h, int* status, int bx_, int by_, T* sm) {
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int i0 = g.nabc + 1 + bx_ * FBC_TX, k0 = g.nabc + 1 + by_ * FBC_TZ;
    const int ie = g.nxt - g.nabc, ks = g.ks();
    const int it = *it_dev;
    const T* avdz_rd = pp_rd(q.avdz, it, q.n2); T* avdz_wr = pp_wr(q.avdz, it, q.n2);
    const T* avdx_rd = pp_rd(q.avdx, it, q.n2); T* avdx_wr = pp_wr(q.avdx, it, q.n2);
    const double* distX_rd = pp_rd(q.distX, it, q.n2); double* distX_wr = pp_wr(q.distX, it, q.n2);
    T* s_txt = sm;                        // [FBC_HZ][FBC_HX], node (i,k) at (i-i0+1) + (k-k0+1)*FBC_HX
    T* s_tzt = sm + FBC_HX * FBC_HZ;
    T* s_tx = sm + 2 * FBC_HX * FBC_HZ;   // [FBC_PZ][FBC_PX], node (i,k) at (i-i0) + (k-k0)*FBC_PX
    __syncthreads();                      // the shared memory may hold the previous item's values

    // 1. trial tractions of the tile and its ring; the owner stores a node's state
    for (int n = tid; n < FBC_HX * FBC_HZ; n += 256) {
        const int ri = n % FBC_HX, rk = n / FBC_HX;
        const int i = i0 - 1 + ri, k = k0 - 1 + rk;
        T tx_ = 0, tz_ = 0;   // outside the traction loops the reference's tx, tz stay 0
        if (i >= g.nabc + 1 && i <= ie) {
            if (k >= g.nabc + 1 && k <= ks) {
                const TrialTraction<T> t = trial_traction<T, true>(g, f, c, avdz_rd, avdx_rd, i, k);
                tx_ = t.txv;
                tz_ = t.tzv;
                if (ri >= 1 && ri <= FBC_TX && rk >= 1 && rk <= FBC_TZ) {
                    const int n2 = g.at2(i, k);
                    q.RFz[n2] = t.rfz;
                    q.RFx[n2] = t.rfx;
                    avdz_wr[n2] = t.pdz;
                    avdx_wr[n2] = t.pdx;
                }
            } else if (!g.fspace && k == ks + 1) {  // ghost row: tx(nzt-1) = tx(nzt-2), tz(nzt-1) = -tz(nzt-3)
                tx_ = +trial_traction<T, true>(g, f, c, avdz_rd, avdx_rd, i, ks).txv;
                tz_ = -trial_traction<T, true>(g, f, c, avdz_rd, avdx_rd, i, ks - 1).tzv;
            }
        }
        s_txt[n] = tx_;
        s_tzt[n] = tz_;
    }
    __syncthreads();
    auto TXT = [&](int i, int k) { return s_txt[(i - i0 + 1) + (k - k0 + 1) * FBC_HX]; };
    auto TZT = [&](int i, int k) { return s_tzt[(i - i0 + 1) + (k - k0 + 1) * FBC_HX]; };
    auto TINT_X = [&](int i, int k) {  // 4-point average of tz + T0Z around X node (i,k)
        const int n2 = g.at2(i, k), w1 = g.at2(i - 1, k), w2 = g.at2(i, k - 1), w3 = g.at2(i - 1, k - 1);
        return (TZT(i, k) + q.T0Z[n2] + TZT(i - 1, k) + q.T0Z[w1] + TZT(i, k - 1) + q.T0Z[w2] + TZT(i - 1, k - 1) +
                q.T0Z[w3]) / (T)4;
    };

    // 2. friction: the Z and X nodes of the tile (thread = node), then the X nodes of the
    //    column and row beyond it (their tractions after friction, for the output)
    const int ti = threadIdx.x, tk = threadIdx.y;
    const int i = i0 + ti, k = k0 + tk;
    const bool own = i <= ie && k <= ks;
    T tzn = 0, txo = 0;   // beyond the interior plane the reference's tx stays 0
    if (own) {
        const double time = (double)it * c.dtA;
        const int n2 = g.at2(i, k), e1 = g.at2(i + 1, k), e2 = g.at2(i, k + 1), e3 = g.at2(i + 1, k + 1);
        const T tintz = (TXT(i, k) + q.T0X[n2] + TXT(i + 1, k) + q.T0X[e1] + TXT(i, k + 1) + q.T0X[e2] +
                         TXT(i + 1, k + 1) + q.T0X[e3]) / (T)4;
        tzn = friction_z<T>(g, f, q, c, law, s, time, TZT(i, k), tintz, i, k);
        txo = friction_x<T, true>(g, f, q, c, law, s, distX_rd, distX_wr, TXT(i, k), TINT_X(i, k), i, k);
        if (k == ks) {  // the reference's tx/tz arrays also carry the ghost row nzt-1
            const int gh = g.at2(i, k + 1);
            q.tx[gh] = TXT(i, k + 1);
            q.tz[gh] = TZT(i, k + 1);
        }
    }
    s_tx[ti + tk * FBC_PX] = txo;
    if (tid < FBC_PX + FBC_TZ) {  // column i0+FBC_TX (k0..k0+FBC_TZ), then row k0+FBC_TZ (i0..i0+FBC_TX-1)
        const int hi = tid < FBC_PZ ? i0 + FBC_TX : i0 + (tid - FBC_PZ);
        const int hk = tid < FBC_PZ ? k0 + tid : k0 + FBC_TZ;
        T txh = 0;
        if (hi <= ie && hk <= ks && law == 0)
            txh = friction_x<T, false>(g, f, q, c, law, s, distX_rd, distX_wr, TXT(hi, hk), TINT_X(hi, hk), hi, hk);
        else if (hi <= ie && hk <= ks)
            txh = TXT(hi, hk);
        s_tx[(hi - i0) + (hk - k0) * FBC_PX] = txh;
    }
    __syncthreads();

    // 3. output planes, stations, history ring (fd3d_theo.f90:413-467) of the tile's nodes
    if (bx_ == 0 && by_ == 0 && tid < h.nst && it % h.stride == 0) {
        const long long slot = (long long)((it / h.stride - 1) % h.cap);
        const long long p = g.at(h.sta[3 * tid], h.sta[3 * tid + 1], h.sta[3 * tid + 2]);
        T* sp = (T*)h.seis + slot * (3 * h.nst) + 3 * tid;
        sp[0] = f.u[p]; sp[1] = f.v[p]; sp[2] = f.w[p];
    }
    if (!own) return;
    auto TX = [&](int ii, int kk) { return s_tx[(ii - i0) + (kk - k0) * FBC_PX]; };
    const bool top = (k == ks);
    const long long p = g.at(i, g.nyt, k), sz = g.plane;
    const int n2 = g.at2(i, k), e1 = g.at2(i + 1, k), e2 = g.at2(i, k + 1), e3 = g.at2(i + 1, k + 1);
    const T U = f.u[p], U2 = f.u[p + 1], W = f.w[p];
    T srx, srz, scx, scz;
    srz = (T)-2 * W;
    if (!top) {
        const T U3 = f.u[p + sz], U4 = f.u[p + 1 + sz];
        srx = ((T)-2 * U - (T)2 * U2 - (T)2 * U3 - (T)2 * U4) / (T)4;
        if (law == 0) {
            scz = tzn + q.T0Z[n2];
            scx = (TX(i, k) + q.T0X[n2] + TX(i + 1, k) + q.T0X[e1] + TX(i, k + 1) + q.T0X[e2] + TX(i + 1, k + 1) +
                   q.T0X[e3]) / (T)4;
        }
    } else {
        if (law == 1) {
            srx = ((T)-2 * U - (T)2 * U2) / (T)4;
        } else {
            scz = tzn + q.T0Z[n2];
            scx = (TX(i, k) + q.T0X[n2] + TX(i + 1, k) + q.T0X[e1]) / (T)2;
            srx = ((T)-2 * U - (T)2 * U2) / (T)2;
        }
    }
    if (law == 1) { scx = q.schangeX[n2]; scz = q.schangeZ[n2]; }
    else { q.schangeX[n2] = scx; q.schangeZ[n2] = scz; }
    if (!(isfinite((double)srx) && isfinite((double)srz) && isfinite((double)scx) && isfinite((double)scz)))
        atomicOr(status, ST_NONFINITE);
    if (it % h.stride == 0) {
        const int nxT = g.nxt - 2 * g.nabc, nzT = ks - g.nabc;
        const long long slot = (long long)((it / h.stride - 1) % h.cap);
        const long long plane = (long long)nxT * nzT;
        T* r = (T*)h.ring + slot * h.nf * plane + (long long)(k - g.nabc - 1) * nxT + (i - g.nabc - 1);
        r[0] = srx;
        r[plane] = srz;
        r[2 * plane] = scx;
        r[3 * plane] = scz;
        if (h.nf > 4) r[4 * plane] = (T)q.psiZ[n2];
    }
}

// grid of the fused fault BC: fres CTAs (32 x 8 (i,j) each), then the fault tiles
inline void fault_bc_grid(const Grid& g, int& nfres, int& tiles_x, int& tiles) {
    nfres = g.fspace ? 0 : ((g.nxt + 31) / 32) * ((g.nyt + 7) / 8);
    const int nxT = g.nxt - 2 * g.nabc, nzT = g.ks() - g.nabc;
    tiles_x = (nxT + FBC_TX - 1) / FBC_TX;
    tiles = tiles_x * ((nzT + FBC_TZ - 1) / FBC_TZ);
}

// TPV103/104 smooth nucleation of T0X (fd3d_theo.f90:487-542)
template <class T>
__device__ __forceinline__ void nucleation_body(Grid g, Fault<T> q, StepConst<T> c, FvwScalars s, const int* it_dev, int bx_, int by_, int bz_) {
    const int i = g.nabc - 1 + bx_ * blockDim.x + threadIdx.x;
    const int k = g.nabc - 1 + by_ * blockDim.y + threadIdx.y;
    if (i > g.nxt - g.nabc || k > g.ks()) return;
    const double time = (double)(*it_dev) * c.dtA;
    const double th = time - c.dtA / 2.0;
    if (!(th <= s.TT2)) return;
    const double GT = (th < s.TT2) ? exp((th - s.TT2) * (th - s.TT2) / (th * (th - 2.0 * s.TT2))) : 1.0;
    const double hx = (double)i * c.dhA, hz = (double)k * c.dhA;
    const double rr = (hx - s.hx0) * (hx - s.hx0) + (hz - s.hz0) * (hz - s.hz0);
    const double FXZ = (rr < s.RR2 - c.dhA) ? exp(rr / (rr - s.RR2 - c.dhA)) : 0.0;
    const double base = s.nucleation == 2 ? (double)q.T0Xb[g.at2(i, k)] : s.strinixI;
    q.T0X[g.at2(i, k)] = (T)(base + s.perturb * FXZ * GT);
}

// ---------------------------------------------------------------- launch wrappers
template <class T>
__global__ void k_vel_fault(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, int law, FvwScalars s,
                            int* it_dev, int* status) {
    vel_fault_body<T>(g, f, q, c, law, s, it_dev, status, blockIdx.x, blockIdx.y, blockIdx.z);
}

// One PML tile per CTA of PML_TILE threads.  MINB: CTAs that must fit one SM
// (register cap); 1 leaves it free.
template <class T, int MINB = 1, bool SLAB = false>
__global__ void __launch_bounds__(PML_TILE, MINB) k_vel_pml(Grid g, Fields<T> f, const __grid_constant__ PmlDesc D,
                                                             const __grid_constant__ PmlAux<T> X, StepConst<T> c,
                                                             int* status, long long tile0) {
    __shared__ __align__(128) T sm[PML_TILE * AUX_NV];
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) { mbar_init(smem_addr(&bar), 1); fence_mbar_init(); }
    vel_pml_tile<T, SLAB>(g, f, D, X, c, tile0 + blockIdx.x, sm, smem_addr(&bar), 0u, status);
}

template <class T>
__global__ void k_vel_fs(Grid g, Fields<T> f) {
    vel_fs_body<T>(g, f, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class T>
__global__ void k_str_fault(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c) {
    str_fault_body<T>(g, f, q, c, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class T, int MINB = 1, bool SLAB = false>
__global__ void __launch_bounds__(PML_TILE, MINB) k_str_pml(Grid g, Fields<T> f, const __grid_constant__ PmlDesc D,
                                                             const __grid_constant__ PmlAux<T> X, StepConst<T> c,
                                                             int* status, long long tile0) {
    __shared__ __align__(128) T sm[PML_TILE * AUX_NS];
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) { mbar_init(smem_addr(&bar), 1); fence_mbar_init(); }
    str_pml_tile<T, SLAB>(g, f, D, X, c, tile0 + blockIdx.x, sm, smem_addr(&bar), 0u, status);
}

// The tiles of strip s that hold cells of planes klo..khi: [t0, t1) (k is the slowest
// index of a strip's compact range)
inline void pml_strip_tiles(const PmlDesc& D, int s, long long& t0, long long& t1) {
    const Strip& S = D.s[s];
    const int kb = std::max(S.nzb, D.klo), ke = std::min(S.nze, D.khi);
    t0 = t1 = D.cum[s] / PML_TILE;
    if (D.cnt[s] == 0 || kb > ke) return;
    const long long per_k = D.cnt[s] / S.nk;
    t0 = (D.cum[s] + (long long)(kb - S.nzb) * per_k) / PML_TILE;
    t1 = (D.cum[s] + (long long)(ke - S.nzb + 1) * per_k + PML_TILE - 1) / PML_TILE;
}

// launch of a PML sweep: one launch over every tile for a whole model (with a register
// cap picked at run time), one per strip over the tiles of its planes for a z-slab
template <class T>
inline void launch_pml(bool stress, int minb, cudaStream_t st, const Grid& g, const Fields<T>& f, const PmlDesc& D,
                       const PmlAux<T>& X, const StepConst<T>& c, int* status) {
    if (D.klo > 1 || D.khi < g.nzt) {  // a z-slab: the tiles of its planes, strip by strip
        for (int s = 0; s < D.ns; ++s) {
            long long t0, t1;
            pml_strip_tiles(D, s, t0, t1);
            if (t1 <= t0) continue;
            if (stress) k_str_pml<T, 1, true><<<(unsigned)(t1 - t0), PML_TILE, 0, st>>>(g, f, D, X, c, status, t0);
            else k_vel_pml<T, 1, true><<<(unsigned)(t1 - t0), PML_TILE, 0, st>>>(g, f, D, X, c, status, t0);
        }
        return;
    }
    const unsigned nblk = (unsigned)((D.cum[PML_MAXS] + PML_TILE - 1) / PML_TILE);
    if (nblk == 0) return;
#define FD3D_PML_CASE(MB)                                                                  \
    case MB:                                                                               \
        if (stress) k_str_pml<T, MB><<<nblk, PML_TILE, 0, st>>>(g, f, D, X, c, status, 0);  \
        else k_vel_pml<T, MB><<<nblk, PML_TILE, 0, st>>>(g, f, D, X, c, status, 0);         \
        break;
    switch (minb) {
        FD3D_PML_CASE(2)
        FD3D_PML_CASE(3)
        FD3D_PML_CASE(4)
        default:
            if (stress) k_str_pml<T, 1><<<nblk, PML_TILE, 0, st>>>(g, f, D, X, c, status, 0);
            else k_vel_pml<T, 1><<<nblk, PML_TILE, 0, st>>>(g, f, D, X, c, status, 0);
    }
#undef FD3D_PML_CASE
}

template <class T>
__global__ void k_str_fs(Grid g, Fields<T> f) {
    str_fs_body<T>(g, f, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class T>
__global__ void k_traction(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, const int* it_dev) {
    traction_body<T>(g, f, q, c, it_dev, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class T>
__global__ void k_friction(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, int law, FvwScalars s,
                           const int* it_dev) {
    friction_body<T>(g, f, q, c, law, s, it_dev, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class T>
__global__ void k_output(Grid g, Fields<T> f, Fault<T> q, int law, const int* it_dev, const __grid_constant__ HistDesc h,
                         int* status) {
    output_body<T>(g, f, q, law, it_dev, h, status, blockIdx.x, blockIdx.y, blockIdx.z);
}

// The fused fault boundary condition of one step: nfres CTAs of fres, then the fault tiles
// (tiles_x per row of tiles); CTA of 32 x 8 threads.
template <class T>
__global__ void __launch_bounds__(256) k_fault_bc(Grid g, Fields<T> f, Fault<T> q, StepConst<T> c, int law,
                                                  FvwScalars s, const int* it_dev, const __grid_constant__ HistDesc h,
                                                  int* status, int nfres, int tiles_x) {
    __shared__ T sm[FBC_SMEM];
    const int b = blockIdx.x;
    if (b < nfres) {
        const int sx = (g.nxt + 31) / 32;
        str_fs_body<T>(g, f, b % sx, b / sx, 0);
        return;
    }
    const int t = b - nfres;
    fault_bc_body<T>(g, f, q, c, law, s, it_dev, h, status, t % tiles_x, t / tiles_x, sm);
}

template <class T>
__global__ void k_nucleation(Grid g, Fault<T> q, StepConst<T> c, FvwScalars s, const int* it_dev) {
    nucleation_body<T>(g, q, c, s, it_dev, blockIdx.x, blockIdx.y, blockIdx.z);
}

}  // namespace fd3d
