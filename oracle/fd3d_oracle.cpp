// fd3d_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A CPU restatement, loop by loop, of the FD3D_TSN time step:
//   src/fd3d_deriv.f90  dvel/uxx1/vyy1/wzz1, bnd2d/uxx0a/vyy0a/wzz0a, dstres,
//                       strbnd/sxx/sxy0/sxz0/syz0, sxz1 (tasxz), tasii, tasu1, tasw1,
//                       fuvw, fres, init_pml, pml_uvw, pml_xyz, interp_fric
//                       (with the FSPACE build's top PML strip, fspace = 1)
//   src/fd3d_theo.f90   fd3d(): initialisation, loop order, traction, friction,
//                       output planes, stations, TPV103/104 nucleation ramp
// Every region keeps the reference's index ranges, evaluation order of sums and
// the quirks it has (one-sided fault, mirrors of v/xy/yz into j=nyt, diagonal mu
// average for yz, Dc vs DcX at X nodes, /4 top row of FVW slip rate, ...).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
// library.  The GPU library never links or calls it.
//
// PARITY UNPINNED: the reference ships no golden outputs and no tests, and it is
// Fortran with no Fortran compiler on either machine, so this restatement cannot
// be checked against the reference's own output.  It is cross-checked against
// physics invariants (rest state, symmetry, PML energy decay) in tests/.
//
// Precision variants (template <F,A>):
//   F = field type (the reference's `real`), A = accumulator type used for slip,
//   slip path, rupture/rise/slip time, time, psi and the FVW Newton solve.
//   variant 0: F=float,  A=double  -- the arithmetic of the GPU FP32 build
//   variant 1: F=double, A=double  -- the reference built with -r8
//   variant 2: F=float,  A=float   -- the reference built without -r8
// Built with -ffp-contract=off so every + - * / sqrt is a single IEEE operation.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <cstdlib>
#include <thread>
#include "../include/fd3d_gpu.h"

namespace {

// Host threads for the order-independent 3-D regions (every iteration writes only
// its own elements), so results do not depend on the thread count.
int g_threads = 0;
int oracle_threads() {
    if (g_threads > 0) return g_threads;
    const char* e = std::getenv("FD3D_ORACLE_THREADS");
    int n = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
    return n > 0 ? n : 1;
}
// grids below this many cells run every region on the calling thread
long long g_serial_below = 1 << 21;
thread_local long long t_cells = 0;
template <class Fn> void par_for(int lo, int hi, Fn fn) {
    int n = hi - lo + 1;
    int nt = t_cells < g_serial_below ? 1 : std::min(oracle_threads(), n);
    if (nt <= 1 || n < 4) { for (int k = lo; k <= hi; ++k) fn(k); return; }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; ++t) {
        int a = lo + (int)((long)n * t / nt), b = lo + (int)((long)n * (t + 1) / nt) - 1;
        th.emplace_back([=]() { for (int k = a; k <= b; ++k) fn(k); });
    }
    for (auto& x : th) x.join();
}

template <class F, class A>
struct Oracle {
    // ---------------- parameters (fd3dparam_com, pml_com, traction_com)
    int nxt, nyt, nzt, nabc, nfs, nysc, ntfd;
    int fspace = 0;  // FSPACE build (fd3d_init.f90:161-165): PML strip 5 above, no free surface
    int nstrip = 4;  // PML strips: 4, or 5 under FSPACE
    F dh, dt, damp_s, omegaM_pml;
    A dtA;
    int law;
    int nst;
    int staX[FD3D_MAX_STATIONS], staY[FD3D_MAX_STATIONS], staZ[FD3D_MAX_STATIONS];
    int it = 0;  // steps done
    int newton_fail = 0;

    // ---------------- 3-D arrays (medium_com, displt_com, strfld_com)
    std::vector<F> lam1, mu1, d1, u1, v1, w1, xx, yy, zz, xy, yz, xz;
    // ---------------- plane arrays (traction_com, friction_com, source_com)
    std::vector<F> tx, tz, v1t, avdx, avdz, RFx, RFz, au1, av1, aw1;
    std::vector<F> uZ, wX, tabsX, tabsZ, T0X, T0Z, T0Xb, striniX, striniZ, Dc;
    std::vector<F> peakX, dynX, DcX, peakZ, dynZ, DcZ, coh;
    std::vector<F> aX, bX, vwX, aZ, bZ, vwZ, fwX, fwZ;
    std::vector<A> psiX, psiZ, psiX0, psiZ0;
    std::vector<A> distX, distZ, slipX, slipZ, ruptime, rise, sliptime;
    std::vector<F> sliprateoutX, sliprateoutZ, schangeX, schangeZ;
    std::vector<A> psiout;
    std::vector<A> moment_rate;  // per step (fd3d_theo.f90:574-578, dtseis = dt)
    std::vector<F> seis;  // nst*3 of the last step
    A Sn = 0, v0 = 0, f0 = 0, fw = 0, uini = 0, wini = 0;
    int nucleation = 0;
    A hx0 = 0, hz0 = 0, perturb = 0, RR2 = 0, TT2 = 0, strinixI = 0;

    // ---------------- PML (pml_com), per strip s=1..4 (5 under FSPACE)
    struct Strip {
        int nxb, nxe, nyb, nye, nzb, nze;
        int ni, nj1, nk;  // nj1 = nye-nyb+2 (the "+1" arrays)
        std::vector<F> u[3], v[3], w[3], sxx[3], syy[3], szz[3], sxy[2], sxz[2], syz[2];
        std::vector<F> ox, oy, oz, oxS, oyS, ozS;  // damping profiles (index 1-based -> [i-1])
        size_t at(int i2, int j2, int k2) const { return (size_t)(i2 - 1) + (size_t)ni * ((size_t)(j2 - 1) + (size_t)nj1 * (size_t)(k2 - 1)); }
    } S[6];  // 1-based
    std::vector<F> omega_pml, omegaR_pml, omega_pmlM, omegaR_pmlM;  // 1-based by [i-1]

    inline size_t I3(int i, int j, int k) const { return (size_t)(i - 1) + (size_t)nxt * ((size_t)(j - 1) + (size_t)nyt * (size_t)(k - 1)); }
    inline size_t I2(int i, int k) const { return (size_t)(i - 1) + (size_t)nxt * (size_t)(k - 1); }

    explicit Oracle(const fd3d_params& p) {
        nxt = p.nxt; nyt = p.nyt; nzt = p.nzt; nabc = p.nabc; nfs = p.nfs; nysc = nyt; ntfd = p.ntfd;
        fspace = p.fspace; nstrip = fspace ? 5 : 4;
        dh = (F)p.dh; dt = (F)p.dt; damp_s = (F)p.damp_s; dtA = (A)p.dt;
        law = p.law;
        // omegaM_pml=pml_fact*pml_vp/(2.*dh*(nabc-1))  fd3d_init.f90:171
        omegaM_pml = (F)p.pml_fact * (F)p.pml_vp / ((F)2 * dh * (F)(nabc - 1));
        nst = p.nstations;
        for (int s = 0; s < nst; ++s) { staX[s] = p.staX[s]; staY[s] = p.staY[s]; staZ[s] = p.staZ[s]; }
        size_t n3 = (size_t)nxt * nyt * nzt, n2 = (size_t)nxt * nzt;
        for (auto* a : {&lam1, &mu1, &d1, &u1, &v1, &w1, &xx, &yy, &zz, &xy, &yz, &xz}) a->assign(n3, (F)0);
        for (auto* a : {&tx, &tz, &v1t, &avdx, &avdz, &RFx, &RFz, &au1, &av1, &aw1, &uZ, &wX, &tabsX, &tabsZ,
                        &T0X, &T0Z, &T0Xb, &striniX, &striniZ, &Dc, &peakX, &dynX, &DcX, &peakZ, &dynZ, &DcZ, &coh,
                        &aX, &bX, &vwX, &aZ, &bZ, &vwZ, &fwX, &fwZ, &sliprateoutX, &sliprateoutZ, &schangeX, &schangeZ})
            a->assign(n2, (F)0);
        for (auto* a : {&psiX, &psiZ, &distX, &distZ, &slipX, &slipZ, &ruptime, &rise, &sliptime, &psiout}) a->assign(n2, (A)0);
        seis.assign((size_t)std::max(nst, 1) * 3, (F)0);
        init_pml();
        reset();
    }

    // fd3d_theo.f90:59-88 (zeroing) -- PML aux zeroed as in init_pml fd3d_deriv.f90:1342-1410
    void reset() {
        for (auto* a : {&u1, &v1, &w1, &xx, &yy, &zz, &xy, &yz, &xz}) std::fill(a->begin(), a->end(), (F)0);
        for (auto* a : {&tx, &tz, &v1t, &avdx, &avdz, &RFx, &RFz, &au1, &av1, &aw1, &uZ, &wX, &sliprateoutX,
                        &sliprateoutZ, &schangeX, &schangeZ}) std::fill(a->begin(), a->end(), (F)0);
        moment_rate.clear();
        std::fill(ruptime.begin(), ruptime.end(), (A)1.e4);
        std::fill(rise.begin(), rise.end(), (A)0);
        std::fill(sliptime.begin(), sliptime.end(), (A)1.e4);
        for (auto* a : {&distX, &distZ, &slipX, &slipZ, &psiout}) std::fill(a->begin(), a->end(), (A)0);
        F t0 = law == FD3D_LAW_FVW ? (F)1 : (F)0;  // FVW: tabsX=tabsZ=1 (fd3d_theo.f90:78-82)
        std::fill(tabsX.begin(), tabsX.end(), t0);
        std::fill(tabsZ.begin(), tabsZ.end(), t0);
        for (int s = 1; s <= nstrip; ++s) {
            Strip& st = S[s];
            for (auto& a : st.u) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.v) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.w) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.sxx) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.syy) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.szz) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.sxy) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.sxz) std::fill(a.begin(), a.end(), (F)0);
            for (auto& a : st.syz) std::fill(a.begin(), a.end(), (F)0);
        }
        if (!T0Xb.empty()) T0X = T0Xb;          // undo the nucleation ramp
        if (!psiX0.empty()) { psiX = psiX0; psiZ = psiZ0; }
        it = 0; newton_fail = 0;
    }

    // init_pml  fd3d_deriv.f90:1319-1493 (strip 5: the FSPACE top strip, :1413-1437)
    void init_pml() {
        const int bx[6][6] = {{0, 0, 0, 0, 0, 0},
                              {2, nabc, nabc + 1, nyt - 1, nabc + 1, nzt - nfs},
                              {nxt - nabc + 1, nxt - 1, nabc + 1, nyt - 1, nabc + 1, nzt - nfs},
                              {2, nxt - 1, 2, nabc, nabc + 1, nzt - nfs},
                              {2, nxt - 1, 2, nyt - 1, 2, nabc},
                              {2, nxt - 1, 2, nyt - 1, nzt - nabc + 1, nzt - 1}};
        for (int s = 1; s <= nstrip; ++s) {
            Strip& st = S[s];
            st.nxb = bx[s][0]; st.nxe = bx[s][1]; st.nyb = bx[s][2]; st.nye = bx[s][3]; st.nzb = bx[s][4]; st.nze = bx[s][5];
            st.ni = st.nxe - st.nxb + 1; st.nk = st.nze - st.nzb + 1;
            st.nj1 = st.nye - st.nyb + 2;  // every aux array allocated with the +1 (superset of the reference's)
            size_t n = (size_t)st.ni * st.nj1 * st.nk;
            for (auto& a : st.u) a.assign(n, (F)0);
            for (auto& a : st.v) a.assign(n, (F)0);
            for (auto& a : st.w) a.assign(n, (F)0);
            for (auto& a : st.sxx) a.assign(n, (F)0);
            for (auto& a : st.syy) a.assign(n, (F)0);
            for (auto& a : st.szz) a.assign(n, (F)0);
            for (auto& a : st.sxy) a.assign(n, (F)0);
            for (auto& a : st.sxz) a.assign(n, (F)0);
            for (auto& a : st.syz) a.assign(n, (F)0);
            st.ox.assign(st.ni, (F)0); st.oxS.assign(st.ni, (F)0);
            st.oy.assign(st.nj1, (F)0); st.oyS.assign(st.nj1, (F)0);
            st.oz.assign(st.nk, (F)0); st.ozS.assign(st.nk, (F)0);
        }
        int n = nabc - 1;
        omega_pml.assign(n, 0); omegaR_pml.assign(n, 0); omega_pmlM.assign(n, 0); omegaR_pmlM.assign(n, 0);
        for (int i = 1; i <= n; ++i) {  // fd3d_deriv.f90:1439-1444
            F r = (F)i / (F)n;
            F rM = ((F)i - (F)0.5) / (F)n;
            omega_pml[i - 1] = (F)0.5 * dt * omegaM_pml * ((r * r) * (r * r));
            omegaR_pml[nabc - i - 1] = omega_pml[i - 1];
            omega_pmlM[i - 1] = (F)0.5 * dt * omegaM_pml * ((rM * rM) * (rM * rM));
            omegaR_pmlM[nabc - i - 1] = omega_pmlM[i - 1];
        }
        for (int i = 1; i <= n; ++i) {  // fd3d_deriv.f90:1456-1491
            S[1].ox[i - 1] = omegaR_pml[i - 1];
            S[1].oxS[i - 1] = omegaR_pmlM[i - 1];
            S[2].ox[i - 1] = omega_pmlM[i - 1];
            S[2].oxS[i - 1] = omega_pml[i - 1];
            S[3].oy[i - 1] = omegaR_pml[i - 1];
            S[3].ox[i - 1] = omegaR_pml[i - 1];
            S[3].ox[nxt - i - 1 - 1] = omega_pmlM[i - 1];
            S[3].oyS[i - 1] = omegaR_pmlM[i - 1];
            S[3].oxS[i - 1] = omegaR_pmlM[i - 1];
            S[3].oxS[nxt - i - 1 - 1] = omega_pml[i - 1];
            S[4].oz[i - 1] = omegaR_pml[i - 1];
            S[4].ox[i - 1] = omegaR_pml[i - 1];
            S[4].ox[nxt - i - 1 - 1] = omega_pmlM[i - 1];
            S[4].oy[i - 1] = omegaR_pml[i - 1];
            S[4].ozS[i - 1] = omegaR_pmlM[i - 1];
            S[4].oxS[i - 1] = omegaR_pmlM[i - 1];
            S[4].oxS[nxt - i - 1 - 1] = omega_pml[i - 1];
            S[4].oyS[i - 1] = omegaR_pmlM[i - 1];
            if (fspace) {  // fd3d_deriv.f90:1481-1490
                S[5].oz[i - 1] = omega_pmlM[i - 1];
                S[5].ox[i - 1] = omegaR_pml[i - 1];
                S[5].ox[nxt - i - 1 - 1] = omega_pmlM[i - 1];
                S[5].oy[i - 1] = omegaR_pml[i - 1];
                S[5].ozS[i - 1] = omega_pml[i - 1];
                S[5].oxS[i - 1] = omegaR_pmlM[i - 1];
                S[5].oxS[nxt - i - 1 - 1] = omega_pml[i - 1];
                S[5].oyS[i - 1] = omegaR_pmlM[i - 1];
            }
        }
    }

    // ------------------------------------------------------------------ setup
    void set_medium(const double* l, const double* m, const double* d) {
        size_t n3 = lam1.size();
        for (size_t q = 0; q < n3; ++q) { lam1[q] = (F)l[q]; mu1[q] = (F)m[q]; d1[q] = (F)d[q]; }
    }

    // friction arrays + interp_fric  fd3d_deriv.f90:3150-3190
    void set_fault(const fd3d_fault& f) {
        size_t n2 = tx.size();
        auto cp = [&](std::vector<F>& dst, const double* src, double dflt) {
            for (size_t q = 0; q < n2; ++q) dst[q] = (F)(src ? src[q] : dflt);
        };
        cp(striniX, f.striniX, 0); cp(striniZ, f.striniZ, 0); cp(Dc, f.Dc, 0);
        std::fill(peakX.begin(), peakX.end(), (F)0); std::fill(DcX.begin(), DcX.end(), (F)0);
        std::fill(dynX.begin(), dynX.end(), (F)0); std::fill(T0X.begin(), T0X.end(), (F)0);
        std::fill(peakZ.begin(), peakZ.end(), (F)0); std::fill(DcZ.begin(), DcZ.end(), (F)0);
        std::fill(dynZ.begin(), dynZ.end(), (F)0); std::fill(T0Z.begin(), T0Z.end(), (F)0);
        if (law == FD3D_LAW_FVW) {
            cp(aZ, f.a, 0); cp(bZ, f.b, 0); cp(vwZ, f.vw, 0);
            for (size_t q = 0; q < n2; ++q) psiZ[q] = (A)(f.psi ? f.psi[q] : 0.0);
            cp(aX, f.aX, 0); cp(bX, f.bX, 0); cp(vwX, f.vwX, 0);
            for (size_t q = 0; q < n2; ++q) psiX[q] = (A)(f.psiX ? f.psiX[q] : 0.0);
            cp(fwZ, f.fwZ, f.fw); cp(fwX, f.fwX, f.fw);
            T0Z = striniZ;
            Sn = (A)f.Sn; v0 = (A)f.v0; f0 = (A)f.f0; fw = (A)f.fw;
            uini = (A)f.uini; wini = (A)f.wini;
            nucleation = f.nucleation;
            hx0 = (A)f.hx0; hz0 = (A)f.hz0; perturb = (A)f.perturb; RR2 = (A)f.RR2;
            TT2 = (A)f.TT2; strinixI = (A)f.strinixI;
            psiX0 = psiX; psiZ0 = psiZ;
        } else {
            std::vector<F> pk(n2), dy(n2);
            cp(pk, f.peak_xz, 0); cp(dy, f.dyn_xz, 0); cp(coh, f.coh, 0);
            peakZ = pk; dynZ = dy; DcZ = Dc; T0Z = striniZ;
            nucleation = 0;
        }
        for (int i = 2; i <= nxt - 1; ++i)
            for (int k = 2; k <= nzt - 1; ++k) {
                if (law != FD3D_LAW_FVW) {
                    peakX[I2(i, k)] = (peakZ[I2(i, k)] + peakZ[I2(i - 1, k)] + peakZ[I2(i, k - 1)] + peakZ[I2(i - 1, k - 1)]) / (F)4;
                    dynX[I2(i, k)] = (dynZ[I2(i, k)] + dynZ[I2(i - 1, k)] + dynZ[I2(i, k - 1)] + dynZ[I2(i - 1, k - 1)]) / (F)4;
                    DcX[I2(i, k)] = (DcZ[I2(i, k)] + DcZ[I2(i - 1, k)] + DcZ[I2(i, k - 1)] + DcZ[I2(i - 1, k - 1)]) / (F)4;
                }
                T0X[I2(i, k)] = (striniX[I2(i, k)] + striniX[I2(i - 1, k)] + striniX[I2(i, k - 1)] + striniX[I2(i - 1, k - 1)]) / (F)4;
            }
        T0Xb = T0X;
    }

    // ------------------------------------------------------------------ velocity
    // uxx1/vyy1/wzz1  fd3d_deriv.f90:50-193, called by dvel with nyt-2 (fd3d_theo.f90:208)
    void dvel() {
        const F dth = dt / dh, c1 = (F)9 / (F)8, c2 = (F)-1 / (F)24;
        const int nyb = nabc + 1, nye = nyt - 2;
        par_for(nabc + 1, nzt - nfs, [&](int k) {
            for (int j = nyb; j <= nye; ++j)
                for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                    const F d = d1[I3(i, j, k)];
                    u1[I3(i, j, k)] = u1[I3(i, j, k)] + (dth / d) * (
                        c1 * (xx[I3(i, j, k)] - xx[I3(i - 1, j, k)]) + c2 * (xx[I3(i + 1, j, k)] - xx[I3(i - 2, j, k)]) +
                        c1 * (xy[I3(i, j, k)] - xy[I3(i, j - 1, k)]) + c2 * (xy[I3(i, j + 1, k)] - xy[I3(i, j - 2, k)]) +
                        c1 * (xz[I3(i, j, k)] - xz[I3(i, j, k - 1)]) + c2 * (xz[I3(i, j, k + 1)] - xz[I3(i, j, k - 2)]));
                    v1[I3(i, j, k)] = v1[I3(i, j, k)] + (dth / d) * (
                        c1 * (xy[I3(i + 1, j, k)] - xy[I3(i, j, k)]) + c2 * (xy[I3(i + 2, j, k)] - xy[I3(i - 1, j, k)]) +
                        c1 * (yy[I3(i, j + 1, k)] - yy[I3(i, j, k)]) + c2 * (yy[I3(i, j + 2, k)] - yy[I3(i, j - 1, k)]) +
                        c1 * (yz[I3(i, j, k)] - yz[I3(i, j, k - 1)]) + c2 * (yz[I3(i, j, k + 1)] - yz[I3(i, j, k - 2)]));
                    w1[I3(i, j, k)] = w1[I3(i, j, k)] + (dth / d) * (
                        c1 * (xz[I3(i + 1, j, k)] - xz[I3(i, j, k)]) + c2 * (xz[I3(i + 2, j, k)] - xz[I3(i - 1, j, k)]) +
                        c1 * (yz[I3(i, j, k)] - yz[I3(i, j - 1, k)]) + c2 * (yz[I3(i, j + 1, k)] - yz[I3(i, j - 2, k)]) +
                        c1 * (zz[I3(i, j, k + 1)] - zz[I3(i, j, k)]) + c2 * (zz[I3(i, j, k + 2)] - zz[I3(i, j, k - 1)]));
                }
        });
    }

    // bnd2d -> uxx0a, vyy0a, wzz0a at j=nyt-1 + v mirror  fd3d_deriv.f90:198-235,284-508
    void bnd2d() {
        const F dth = dt / dh;
        const int j = nyt - 1;
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                F pdx = (xx[I3(i, j, k)] - xx[I3(i - 1, j, k)]) + (xy[I3(i, j, k)] - xy[I3(i, j - 1, k)]) +
                        (xz[I3(i, j, k)] - xz[I3(i, j, k - 1)]);
                au1[p] = pdx - au1[p];
                F d = d1[I3(i, j, k)];
                u1[I3(i, j, k)] = u1[I3(i, j, k)] + (dth / d) * (pdx + damp_s * au1[p]);
                au1[p] = pdx;
                F pdy = (xy[I3(i + 1, j, k)] - xy[I3(i, j, k)]) + (yy[I3(i, j + 1, k)] - yy[I3(i, j, k)]) +
                        (yz[I3(i, j, k)] - yz[I3(i, j, k - 1)]);
                av1[p] = pdy - av1[p];
                v1[I3(i, j, k)] = v1[I3(i, j, k)] + (dth / d) * (pdy + damp_s * av1[p]);
                av1[p] = pdy;
                F pdz = (xz[I3(i + 1, j, k)] - xz[I3(i, j, k)]) + (yz[I3(i, j, k)] - yz[I3(i, j - 1, k)]) +
                        (zz[I3(i, j, k + 1)] - zz[I3(i, j, k)]);
                aw1[p] = pdz - aw1[p];
                w1[I3(i, j, k)] = w1[I3(i, j, k)] + (dth / d) * (pdz + damp_s * aw1[p]);
                aw1[p] = pdz;
            }
        for (int i = 1; i <= nxt; ++i)
            for (int k = 1; k <= nzt; ++k) v1[I3(i, nyt, k)] = v1[I3(i, nyt - 1, k)];
    }

    // FVW Newton solve on one node, fd3d_deriv.f90:1148-1161 (iteration cap added)
    A newton(A vtilde, A cdelta, A uw, A psi, A a) {
        A e = v0 * std::exp(-psi / a);
        A ferr = 10;
        int j = 0;
        while (std::fabs(ferr) > (A)1e-10) {
            ++j;
            A fwv = vtilde + cdelta * uw + std::sinh(uw) * e;
            A dfw = cdelta + std::cosh(uw) * e;
            ferr = fwv / dfw;
            uw = uw - ferr;
            if (j > 200) { ++newton_fail; break; }
        }
        return uw;
    }

    // tasu1 / tasw1  fd3d_deriv.f90:1109-1234
    void tasuw() {
        const F dth = dt / dh;
        const int j = nysc;
        if (law != FD3D_LAW_FVW) {
            for (int k = nabc + 1; k <= nzt - nfs; ++k)
                for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                    F d = d1[I3(i, j, k)];
                    u1[I3(i, j, k)] = u1[I3(i, j, k)] + (dth / d) * (F)2 * (tx[I2(i, k)] + RFx[I2(i, k)]);
                }
            for (int k = nabc + 1; k <= nzt - nfs; ++k)
                for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                    F d = d1[I3(i, j, k)];
                    w1[I3(i, j, k)] = w1[I3(i, j, k)] + (dth / d) * ((F)2 * (tz[I2(i, k)] + RFz[I2(i, k)]));
                }
            return;
        }
        const A dthA = dtA / (A)dh;
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                A d = (A)d1[I3(i, j, k)];
                A u = (A)u1[I3(i, j, k)];
                A a = (A)aX[p];
                A s1 = (A)2 * (std::fabs((A)wX[p]) + std::fabs(wini)), s2 = (A)2 * (std::fabs(u) + std::fabs(uini));
                A sr = std::sqrt(s1 * s1 + s2 * s2);
                A cdelta = (A)2 * (dthA / d) * Sn * a;
                A uw = std::asinh(std::exp(psiX[p] / a) * sr / ((A)2 * v0));
                A rfz = ((A)RFz[I2(i, k)] + (A)RFz[I2(i - 1, k)] + (A)RFz[I2(i, k - 1)] + (A)RFz[I2(i - 1, k - 1)]) / (A)4;
                A q1 = (A)wX[p] + (A)2 * (dthA / d) * (rfz - (A)T0Z[p]);
                A q2 = u + (A)2 * (dthA / d) * ((A)RFx[p] - (A)T0X[p]);
                A vtilde = -std::sqrt(q1 * q1 + q2 * q2);
                uw = newton(vtilde, cdelta, uw, psiX[p], a);
                u1[I3(i, j, k)] = (F)(((A)tx[p] + (A)T0X[p]) * (-std::sinh(uw)) * v0 * std::exp(-psiX[p] / a) / (A)tabsX[p] + uini);
            }
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                A d = (A)d1[I3(i, j, k)];
                A w = (A)w1[I3(i, j, k)];
                A a = (A)aZ[p];
                A s1 = (A)2 * (w - wini), s2 = (A)2 * ((A)uZ[p] - uini);
                A sr = std::sqrt(s1 * s1 + s2 * s2);
                A cdelta = (A)2 * (dthA / d) * Sn * a;
                A uw = std::asinh(std::exp(psiZ[p] / a) * sr / ((A)2 * v0));
                A rfx = ((A)RFx[p] + (A)RFx[I2(i + 1, k)] + (A)RFx[I2(i, k + 1)] + (A)RFx[I2(i + 1, k + 1)]) / (A)4;
                A t0x = ((A)T0X[p] + (A)T0X[I2(i + 1, k)] + (A)T0X[I2(i, k + 1)] + (A)T0X[I2(i + 1, k + 1)]) / (A)4;
                A q1 = w + (A)2 * (dthA / d) * ((A)RFz[p] - (A)T0Z[p]);
                A q2 = (A)uZ[p] + (A)2 * (dthA / d) * (rfx - t0x);
                A vtilde = -std::sqrt(q1 * q1 + q2 * q2);
                uw = newton(vtilde, cdelta, uw, psiZ[p], a);
                w1[I3(i, j, k)] = (F)(((A)tz[p] + (A)T0Z[p]) * (-std::sinh(uw) * v0 * std::exp(-psiZ[p] / a)) / (A)tabsZ[p] + wini);
            }
    }

    // pml_uvw  fd3d_deriv.f90:1927-2299 (strip 5: :2223-2293)
    void pml_uvw() {
        for (int s = 1; s <= nstrip; ++s) {
            Strip& st = S[s];
            const bool y3 = (s == 3);
            const int jue = y3 ? st.nye : st.nye + 1;  // u,w loops run to nye+1 except in strip 3
            par_for(st.nzb, st.nze, [&](int k) {
                for (int j = st.nyb; j <= jue; ++j)
                    for (int i = st.nxb; i <= st.nxe; ++i) {
                        int k2 = 1 - st.nzb + k, j2 = 1 - st.nyb + j, i2 = 1 - st.nxb + i;
                        size_t q = st.at(i2, j2, k2);
                        F d = d1[I3(i, j, k)];
                        F pt;
                        pt = (st.u[0][q] * ((F)1 - st.ox[i2 - 1]) + (dt / d) * (xx[I3(i, j, k)] - xx[I3(i - 1, j, k)]) / dh);
                        st.u[0][q] = pt / ((F)1 + st.ox[i2 - 1]);
                        pt = (st.u[1][q] * ((F)1 - st.oy[j2 - 1]) + (dt / d) * (xy[I3(i, j, k)] - xy[I3(i, j - 1, k)]) / dh);
                        st.u[1][q] = pt / ((F)1 + st.oy[j2 - 1]);
                        pt = (st.u[2][q] * ((F)1 - st.oz[k2 - 1]) + (dt / d) * (xz[I3(i, j, k)] - xz[I3(i, j, k - 1)]) / dh);
                        st.u[2][q] = pt / ((F)1 + st.oz[k2 - 1]);
                        u1[I3(i, j, k)] = st.u[0][q] + st.u[1][q] + st.u[2][q];
                        if (y3) {  // strip 3 keeps u, v, w in one loop (fd3d_deriv.f90:2096-2143)
                            pt = st.v[0][q] * ((F)1 - st.oxS[i2 - 1]) + (dt / d) * (xy[I3(i + 1, j, k)] - xy[I3(i, j, k)]) / dh;
                            st.v[0][q] = pt / ((F)1 + st.oxS[i2 - 1]);
                            pt = st.v[1][q] * ((F)1 - st.oy[j2 - 1]) + (dt / d) * (yy[I3(i, j + 1, k)] - yy[I3(i, j, k)]) / dh;
                            st.v[1][q] = pt / ((F)1 + st.oy[j2 - 1]);
                            pt = st.v[2][q] * ((F)1 - st.oz[k2 - 1]) + (dt / d) * (yz[I3(i, j, k)] - yz[I3(i, j, k - 1)]) / dh;
                            st.v[2][q] = pt / ((F)1 + st.oz[k2 - 1]);
                            v1[I3(i, j, k)] = st.v[0][q] + st.v[1][q] + st.v[2][q];
                        }
                        pt = st.w[0][q] * ((F)1 - st.oxS[i2 - 1]) + (dt / d) * (xz[I3(i + 1, j, k)] - xz[I3(i, j, k)]) / dh;
                        st.w[0][q] = pt / ((F)1 + st.oxS[i2 - 1]);
                        pt = st.w[1][q] * ((F)1 - st.oy[j2 - 1]) + (dt / d) * (yz[I3(i, j, k)] - yz[I3(i, j - 1, k)]) / dh;
                        st.w[1][q] = pt / ((F)1 + st.oy[j2 - 1]);
                        pt = st.w[2][q] * ((F)1 - st.oz[k2 - 1]) + (dt / d) * (zz[I3(i, j, k + 1)] - zz[I3(i, j, k)]) / dh;
                        st.w[2][q] = pt / ((F)1 + st.oz[k2 - 1]);
                        w1[I3(i, j, k)] = st.w[0][q] + st.w[1][q] + st.w[2][q];
                    }
            });
            if (y3) continue;
            par_for(st.nzb, st.nze, [&](int k) {
                for (int j = st.nyb; j <= st.nye; ++j)
                    for (int i = st.nxb; i <= st.nxe; ++i) {
                        int k2 = 1 - st.nzb + k, j2 = 1 - st.nyb + j, i2 = 1 - st.nxb + i;
                        size_t q = st.at(i2, j2, k2);
                        F d = d1[I3(i, j, k)];
                        F pt;
                        pt = st.v[0][q] * ((F)1 - st.oxS[i2 - 1]) + (dt / d) * (xy[I3(i + 1, j, k)] - xy[I3(i, j, k)]) / dh;
                        st.v[0][q] = pt / ((F)1 + st.oxS[i2 - 1]);
                        pt = st.v[1][q] * ((F)1 - st.oy[j2 - 1]) + (dt / d) * (yy[I3(i, j + 1, k)] - yy[I3(i, j, k)]) / dh;
                        st.v[1][q] = pt / ((F)1 + st.oy[j2 - 1]);
                        pt = st.v[2][q] * ((F)1 - st.oz[k2 - 1]) + (dt / d) * (yz[I3(i, j, k)] - yz[I3(i, j, k - 1)]) / dh;
                        st.v[2][q] = pt / ((F)1 + st.oz[k2 - 1]);
                        v1[I3(i, j, k)] = st.v[0][q] + st.v[1][q] + st.v[2][q];
                    }
            });
        }
    }

    // fuvw  fd3d_deriv.f90:1018-1062, called with nzt-nfs (fd3d_theo.f90:214)
    void fuvw() {
        const int n = nzt - nfs;
        for (int j = 1; j <= nyt; ++j)
            for (int i = 2; i <= nxt - 1; ++i)
                u1[I3(i, j, n + 1)] = u1[I3(i, j, n)] - (w1[I3(i, j, n)] - w1[I3(i - 1, j, n)]);
        for (int j = 2; j <= nyt - 1; ++j)
            for (int i = 2; i <= nxt - 1; ++i)
                v1[I3(i, j, n + 1)] = v1[I3(i, j, n)] - (w1[I3(i, j + 1, n)] - w1[I3(i, j, n)]);
        for (int j = 2; j <= nyt; ++j)
            for (int i = 2; i <= nxt - 2; ++i) {
                F xl = lam1[I3(i, j, n + 1)], xm = mu1[I3(i, j, n + 1)];
                F a = (F)2 * xl, b = xl + (F)2 * xm;
                w1[I3(i, j, n + 1)] = +(w1[I3(i, j, n - 1)] - (a / b) * (
                    u1[I3(i + 1, j, n)] - u1[I3(i, j, n)] + u1[I3(i + 1, j, n + 1)] - u1[I3(i, j, n + 1)] +
                    v1[I3(i, j, n)] - v1[I3(i, j - 1, n)] + v1[I3(i, j, n + 1)] - v1[I3(i, j - 1, n + 1)]));
            }
    }

    // ------------------------------------------------------------------ stress
    // dstres  fd3d_deriv.f90:513-622, called with nyt-2 (fd3d_theo.f90:220)
    void dstres() {
        const F dth = dt / dh, c1 = (F)9 / (F)8, c2 = (F)-1 / (F)24;
        par_for(nabc + 1, nzt - nfs, [&](int k) {
            for (int j = nabc + 1; j <= nyt - 2; ++j)
                for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                    F xl = lam1[I3(i, j, k)], xm = mu1[I3(i, j, k)];
                    F a = xl + (F)2 * xm, b = xl;
                    F dxu = c1 * (u1[I3(i + 1, j, k)] - u1[I3(i, j, k)]) + c2 * (u1[I3(i + 2, j, k)] - u1[I3(i - 1, j, k)]);
                    F dyv1 = c1 * (v1[I3(i, j, k)] - v1[I3(i, j - 1, k)]);
                    F dyv2 = c2 * (v1[I3(i, j + 1, k)] - v1[I3(i, j - 2, k)]);
                    F dzw1 = c1 * (w1[I3(i, j, k)] - w1[I3(i, j, k - 1)]);
                    F dzw2 = c2 * (w1[I3(i, j, k + 1)] - w1[I3(i, j, k - 2)]);
                    F dxu1 = c1 * (u1[I3(i + 1, j, k)] - u1[I3(i, j, k)]);
                    F dxu2 = c2 * (u1[I3(i + 2, j, k)] - u1[I3(i - 1, j, k)]);
                    xx[I3(i, j, k)] = xx[I3(i, j, k)] + dth * a * (dxu) + dth * b * (dyv1 + dyv2 + dzw1 + dzw2);
                    yy[I3(i, j, k)] = yy[I3(i, j, k)] + dth * a * (dyv1 + dyv2) + dth * b * (dxu1 + dxu2 + dzw1 + dzw2);
                    zz[I3(i, j, k)] = zz[I3(i, j, k)] + dth * a * (dzw1 + dzw2) + dth * b * (dxu1 + dxu2 + dyv1 + dyv2);
                    F xmu = (F)0.5 * (mu1[I3(i, j, k)] + mu1[I3(i, j + 1, k)]);
                    xy[I3(i, j, k)] = xy[I3(i, j, k)] + dth * xmu * (
                        c1 * (u1[I3(i, j + 1, k)] - u1[I3(i, j, k)]) + c2 * (u1[I3(i, j + 2, k)] - u1[I3(i, j - 1, k)]) +
                        c1 * (v1[I3(i, j, k)] - v1[I3(i - 1, j, k)]) + c2 * (v1[I3(i + 1, j, k)] - v1[I3(i - 2, j, k)]));
                    xmu = (F)0.5 * (mu1[I3(i, j, k)] + mu1[I3(i, j, k + 1)]);
                    xz[I3(i, j, k)] = xz[I3(i, j, k)] + dth * xmu * (
                        c1 * (u1[I3(i, j, k + 1)] - u1[I3(i, j, k)]) + c2 * (u1[I3(i, j, k + 2)] - u1[I3(i, j, k - 1)]) +
                        c1 * (w1[I3(i, j, k)] - w1[I3(i - 1, j, k)]) + c2 * (w1[I3(i + 1, j, k)] - w1[I3(i - 2, j, k)]));
                    xmu = (F)0.5 * (mu1[I3(i, j, k)] + mu1[I3(i + 1, j + 1, k + 1)]);
                    yz[I3(i, j, k)] = yz[I3(i, j, k)] + dth * xmu * (
                        c1 * (v1[I3(i, j, k + 1)] - v1[I3(i, j, k)]) + c2 * (v1[I3(i, j, k + 2)] - v1[I3(i, j, k - 1)]) +
                        c1 * (w1[I3(i, j + 1, k)] - w1[I3(i, j, k)]) + c2 * (w1[I3(i, j + 2, k)] - w1[I3(i, j - 1, k)]));
                }
        });
    }

    // strbnd -> sxx, sxy0, sxz0, syz0 at j=nyt-1 + xy,yz mirror  fd3d_deriv.f90:777-1012
    void strbnd() {
        const F dth = dt / dh, dth2 = (F)0.5 * dt / dh;
        const int j = nyt - 1;
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                F xl = lam1[I3(i, j, k)], xm = mu1[I3(i, j, k)];
                F a = xl + (F)2 * xm, b = xl;
                F du = u1[I3(i + 1, j, k)] - u1[I3(i, j, k)];
                xx[I3(i, j, k)] = xx[I3(i, j, k)] + dth * a * (du) +
                                  dth * b * (v1[I3(i, j, k)] - v1[I3(i, j - 1, k)] + w1[I3(i, j, k)] - w1[I3(i, j, k - 1)]);
                yy[I3(i, j, k)] = yy[I3(i, j, k)] + dth * a * (v1[I3(i, j, k)] - v1[I3(i, j - 1, k)]) +
                                  dth * b * (u1[I3(i + 1, j, k)] - u1[I3(i, j, k)] + w1[I3(i, j, k)] - w1[I3(i, j, k - 1)]);
                zz[I3(i, j, k)] = zz[I3(i, j, k)] + dth * a * (w1[I3(i, j, k)] - w1[I3(i, j, k - 1)]) +
                                  dth * b * (u1[I3(i + 1, j, k)] - u1[I3(i, j, k)] + v1[I3(i, j, k)] - v1[I3(i, j - 1, k)]);
                F xmu = mu1[I3(i, j, k)] + mu1[I3(i, j + 1, k)];
                xy[I3(i, j, k)] = xy[I3(i, j, k)] + dth2 * xmu * (u1[I3(i, j + 1, k)] - u1[I3(i, j, k)] + v1[I3(i, j, k)] - v1[I3(i - 1, j, k)]);
                xmu = mu1[I3(i, j, k)] + mu1[I3(i, j, k + 1)];
                xz[I3(i, j, k)] = xz[I3(i, j, k)] + dth2 * xmu * (u1[I3(i, j, k + 1)] - u1[I3(i, j, k)] + w1[I3(i, j, k)] - w1[I3(i - 1, j, k)]);
                xmu = mu1[I3(i, j, k)] + mu1[I3(i + 1, j + 1, k + 1)];
                yz[I3(i, j, k)] = yz[I3(i, j, k)] + dth2 * xmu * (v1[I3(i, j, k + 1)] - v1[I3(i, j, k)] + w1[I3(i, j + 1, k)] - w1[I3(i, j, k)]);
            }
        for (int i = 1; i <= nxt; ++i)
            for (int k = 1; k <= nzt; ++k) {
                xy[I3(i, nyt, k)] = xy[I3(i, nyt - 1, k)];
                yz[I3(i, nyt, k)] = yz[I3(i, nyt - 1, k)];
            }
    }

    // tasxz (sxz1 at j=nyt) and tasii  fd3d_deriv.f90:677-722,1239-1314
    void tasxz_tasii() {
        const F dth2 = (F)0.5 * dt / dh, dth = dt / dh, c1 = (F)9 / (F)8, c2 = (F)-1 / (F)24;
        const int j = nysc;
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                F xmu = mu1[I3(i, j, k)] + mu1[I3(i, j, k + 1)];
                xz[I3(i, j, k)] = xz[I3(i, j, k)] + dth2 * xmu * (
                    c1 * (u1[I3(i, j, k + 1)] - u1[I3(i, j, k)]) + c2 * (u1[I3(i, j, k + 2)] - u1[I3(i, j, k - 1)]) +
                    c1 * (w1[I3(i, j, k)] - w1[I3(i - 1, j, k)]) + c2 * (w1[I3(i + 1, j, k)] - w1[I3(i - 2, j, k)]));
            }
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                F xl = lam1[I3(i, j, k)], xm = mu1[I3(i, j, k)];
                F a = xl + (F)2 * xm, b = xl;
                F diff1 = c1 * (u1[I3(i + 1, j, k)] - u1[I3(i, j, k)]) + c2 * (u1[I3(i + 2, j, k)] - u1[I3(i - 1, j, k)]);
                F diff3 = c1 * (w1[I3(i, j, k)] - w1[I3(i, j, k - 1)]) + c2 * (w1[I3(i, j, k + 1)] - w1[I3(i, j, k - 2)]);
                const size_t p = I2(i, k);
                F vb = v1[I3(i, j - 1, k)];
                v1t[p] = vb - b * (diff1 + diff3) / ((F)2 * a);
                F dv = v1t[p] - vb;
                xx[I3(i, j, k)] = xx[I3(i, j, k)] + dth * a * (diff1) + dth * b * ((F)2 * dv + diff3);
                yy[I3(i, j, k)] = yy[I3(i, j, k)] + dth * a * (F)2 * dv + dth * b * (diff1 + diff3);
                zz[I3(i, j, k)] = zz[I3(i, j, k)] + dth * a * (diff3) + dth * b * (diff1 + (F)2 * dv);
            }
    }

    // pml_xyz  fd3d_deriv.f90:2304-2992 (strip 5: :2996-3143)
    void pml_xyz() {
        for (int s = 1; s <= nstrip; ++s) {
            Strip& st = S[s];
            const bool y3 = (s == 3);
            const int jn = y3 ? st.nye : st.nye + 1;  // normal-stress and xz loops reach nye+1 except in strip 3
            const std::vector<F>& oyxy = (s >= 3) ? st.oyS : st.oy;   // xy: omegay in strips 1,2; omegayS in 3-5
            const std::vector<F>& ozxz = (s >= 4) ? st.ozS : st.oz;   // xz,yz: omegazS in strips 4, 5
            par_for(st.nzb, st.nze, [&](int k) {
                for (int j = st.nyb; j <= jn; ++j)
                    for (int i = st.nxb; i <= st.nxe; ++i) {
                        int i2 = 1 - st.nxb + i, j2 = 1 - st.nyb + j, k2 = 1 - st.nzb + k;
                        size_t q = st.at(i2, j2, k2);
                        F xl = lam1[I3(i, j, k)], xm = mu1[I3(i, j, k)];
                        F a = xl + (F)2 * xm, b = xl;
                        F diff1 = u1[I3(i + 1, j, k)] - u1[I3(i, j, k)];
                        F diff2 = v1[I3(i, j, k)] - v1[I3(i, j - 1, k)];
                        F diff3 = w1[I3(i, j, k)] - w1[I3(i, j, k - 1)];
                        F ox = st.oxS[i2 - 1], oy = st.oy[j2 - 1], oz = st.oz[k2 - 1];
                        F pt;
                        pt = st.sxx[0][q] * ((F)1 - ox) + dt * a * diff1 / dh; st.sxx[0][q] = pt / ((F)1 + ox);
                        pt = st.sxx[1][q] * ((F)1 - oy) + dt * b * diff2 / dh; st.sxx[1][q] = pt / ((F)1 + oy);
                        pt = st.sxx[2][q] * ((F)1 - oz) + dt * b * diff3 / dh; st.sxx[2][q] = pt / ((F)1 + oz);
                        xx[I3(i, j, k)] = st.sxx[0][q] + st.sxx[1][q] + st.sxx[2][q];
                        pt = st.syy[0][q] * ((F)1 - ox) + dt * b * diff1 / dh; st.syy[0][q] = pt / ((F)1 + ox);
                        pt = st.syy[1][q] * ((F)1 - oy) + dt * a * diff2 / dh; st.syy[1][q] = pt / ((F)1 + oy);
                        pt = st.syy[2][q] * ((F)1 - oz) + dt * b * diff3 / dh; st.syy[2][q] = pt / ((F)1 + oz);
                        yy[I3(i, j, k)] = st.syy[0][q] + st.syy[1][q] + st.syy[2][q];
                        pt = st.szz[0][q] * ((F)1 - ox) + dt * b * diff1 / dh; st.szz[0][q] = pt / ((F)1 + ox);
                        pt = st.szz[1][q] * ((F)1 - oy) + dt * b * diff2 / dh; st.szz[1][q] = pt / ((F)1 + oy);
                        pt = st.szz[2][q] * ((F)1 - oz) + dt * a * diff3 / dh; st.szz[2][q] = pt / ((F)1 + oz);
                        zz[I3(i, j, k)] = st.szz[0][q] + st.szz[1][q] + st.szz[2][q];
                    }
            });
            par_for(st.nzb, st.nze, [&](int k) {
                for (int j = st.nyb; j <= st.nye; ++j)
                    for (int i = st.nxb; i <= st.nxe; ++i) {
                        int i2 = 1 - st.nxb + i, j2 = 1 - st.nyb + j, k2 = 1 - st.nzb + k;
                        size_t q = st.at(i2, j2, k2);
                        F xmu = (mu1[I3(i, j, k)] + mu1[I3(i, j + 1, k)]) / (F)2;
                        F oy = oyxy[j2 - 1], ox = st.ox[i2 - 1];
                        F pt = st.sxy[0][q] * ((F)1 - oy) + dt * xmu * (u1[I3(i, j + 1, k)] - u1[I3(i, j, k)]) / dh;
                        st.sxy[0][q] = pt / ((F)1 + oy);
                        pt = st.sxy[1][q] * ((F)1 - ox) + dt * xmu * (v1[I3(i, j, k)] - v1[I3(i - 1, j, k)]) / dh;
                        st.sxy[1][q] = pt / ((F)1 + ox);
                        xy[I3(i, j, k)] = st.sxy[0][q] + st.sxy[1][q];
                    }
            });
            par_for(st.nzb, st.nze, [&](int k) {
                for (int j = st.nyb; j <= jn; ++j)
                    for (int i = st.nxb; i <= st.nxe; ++i) {
                        int i2 = 1 - st.nxb + i, j2 = 1 - st.nyb + j, k2 = 1 - st.nzb + k;
                        size_t q = st.at(i2, j2, k2);
                        F xmu = (mu1[I3(i, j, k)] + mu1[I3(i, j, k + 1)]) / (F)2;
                        F oz = ozxz[k2 - 1], ox = st.ox[i2 - 1];
                        F pt = st.sxz[0][q] * ((F)1 - oz) + dt * xmu * (u1[I3(i, j, k + 1)] - u1[I3(i, j, k)]) / dh;
                        st.sxz[0][q] = pt / ((F)1 + oz);
                        pt = st.sxz[1][q] * ((F)1 - ox) + dt * xmu * (w1[I3(i, j, k)] - w1[I3(i - 1, j, k)]) / dh;
                        st.sxz[1][q] = pt / ((F)1 + ox);
                        xz[I3(i, j, k)] = st.sxz[0][q] + st.sxz[1][q];
                    }
            });
            par_for(st.nzb, st.nze, [&](int k) {
                for (int j = st.nyb; j <= st.nye; ++j)
                    for (int i = st.nxb; i <= st.nxe; ++i) {
                        int i2 = 1 - st.nxb + i, j2 = 1 - st.nyb + j, k2 = 1 - st.nzb + k;
                        size_t q = st.at(i2, j2, k2);
                        F xmu = (mu1[I3(i, j, k)] + mu1[I3(i + 1, j + 1, k + 1)]) / (F)2;
                        F oz = ozxz[k2 - 1], oy = oyxy[j2 - 1];
                        F pt = st.syz[0][q] * ((F)1 - oz) + dt * xmu * (v1[I3(i, j, k + 1)] - v1[I3(i, j, k)]) / dh;
                        st.syz[0][q] = pt / ((F)1 + oz);
                        pt = st.syz[1][q] * ((F)1 - oy) + dt * xmu * (w1[I3(i, j + 1, k)] - w1[I3(i, j, k)]) / dh;
                        st.syz[1][q] = pt / ((F)1 + oy);
                        yz[I3(i, j, k)] = st.syz[0][q] + st.syz[1][q];
                    }
            });
            // zero xz/yz aux at the top row (fd3d_deriv.f90:2471-2491, 2649-2669, 2826-2846), not under FSPACE
            if (s <= 3 && !fspace) {
                int k2 = st.nze - st.nzb + 1;
                for (int i2 = 1; i2 <= st.ni; ++i2) {
                    for (int j2 = 1; j2 <= (y3 ? st.nye - st.nyb + 1 : st.nye - st.nyb + 2); ++j2) {
                        st.sxz[0][st.at(i2, j2, k2)] = 0; st.sxz[1][st.at(i2, j2, k2)] = 0;
                    }
                    for (int j2 = 1; j2 <= st.nye - st.nyb + 1; ++j2) {
                        st.syz[0][st.at(i2, j2, k2)] = 0; st.syz[1][st.at(i2, j2, k2)] = 0;
                    }
                }
            }
        }
    }

    // fres  fd3d_deriv.f90:1067-1104, called with nzt-nfs
    void fres() {
        const int n = nzt - nfs;
        for (int j = 1; j <= nyt; ++j)
            for (int i = 1; i <= nxt; ++i) {
                zz[I3(i, j, n + 1)] = -zz[I3(i, j, n)];
                zz[I3(i, j, n + 2)] = -zz[I3(i, j, n - 1)];
                xz[I3(i, j, n + 1)] = -xz[I3(i, j, n - 1)];
                xz[I3(i, j, n + 2)] = -xz[I3(i, j, n - 2)];
                yz[I3(i, j, n + 1)] = -yz[I3(i, j, n - 1)];
                yz[I3(i, j, n + 2)] = -yz[I3(i, j, n - 2)];
                xz[I3(i, j, n)] = 0;
                yz[I3(i, j, n)] = 0;
            }
    }

    // ------------------------------------------------------------------ fault BC
    // traction  fd3d_theo.f90:233-308 (FSPACE top row :260-283)
    void traction() {
        const F c1 = (F)9 / (F)8, c2 = (F)-1 / (F)24, dht = dh / dt;
        const int j = nysc;
        auto trac = [&](int i, int k, bool top) {
            const size_t p = I2(i, k);
            F pdz;
            if (!top)
                pdz = (c1 * (xz[I3(i + 1, j, k)] - xz[I3(i, j, k)]) + c2 * (xz[I3(i + 2, j, k)] - xz[I3(i - 1, j, k)])) / (F)2 +
                      (c1 * (zz[I3(i, j, k + 1)] - zz[I3(i, j, k)]) + c2 * (zz[I3(i, j, k + 2)] - zz[I3(i, j, k - 1)])) / (F)2 -
                      yz[I3(i, j - 1, k)];
            else
                pdz = ((xz[I3(i + 1, j, k - 1)] - xz[I3(i, j, k - 1)]) / ((F)2 * (F)4) +
                       (zz[I3(i, j, k + 1)] - zz[I3(i, j, k)]) / ((F)2 * (F)2) - yz[I3(i, j - 1, k - 1)] / (F)4);
            avdz[p] = damp_s * (pdz - avdz[p]);
            RFz[p] = pdz + avdz[p];
            if (!top) tz[p] = -RFz[p] - (F)0.5 * d1[I3(i, j, k)] * dht * w1[I3(i, j, k)];
            else      tz[p] = -RFz[p] - (F)0.5 * d1[I3(i, j, k)] * dht * w1[I3(i, j, k)] / (F)2;
            avdz[p] = pdz;
            F pdx = (c1 * (xx[I3(i, j, k)] - xx[I3(i - 1, j, k)]) + c2 * (xx[I3(i + 1, j, k)] - xx[I3(i - 2, j, k)])) / (F)2 +
                    (c1 * (xz[I3(i, j, k)] - xz[I3(i, j, k - 1)]) + c2 * (xz[I3(i, j, k + 1)] - xz[I3(i, j, k - 2)])) / (F)2 -
                    xy[I3(i, j - 1, k)];
            avdx[p] = damp_s * (pdx - avdx[p]);
            RFx[p] = pdx + avdx[p];
            tx[p] = -RFx[p] - (F)0.5 * d1[I3(i, j, k)] * dht * u1[I3(i, j, k)];
            avdx[p] = pdx;
        };
        for (int k = nabc + 1; k <= nzt - nfs - 1; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) trac(i, k, false);
        if (fspace) {  // FSPACE: the top row takes the interior formula, no ghost row (fd3d_theo.f90:260-283)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) trac(i, nzt - nfs, false);
            return;
        }
        for (int i = nabc + 1; i <= nxt - nabc; ++i) trac(i, nzt - nfs, true);
        for (int i = nabc + 1; i <= nxt - nabc; ++i) {
            tx[I2(i, nzt - 1)] = +tx[I2(i, nzt - 2)];
            tz[I2(i, nzt - 1)] = -tz[I2(i, nzt - 3)];
        }
    }

    // |T| at staggered nodes, friction, slip, rupture time, outputs  fd3d_theo.f90:313-467
    void friction(A time) {
        const int j = nysc;
        const A rup_tresh = (A)1.e-3;
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                F tint = (tx[p] + T0X[p] + tx[I2(i + 1, k)] + T0X[I2(i + 1, k)] + tx[I2(i, k + 1)] + T0X[I2(i, k + 1)] +
                          tx[I2(i + 1, k + 1)] + T0X[I2(i + 1, k + 1)]) / (F)4;
                F sz = tz[p] + T0Z[p];
                tabsZ[p] = std::sqrt(tint * tint + sz * sz);
                tint = (tz[p] + T0Z[p] + tz[I2(i - 1, k)] + T0Z[I2(i - 1, k)] + tz[I2(i, k - 1)] + T0Z[I2(i, k - 1)] +
                        tz[I2(i - 1, k - 1)] + T0Z[I2(i - 1, k - 1)]) / (F)4;
                F sx = tx[p] + T0X[p];
                tabsX[p] = std::sqrt(sx * sx + tint * tint);
            }
        // Z nodes  fd3d_theo.f90:326-373
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                F tabs = tabsZ[p];
                uZ[p] = (u1[I3(i, j, k)] + u1[I3(i + 1, j, k)] + u1[I3(i, j, k + 1)] + u1[I3(i + 1, j, k + 1)]) / (F)4;
                F w = w1[I3(i, j, k)];
                F u1out = -std::sqrt(w * w + uZ[p] * uZ[p]);
                if (law == FD3D_LAW_FVW) {
                    A a = (A)aZ[p];
                    A s1 = (A)2 * (std::fabs((A)w) + std::fabs(wini)), s2 = (A)2 * (std::fabs((A)uZ[p]) + std::fabs(uini));
                    A sr = std::sqrt(s1 * s1 + s2 * s2);
                    A flv = f0 - ((A)bZ[p] - a) * std::log(sr / v0);
                    A fss = (A)fwZ[p] + (flv - (A)fwZ[p]) / std::pow((A)1 + std::pow(sr / (A)vwZ[p], 8), (A)1 / (A)8);
                    A psiss = a * (std::log(std::sinh(fss / a)) + std::log((A)2 * v0 / sr));
                    psiZ[p] = (psiZ[p] - psiss) * std::exp(-sr * dtA / (A)Dc[p]) + psiss;
                    A fric = Sn * a * std::asinh(sr * std::exp(psiZ[p] / a) / ((A)2 * v0));
                    distZ[p] = distZ[p] - (A)2 * (A)u1out * dtA;
                    schangeZ[p] = (F)fric;
                    psiout[p] = psiZ[p];
                    if (std::fabs((A)2 * (A)u1out) > rup_tresh) {
                        if (ruptime[p] != (A)1.e4) rise[p] = time;
                        if (ruptime[p] == (A)1.e4) ruptime[p] = time;
                    }
                } else {
                    A fric;
                    A dz = distZ[p], dcz = (A)DcZ[p];
                    if (dz <= dcz) fric = (A)peakZ[p] * ((A)1 - dz / dcz) + (A)dynZ[p] * dz / dcz + (A)coh[p];
                    else           fric = (A)dynZ[p] + (A)coh[p];
                    if ((A)tabs >= fric) {
                        distZ[p] = distZ[p] - (A)2 * (A)u1out * dtA;
                        tz[p] = (F)(((A)tz[p] + (A)T0Z[p]) * fric / (A)tabs - (A)T0Z[p]);
                        if (-(A)2 * (A)u1out > rup_tresh) {
                            if (ruptime[p] != (A)1.e4) rise[p] = time;
                            if (ruptime[p] == (A)1.e4) ruptime[p] = time;
                        }
                    }
                }
                slipZ[p] = slipZ[p] - (A)2 * (A)w * dtA;
                slipX[p] = slipX[p] - (A)2 * (A)uZ[p] * dtA;
                if (sliptime[p] == (A)1.e4 && distZ[p] > (A)Dc[p]) sliptime[p] = time;
            }
        // X nodes  fd3d_theo.f90:375-410
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                F tabs = tabsX[p];
                wX[p] = (w1[I3(i, j, k)] + w1[I3(i - 1, j, k)] + w1[I3(i, j, k - 1)] + w1[I3(i - 1, j, k - 1)]) / (F)4;
                F u = u1[I3(i, j, k)];
                F u1out = -std::sqrt(wX[p] * wX[p] + u * u);
                if (law == FD3D_LAW_FVW) {
                    A a = (A)aX[p];
                    A s1 = (A)2 * (std::fabs((A)wX[p]) + std::fabs(wini)), s2 = (A)2 * (std::fabs((A)u) + std::fabs(uini));
                    A sr = std::sqrt(s1 * s1 + s2 * s2);
                    A flv = f0 - ((A)bX[p] - a) * std::log(sr / v0);
                    A fss = (A)fwX[p] + (flv - (A)fwX[p]) / std::pow((A)1 + std::pow(sr / (A)vwX[p], 8), (A)1 / (A)8);
                    A psiss = a * (std::log(std::sinh(fss / a)) + std::log((A)2 * v0 / sr));
                    psiX[p] = (psiX[p] - psiss) * std::exp(-sr * dtA / (A)Dc[p]) + psiss;
                    A fric = Sn * a * std::asinh(sr * std::exp(psiX[p] / a) / ((A)2 * v0));
                    distX[p] = distX[p] - (A)2 * (A)u1out * dtA;
                    schangeX[p] = (F)fric;
                } else {
                    A fric;
                    A dx = distX[p], dcx = (A)DcX[p];
                    if (dx <= (A)Dc[p]) fric = (A)peakX[p] * ((A)1 - dx / dcx) + (A)dynX[p] * dx / dcx + (A)coh[p];
                    else                fric = (A)dynX[p] + (A)coh[p];
                    if ((A)tabs >= fric) {
                        distX[p] = distX[p] - (A)2 * (A)u1out * dtA;
                        tx[p] = (F)(((A)tx[p] + (A)T0X[p]) * fric / (A)tabs - (A)T0X[p]);
                    }
                }
            }
        // output planes  fd3d_theo.f90:413-453
        for (int k = nabc + 1; k <= nzt - nfs; ++k) {
            const bool top = (k == nzt - nfs);
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                F U = u1[I3(i, j, k)], U2 = u1[I3(i + 1, j, k)];
                F W = w1[I3(i, j, k)];
                if (!top) {
                    F U3 = u1[I3(i, j, k + 1)], U4 = u1[I3(i + 1, j, k + 1)];
                    sliprateoutX[p] = ((F)-2 * U - (F)2 * U2 - (F)2 * U3 - (F)2 * U4) / (F)4;
                    sliprateoutZ[p] = (F)-2 * W;
                    if (law != FD3D_LAW_FVW) {
                        schangeZ[p] = tz[p] + T0Z[p];
                        schangeX[p] = (tx[p] + T0X[p] + tx[I2(i + 1, k)] + T0X[I2(i + 1, k)] + tx[I2(i, k + 1)] + T0X[I2(i, k + 1)] +
                                       tx[I2(i + 1, k + 1)] + T0X[I2(i + 1, k + 1)]) / (F)4;
                    }
                } else {
                    sliprateoutZ[p] = (F)-2 * W;
                    if (law == FD3D_LAW_FVW) {
                        sliprateoutX[p] = ((F)-2 * U - (F)2 * U2) / (F)4;
                    } else {
                        schangeZ[p] = tz[p] + T0Z[p];
                        schangeX[p] = (tx[p] + T0X[p] + tx[I2(i + 1, k)] + T0X[I2(i + 1, k)]) / (F)2;
                        sliprateoutX[p] = ((F)-2 * U - (F)2 * U2) / (F)2;
                    }
                }
            }
        }
        for (int s = 0; s < nst; ++s) {  // fd3d_theo.f90:456-467
            size_t q = I3(staX[s], staY[s], staZ[s]);
            seis[3 * s + 0] = u1[q]; seis[3 * s + 1] = v1[q]; seis[3 * s + 2] = w1[q];
        }
    }

    // TPV103/104 nucleation ramp  fd3d_theo.f90:487-542
    void nucleate(A time) {
        if (!nucleation) return;
        A th = time - dtA / (A)2;
        if (!(th <= TT2)) return;
        A GT = (th < TT2) ? std::exp((th - TT2) * (th - TT2) / (th * (th - (A)2 * TT2))) : (A)1;
        const A dhA = (A)dh;
        for (int k = nabc - 1; k <= nzt - nfs; ++k)
            for (int i = nabc - 1; i <= nxt - nabc; ++i) {
                A hx = (A)i * dhA, hz = (A)k * dhA;
                A rr = (hx - hx0) * (hx - hx0) + (hz - hz0) * (hz - hz0);
                A FXZ = (rr < RR2 - dhA) ? std::exp(rr / (rr - RR2 - dhA)) : (A)0;
                // nucleation 1: the reference's form; 2: the bump over the node's own initial T0X
                const A base = nucleation == 2 ? (A)T0Xb[I2(i, k)] : strinixI;
                T0X[I2(i, k)] = (F)(base + perturb * FXZ * GT);
            }
    }

    // one pass of the time loop  fd3d_theo.f90:187-602
    void step() {
        t_cells = (long long)nxt * nyt * nzt;
        ++it;
        A time = (A)it * dtA;
        std::fill(sliprateoutX.begin(), sliprateoutX.end(), (F)0);
        std::fill(sliprateoutZ.begin(), sliprateoutZ.end(), (F)0);
        std::fill(schangeX.begin(), schangeX.end(), (F)0);
        std::fill(schangeZ.begin(), schangeZ.end(), (F)0);
        std::fill(psiout.begin(), psiout.end(), (A)0);
        dvel(); bnd2d(); tasuw(); pml_uvw();
        if (!fspace) fuvw();  // fd3d_theo.f90:213-215
        dstres(); strbnd(); tasxz_tasii(); pml_xyz();
        if (!fspace) fres();  // fd3d_theo.f90:225-227
        traction(); friction(time); nucleate(time);
        // MomentRate(k) += sqrt(srX^2 + srZ^2)*mu1(i,nysc,j)*dh*dh/(dtseis/dt), with dtseis = dt
        // one bin per step (fd3d_theo.f90:560,574-578), in the accumulator type
        A mr = 0;
        for (int j = nabc + 1; j <= nzt - nfs; ++j)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const A x = (A)sliprateoutX[I2(i, j)], z = (A)sliprateoutZ[I2(i, j)];
                mr = mr + std::sqrt(x * x + z * z) * (A)mu1[I3(i, nysc, j)] * (A)dh * (A)dh;
            }
        moment_rate.push_back(mr);
    }

    // readinversionresult + inversion_modeltofd3d (fd3d_init.f90:802-857): the control
    // points (nli x nwi, Fortran order) of prestress T0I, static strength TsI (times the
    // normal stress) and Dc, bilinearly interpolated onto the interior fault plane in
    // `real`; dynamic strength and cohesion 0; then interp_fric through set_fault.
    void set_fault_model(int nli, int nwi, const double* T0Id, const double* TsId, const double* DcId, double dipd,
                         int dipslip) {
        const size_t n2 = tx.size();
        std::vector<F> T0I(T0Id, T0Id + (size_t)nli * nwi), TsI(TsId, TsId + (size_t)nli * nwi),
            DcI(DcId, DcId + (size_t)nli * nwi);
        auto C2 = [&](const std::vector<F>& a, int ii, int kk) { return a[(size_t)(ii - 1) + (size_t)nli * (kk - 1)]; };
        const F pi = (F)3.1415926535, dip = (F)dipd;
        auto normstress = [&](int j) {  // fd3d_init.f90:77-86
            const F c = dipslip ? (F)8520. : (F)16200.;
            return std::max((F)1.e5, c * dh * (F)(nzt - nfs - j) * (F)std::sin(dip / (F)180. * pi));
        };
        std::vector<double> sX(n2, 0.0), sZ(n2, 0.0), pk(n2, 0.0), dy(n2, 0.0), dc(n2, 0.0), ch(n2, 0.0);
        const F DL = dh * (F)(nxt - 2 * nabc) / (F)(nli - 1);
        const F DW = dh * (F)(nzt - nfs - nabc) / (F)(nwi - 1);
        for (int k = nabc + 1; k <= nzt - nfs; ++k) {
            const F ZS = dh * (F)(k - 1 - nabc);
            const int kk = (int)(ZS / DW) + 1;
            const F u = (ZS - DW * (F)(kk - 1)) / DW;
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const F XS = dh * (F)(i - 1 - nabc);
                const int ii = (int)(XS / DL) + 1;
                const F t = (XS - DL * (F)(ii - 1)) / DL;
                auto bil = [&](const std::vector<F>& a) {
                    return ((F)1 - t) * ((F)1 - u) * C2(a, ii, kk) + t * ((F)1 - u) * C2(a, ii + 1, kk) +
                           t * u * C2(a, ii + 1, kk + 1) + ((F)1 - t) * u * C2(a, ii, kk + 1);
                };
                const size_t p = I2(i, k);
                const F t0 = bil(T0I);
                if (dipslip) sZ[p] = (double)t0; else sX[p] = (double)t0;
                pk[p] = (double)(bil(TsI) * normstress(k));
                dc[p] = (double)bil(DcI);
            }
        }
        fd3d_fault f{};
        f.striniX = sX.data(); f.striniZ = sZ.data(); f.Dc = dc.data();
        f.peak_xz = pk.data(); f.dyn_xz = dy.data(); f.coh = ch.data();
        set_fault(f);
    }

    // post-loop quantities  fd3d_theo.f90:604-605, 660-686, 710-749:
    // out = {average rupture speed, seismic moment, rupture area (never assigned by the
    // reference, 0), average stress drop}; rvel, czone planes (nxt*nzt, 0 outside)
    void post(double* out, double* rvel, double* czone) const {
        const A d = (A)dh;
        A m0 = 0, numer = 0, denom = 0, sd = 0;
        std::fill(rvel, rvel + tx.size(), 0.0);
        std::fill(czone, czone + tx.size(), 0.0);
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                const A slip = std::sqrt(slipX[p] * slipX[p] + slipZ[p] * slipZ[p]);
                m0 = m0 + slip * (A)mu1[I3(i, nysc, k)] * (A)(dh * dh);  // dh*dh in `real`
                const A dzs = (A)(F)(schangeZ[p] - T0Z[p]), dxs = (A)(F)(schangeX[p] - T0X[p]);
                numer = numer + dzs * slipZ[p] + dxs * slipX[p];
                denom = denom + slip;
                sd = (denom != 0) ? -(numer / denom) : (A)0;
            }
        A tint = 0, tint2 = 0;
        const A none = (A)1.e4;
        for (int k = nabc + 1; k <= nzt - nfs; ++k)
            for (int i = nabc + 1; i <= nxt - nabc; ++i) {
                const size_t p = I2(i, k);
                A cz = 0, rv = 0;
                const A r0 = ruptime[p], rxp = ruptime[I2(i + 1, k)], rzp = ruptime[I2(i, k + 1)];
                const A rxm = ruptime[I2(i - 1, k)], rzm = ruptime[I2(i, k - 1)];
                if (r0 != none && rxp != none && rzp != none && rxm != none && rzm != none) {
                    if (sliptime[p] != none) {
                        const A den = std::sqrt((rxp - r0) * (rxp - r0) + (rzp - r0) * (rzp - r0)) +
                                      std::sqrt((r0 - rxm) * (r0 - rxm) + (r0 - rzm) * (r0 - rzm));
                        if (den != 0) {
                            rv = (A)2 * d / den;
                            const A slip = std::sqrt(slipX[p] * slipX[p] + slipZ[p] * slipZ[p]);
                            tint = tint + rv * slip;
                            tint2 = tint2 + slip;
                        }
                        cz = rv * (sliptime[p] - r0);
                    }
                }
                rvel[p] = (double)rv;
                czone[p] = (double)cz;
            }
        out[0] = (double)(tint / tint2);
        out[1] = (double)m0;
        out[2] = 0.0;
        out[3] = (double)sd;
    }
};

struct Handle {
    int variant;
    void* o;
};

template <class F, class A> Oracle<F, A>* O(Handle* h) { return static_cast<Oracle<F, A>*>(h->o); }

#define DISPATCH(h, ...)                                                          \
    do {                                                                          \
        if ((h)->variant == 0) { auto* o = O<float, double>(h); __VA_ARGS__; }    \
        else if ((h)->variant == 1) { auto* o = O<double, double>(h); __VA_ARGS__; } \
        else { auto* o = O<float, float>(h); __VA_ARGS__; }                       \
    } while (0)

template <class T> void to_double(const std::vector<T>& v, double* out) {
    for (size_t q = 0; q < v.size(); ++q) out[q] = (double)v[q];
}

}  // namespace

extern "C" {

void* oracle_create(const fd3d_params* p, int variant) {
    if (!p || p->nxt < 2 * p->nabc + 5 || p->nyt < p->nabc + 5 || p->nzt < p->nabc + p->nfs + 5 || p->nabc < 3) return nullptr;
    if ((p->fspace != 0 && p->fspace != 1) || p->nfs != (p->fspace ? p->nabc : 2)) return nullptr;
    Handle* h = new Handle{variant, nullptr};
    if (variant == 0) h->o = new Oracle<float, double>(*p);
    else if (variant == 1) h->o = new Oracle<double, double>(*p);
    else h->o = new Oracle<float, float>(*p);
    return h;
}

void oracle_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    if (!h) return;
    DISPATCH(h, delete o);
    delete h;
}

int oracle_set_medium(void* hv, const double* l, const double* m, const double* d) {
    Handle* h = (Handle*)hv;
    DISPATCH(h, o->set_medium(l, m, d));
    return 0;
}

int oracle_set_fault(void* hv, const fd3d_fault* f) {
    Handle* h = (Handle*)hv;
    DISPATCH(h, o->set_fault(*f));
    return 0;
}

int oracle_reset(void* hv) {
    Handle* h = (Handle*)hv;
    DISPATCH(h, o->reset());
    return 0;
}

// Runs nsteps; if hist != NULL it receives, per step, the 5 output planes over the
// interior plane P (nxtT*nztT each, x fastest): sliprateX, sliprateZ, schangeX,
// schangeZ, psi.  If seis != NULL it receives nstations*3 values per step.
int oracle_step(void* hv, int nsteps, double* hist, double* seis) {
    Handle* h = (Handle*)hv;
    int fails = 0;
    DISPATCH(h, {
        const int nxT = o->nxt - 2 * o->nabc, nzT = o->nzt - o->nfs - o->nabc;
        const size_t plane = (size_t)nxT * nzT;
        for (int s = 0; s < nsteps; ++s) {
            o->step();
            if (hist) {
                double* base = hist + (size_t)s * 5 * plane;
                for (int k = o->nabc + 1; k <= o->nzt - o->nfs; ++k)
                    for (int i = o->nabc + 1; i <= o->nxt - o->nabc; ++i) {
                        size_t q = (size_t)(i - o->nabc - 1) + (size_t)nxT * (k - o->nabc - 1);
                        size_t p = o->I2(i, k);
                        base[0 * plane + q] = o->sliprateoutX[p];
                        base[1 * plane + q] = o->sliprateoutZ[p];
                        base[2 * plane + q] = o->schangeX[p];
                        base[3 * plane + q] = o->schangeZ[p];
                        base[4 * plane + q] = o->psiout[p];
                    }
            }
            if (seis)
                for (int q = 0; q < 3 * o->nst; ++q) seis[(size_t)s * 3 * o->nst + q] = o->seis[q];
        }
        fails = o->newton_fail;
    });
    return fails ? FD3D_ERR_NEWTON : 0;
}

int oracle_get_field(void* hv, int field, double* out) {
    Handle* h = (Handle*)hv;
    int rc = 0;
    DISPATCH(h, {
        switch (field) {
            case FD3D_FIELD_U: to_double(o->u1, out); break;
            case FD3D_FIELD_V: to_double(o->v1, out); break;
            case FD3D_FIELD_W: to_double(o->w1, out); break;
            case FD3D_FIELD_XX: to_double(o->xx, out); break;
            case FD3D_FIELD_YY: to_double(o->yy, out); break;
            case FD3D_FIELD_ZZ: to_double(o->zz, out); break;
            case FD3D_FIELD_XY: to_double(o->xy, out); break;
            case FD3D_FIELD_YZ: to_double(o->yz, out); break;
            case FD3D_FIELD_XZ: to_double(o->xz, out); break;
            default: rc = FD3D_ERR_ARG;
        }
    });
    return rc;
}

int oracle_get_plane(void* hv, int plane, double* out) {
    Handle* h = (Handle*)hv;
    int rc = 0;
    DISPATCH(h, {
        switch (plane) {
            case FD3D_PLANE_TX: to_double(o->tx, out); break;
            case FD3D_PLANE_TZ: to_double(o->tz, out); break;
            case FD3D_PLANE_SLIPX: to_double(o->slipX, out); break;
            case FD3D_PLANE_SLIPZ: to_double(o->slipZ, out); break;
            case FD3D_PLANE_RUPTIME: to_double(o->ruptime, out); break;
            case FD3D_PLANE_RISE: to_double(o->rise, out); break;
            case FD3D_PLANE_SLIPTIME: to_double(o->sliptime, out); break;
            case FD3D_PLANE_DISTX: to_double(o->distX, out); break;
            case FD3D_PLANE_DISTZ: to_double(o->distZ, out); break;
            case FD3D_PLANE_PSIX: to_double(o->psiX, out); break;
            case FD3D_PLANE_PSIZ: to_double(o->psiZ, out); break;
            case FD3D_PLANE_T0X: to_double(o->T0X, out); break;
            case FD3D_PLANE_T0Z: to_double(o->T0Z, out); break;
            case FD3D_PLANE_SCHANGEX: to_double(o->schangeX, out); break;
            case FD3D_PLANE_SCHANGEZ: to_double(o->schangeZ, out); break;
            default: rc = FD3D_ERR_ARG;
        }
    });
    return rc;
}

int oracle_set_fault_model(void* hv, int nli, int nwi, const double* T0I, const double* TsI, const double* DcI,
                           double dip, int dipslip) {
    Handle* h = (Handle*)hv;
    DISPATCH(h, o->set_fault_model(nli, nwi, T0I, TsI, DcI, dip, dipslip));
    return 0;
}

// moment rate of steps [from, from+n) (one value per step)
int oracle_moment_rate(void* hv, int from, int n, double* out) {
    Handle* h = (Handle*)hv;
    int rc = 0;
    DISPATCH(h, {
        if (from < 0 || from + n > (int)o->moment_rate.size()) rc = FD3D_ERR_ARG;
        else for (int q = 0; q < n; ++q) out[q] = (double)o->moment_rate[(size_t)(from + q)];
    });
    return rc;
}

// post-loop quantities (see Oracle::post)
int oracle_post(void* hv, double* out4, double* rvel, double* czone) {
    Handle* h = (Handle*)hv;
    DISPATCH(h, o->post(out4, rvel, czone));
    return 0;
}

int oracle_steps_done(void* hv) {
    Handle* h = (Handle*)hv;
    int n = 0;
    DISPATCH(h, n = o->it);
    return n;
}

int oracle_num_threads(void) { return oracle_threads(); }
void oracle_set_threads(int n) { g_threads = n; }

}  // extern "C"
