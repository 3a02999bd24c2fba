// fd3d_setup.h -- host-side set-up shared by the single-model context and the batch:
// parameter checks, the padded layout, the PML boxes/profiles (init_pml) and the
// per-step scalars in the field type.
#pragma once
#include <algorithm>
#include <vector>
#include "../../include/fd3d_gpu.h"
#include "fd3d_common.cuh"
#include "fd3d_kernels.cuh"

namespace fd3d {

inline
int validate_params(const fd3d_params* p) {
    if (!p) return FD3D_ERR_ARG;
    if (p->nabc < 3 || (p->fspace != 0 && p->fspace != 1)) return FD3D_ERR_ARG;
    if (p->nfs != (p->fspace ? p->nabc : 2)) return FD3D_ERR_ARG;  // fd3d_init.f90:161-165
    if (p->nxt < 2 * p->nabc + 4 || p->nyt < p->nabc + 4 || p->nzt < p->nabc + p->nfs + 4) return FD3D_ERR_ARG;
    if (!(p->dh > 0) || !(p->dt > 0)) return FD3D_ERR_ARG;
    if (p->law != FD3D_LAW_SW && p->law != FD3D_LAW_FVW) return FD3D_ERR_ARG;
    if (p->precision != FD3D_PREC_F32 && p->precision != FD3D_PREC_F64) return FD3D_ERR_ARG;
    if (p->nstations < 0 || p->nstations > FD3D_MAX_STATIONS) return FD3D_ERR_ARG;
    for (int s = 0; s < p->nstations; ++s)
        if (p->staX[s] < 1 || p->staX[s] > p->nxt || p->staY[s] < 1 || p->staY[s] > p->nyt || p->staZ[s] < 1 ||
            p->staZ[s] > p->nzt)
            return FD3D_ERR_ARG;
    if (p->history_stride < 0 || p->history_capacity < 0) return FD3D_ERR_ARG;
    if (p->vp_max > 0 && p->vp_max * p->dt / p->dh > 0.25) return FD3D_ERR_CFL;  // fd3d_init.f90:274-278
    return FD3D_OK;
}

inline Grid make_grid(const fd3d_params& p) {
    Grid g;
    g.nxt = p.nxt; g.nyt = p.nyt; g.nzt = p.nzt; g.nabc = p.nabc; g.nfs = p.nfs;
    g.fspace = p.fspace;
    g.off = (32 - (p.nabc % 32)) % 32;
    g.px = ((p.nxt + g.off + 31) / 32) * 32;
    g.plane = (long long)g.px * p.nyt;
    g.klo = 1; g.khi = p.nzt; g.kofs = 0; g.nzl = p.nzt;
    g.n3 = g.plane * p.nzt + 64;
    return g;
}

// Halo planes a z-slab stores on each side of the planes it owns: the 4th-order sweeps
// read two planes beyond their own, one more is kept as a margin.
constexpr int SLAB_HALO = 3;

// The grid of the z-slab that owns planes klo..khi of the model
inline Grid make_slab_grid(const fd3d_params& p, int klo, int khi) {
    Grid g = make_grid(p);
    g.klo = klo; g.khi = khi;
    const int kb = std::max(1, klo - SLAB_HALO), ke = std::min(p.nzt, khi + SLAB_HALO);
    g.kofs = kb - 1;
    g.nzl = ke - kb + 1;
    g.n3 = g.plane * g.nzl + 64;
    return g;
}

// A valid slab range: at least SLAB_MIN planes, and the top slab of a model with a free
// surface owns the two planes below it (the free-surface rows its fres and fuvw write stay
// out of every neighbour's halo).
constexpr int SLAB_MIN = 4;
inline bool slab_range_ok(const fd3d_params& p, int klo, int khi) {
    if (klo < 1 || khi > p.nzt || khi - klo + 1 < SLAB_MIN) return false;
    const int ks = p.nzt - p.nfs;
    if (khi >= ks && klo > ks - 2) return false;
    if (khi < p.nzt && khi >= ks - 2) return false;  // the slab above would not own ks-2 .. nzt
    return true;
}

// init_pml (fd3d_deriv.f90:1319-1493): strip boxes and damping profiles, in T.
template <class T>
void make_pml(const fd3d_params& p, PmlDesc& D, std::vector<Damp<T>>& prof) {
    const int nxt = p.nxt, nyt = p.nyt, nzt = p.nzt, nabc = p.nabc, nfs = p.nfs;
    const int bx[PML_MAXS][6] = {{2, nabc, nabc + 1, nyt - 1, nabc + 1, nzt - nfs},
                                 {nxt - nabc + 1, nxt - 1, nabc + 1, nyt - 1, nabc + 1, nzt - nfs},
                                 {2, nxt - 1, 2, nabc, nabc + 1, nzt - nfs},
                                 {2, nxt - 1, 2, nyt - 1, 2, nabc},
                                 {2, nxt - 1, 2, nyt - 1, nzt - nabc + 1, nzt - 1}};  // FSPACE top strip
    long long base = 0;
    prof.clear();
    D.ns = p.fspace ? 5 : 4;
    D.klo = 1;
    D.khi = p.nzt;
    D.cum[0] = 0;
    std::vector<std::vector<T>> ox(PML_MAXS), oxS(PML_MAXS), oy(PML_MAXS), oyS(PML_MAXS), oz(PML_MAXS), ozS(PML_MAXS);
    for (int s = 0; s < PML_MAXS; ++s) {
        if (s >= D.ns) {  // absent strip: empty range
            D.s[s] = D.s[s - 1];
            D.s[s].ncells = 0;
            D.cnt[s] = 0;
            D.cum[s + 1] = D.cum[s];
            continue;
        }
        Strip& S = D.s[s];
        S.nxb = bx[s][0]; S.nxe = bx[s][1]; S.nyb = bx[s][2]; S.nye = bx[s][3]; S.nzb = bx[s][4]; S.nze = bx[s][5];
        S.ni = S.nxe - S.nxb + 1; S.nk = S.nze - S.nzb + 1; S.nj1 = S.nye - S.nyb + 2;
        S.jend_uw = (s == 2) ? S.nye : S.nye + 1;
        S.ncells = (long long)S.ni * S.nj1 * S.nk;
        S.base = base;
        base += S.ncells;
        // every strip starts on a tile boundary, so a tile's cells share a strip
        D.cnt[s] = (long long)S.ni * (S.jend_uw - S.nyb + 1) * S.nk;
        D.cum[s + 1] = D.cum[s] + (D.cnt[s] + PML_TILE - 1) / PML_TILE * PML_TILE;
        S.rni = 1.0f / (float)S.ni;
        S.rnj = 1.0f / (float)(S.jend_uw - S.nyb + 1);
        S.fastdiv = D.cnt[s] < (1LL << 24);
        ox[s].assign(S.ni, (T)0); oxS[s].assign(S.ni, (T)0);
        oy[s].assign(S.nj1, (T)0); oyS[s].assign(S.nj1, (T)0);
        oz[s].assign(S.nk, (T)0); ozS[s].assign(S.nk, (T)0);
    }
    const T dt = (T)p.dt, dh = (T)p.dh;
    const T omegaM = (T)p.pml_fact * (T)p.pml_vp / ((T)2 * dh * (T)(nabc - 1));
    const int n = nabc - 1;
    std::vector<T> om(n), omR(n), omM(n), omRM(n);
    for (int i = 1; i <= n; ++i) {
        T r = (T)i / (T)n, rM = ((T)i - (T)0.5) / (T)n;
        om[i - 1] = (T)0.5 * dt * omegaM * ((r * r) * (r * r));
        omR[nabc - i - 1] = om[i - 1];
        omM[i - 1] = (T)0.5 * dt * omegaM * ((rM * rM) * (rM * rM));
        omRM[nabc - i - 1] = omM[i - 1];
    }
    for (int i = 1; i <= n; ++i) {  // 1-based reference index i -> 0-based i-1
        ox[0][i - 1] = omR[i - 1];  oxS[0][i - 1] = omRM[i - 1];
        ox[1][i - 1] = omM[i - 1];  oxS[1][i - 1] = om[i - 1];
        oy[2][i - 1] = omR[i - 1];  ox[2][i - 1] = omR[i - 1];  ox[2][nxt - i - 2] = omM[i - 1];
        oyS[2][i - 1] = omRM[i - 1]; oxS[2][i - 1] = omRM[i - 1]; oxS[2][nxt - i - 2] = om[i - 1];
        oz[3][i - 1] = omR[i - 1];  ox[3][i - 1] = omR[i - 1];  ox[3][nxt - i - 2] = omM[i - 1];
        oy[3][i - 1] = omR[i - 1];
        ozS[3][i - 1] = omRM[i - 1]; oxS[3][i - 1] = omRM[i - 1]; oxS[3][nxt - i - 2] = om[i - 1];
        oyS[3][i - 1] = omRM[i - 1];
        if (D.ns == 5) {  // fd3d_deriv.f90:1481-1490
            oz[4][i - 1] = omM[i - 1];  ox[4][i - 1] = omR[i - 1];  ox[4][nxt - i - 2] = omM[i - 1];
            oy[4][i - 1] = omR[i - 1];
            ozS[4][i - 1] = om[i - 1];  oxS[4][i - 1] = omRM[i - 1]; oxS[4][nxt - i - 2] = om[i - 1];
            oyS[4][i - 1] = omRM[i - 1];
        }
    }
    for (int s = 0; s < D.ns; ++s) {
        Strip& S = D.s[s];
        auto put = [&](const std::vector<T>& v) {
            const int o = (int)prof.size();
            for (T om : v) {
                Damp<T> e;
                e.o = om;
                e.m = (T)1 - om;
                e.p = (T)1 + om;
                e.r = div_pre_recip(e.p);
                prof.push_back(e);
            }
            return o;
        };
        S.ox_off = put(ox[s]); S.oxS_off = put(oxS[s]);
        S.oy_off = put(oy[s]); S.oyS_off = put(oyS[s]);
        S.oz_off = put(oz[s]); S.ozS_off = put(ozS[s]);
    }
}

// The PML sweeps update a split direction as p + inc where its strip class says the
// direction is never damped (split_mode, fd3d_kernels.cuh); that is exact only if every
// omega of that direction's profiles is zero over the strip.  Checked once per set-up.
template <class T>
bool pml_modes_hold(const PmlDesc& D, const std::vector<Damp<T>>& prof) {
    for (int s = 0; s < D.ns; ++s) {
        const Strip& S = D.s[s];
        const int C = pml_class(s);
        const int offs[3][2] = {{S.ox_off, S.oxS_off}, {S.oy_off, S.oyS_off}, {S.oz_off, S.ozS_off}};
        const int len[3] = {S.ni, S.nj1, S.nk};
        for (int dir = 0; dir < 3; ++dir) {
            if (split_mode(C, dir) != SPLIT_NEVER) continue;
            for (int v = 0; v < 2; ++v)
                for (int q = 0; q < len[dir]; ++q)
                    if (prof[(size_t)offs[dir][v] + q].o != (T)0) return false;
        }
    }
    return true;
}

template <class T>
StepConst<T> make_const(const fd3d_params& p) {
    StepConst<T> c;
    c.dt = (T)p.dt; c.dh = (T)p.dh;
    c.dth = c.dt / c.dh;
    c.dth2 = (T)0.5 * c.dt / c.dh;
    c.dht = c.dh / c.dt;
    c.damp_s = (T)p.damp_s;
    c.c1 = (T)9 / (T)8;
    c.c2 = (T)-1 / (T)24;
    c.rdh = div_pre_recip(c.dh);
    c.dtA = p.dt;
    c.dhA = (double)c.dh;
    c.dthA = c.dtA / c.dhA;
    return c;
}

}  // namespace fd3d
