// fd3d_opt.cuh -- tiled interior sweeps (the bulk of every time step).
//
// One CTA owns a 32 x 8 (x,y) column of the interior box and marches a chunk of z.
// Per z-plane the CTA stages the x/y neighbourhood of the fields it differentiates
// in shared memory (one coalesced load per element, halos included) and keeps the
// z-neighbours of its own column in a 4-deep register queue, so each field element
// is read from HBM once per sweep.  The arithmetic and its order are those of
// k_vel_interior / k_str_interior (uxx1/vyy1/wzz1 and dstres of fd3d_deriv.f90).
#pragma once
#include <algorithm>
#include "fd3d_common.cuh"
#include "fd3d_kernels.cuh"

namespace fd3d {

constexpr int TX = 32, TY = 8, NT = TX * TY;

// load an (H x W) window starting at (i0-ox, j0-oy) of plane k into s (row stride W)
template <class T, int H, int W>
__device__ __forceinline__ void stage(T* __restrict__ s, const T* __restrict__ a, const Grid& g, int i0, int j0,
                                      int ox, int oy, int k, int tid) {
    const long long base = g.at(1, 1, k);
#pragma unroll
    for (int e = tid; e < H * W; e += NT) {
        const int r = e / W, cc = e - r * W;
        const int gi = i0 - ox + cc, gj = j0 - oy + r;
        T v = (T)0;
        if (gi <= g.nxt && gj <= g.nyt) v = a[base + (gi - 1) + (long long)g.px * (gj - 1)];
        s[e] = v;
    }
}

template <class T>
__global__ void __launch_bounds__(NT) k_vel_interior_tiled(Grid g, Fields<T> f, StepConst<T> c, int kchunk) {
    __shared__ T s_xx[TY][36];
    __shared__ T s_xy[TY + 3][36];
    __shared__ T s_yy[TY + 3][TX];
    __shared__ T s_xz[TY][36];
    __shared__ T s_yz[TY + 3][TX];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = g.nabc + 1 + blockIdx.x * TX, j0 = g.nabc + 1 + blockIdx.y * TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool act = (i <= g.nxt - g.nabc) && (j <= g.nyt - 2);
    const int kb = g.kin_lo() + blockIdx.z * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const int ic = min(i, g.nxt), jc = min(j, g.nyt);
    const long long sz = g.plane;
    const long long pc = g.at(ic, jc, kb);
    const T* __restrict__ zz = f.zz; const T* __restrict__ xz = f.xz; const T* __restrict__ yz = f.yz;
    // z queues of the own column: zz(k-1..k+2), xz(k-2..k+1), yz(k-2..k+1)
    T zq0, zq1 = zz[pc - sz], zq2 = zz[pc], zq3 = zz[pc + sz];
    T xq0, xq1 = xz[pc - 2 * sz], xq2 = xz[pc - sz], xq3 = xz[pc];
    T yq0, yq1 = yz[pc - 2 * sz], yq2 = yz[pc - sz], yq3 = yz[pc];
    const T c1 = c.c1, c2 = c.c2, dth = c.dth;
    for (int k = kb; k <= ke; ++k) {
        const long long pk = pc + (long long)(k - kb) * sz;
        __syncthreads();
        stage<T, TY, 36>(&s_xx[0][0], f.xx, g, i0, j0, 2, 0, k, tid);
        stage<T, TY + 3, 36>(&s_xy[0][0], f.xy, g, i0, j0, 1, 2, k, tid);
        stage<T, TY + 3, TX>(&s_yy[0][0], f.yy, g, i0, j0, 0, 1, k, tid);
        stage<T, TY, 36>(&s_xz[0][0], f.xz, g, i0, j0, 1, 0, k, tid);
        stage<T, TY + 3, TX>(&s_yz[0][0], f.yz, g, i0, j0, 0, 2, k, tid);
        zq0 = zq1; zq1 = zq2; zq2 = zq3; zq3 = zz[pk + 2 * sz];
        xq0 = xq1; xq1 = xq2; xq2 = xq3; xq3 = xz[pk + sz];
        yq0 = yq1; yq1 = yq2; yq2 = yq3; yq3 = yz[pk + sz];
        __syncthreads();
        if (!act) continue;
        const T r = dth / f.d[pk];
        f.u[pk] = f.u[pk] + r * (c1 * (s_xx[ty][tx + 2] - s_xx[ty][tx + 1]) + c2 * (s_xx[ty][tx + 3] - s_xx[ty][tx]) +
                                 c1 * (s_xy[ty + 2][tx + 1] - s_xy[ty + 1][tx + 1]) + c2 * (s_xy[ty + 3][tx + 1] - s_xy[ty][tx + 1]) +
                                 c1 * (xq2 - xq1) + c2 * (xq3 - xq0));
        f.v[pk] = f.v[pk] + r * (c1 * (s_xy[ty + 2][tx + 2] - s_xy[ty + 2][tx + 1]) + c2 * (s_xy[ty + 2][tx + 3] - s_xy[ty + 2][tx]) +
                                 c1 * (s_yy[ty + 2][tx] - s_yy[ty + 1][tx]) + c2 * (s_yy[ty + 3][tx] - s_yy[ty][tx]) +
                                 c1 * (yq2 - yq1) + c2 * (yq3 - yq0));
        f.w[pk] = f.w[pk] + r * (c1 * (s_xz[ty][tx + 2] - s_xz[ty][tx + 1]) + c2 * (s_xz[ty][tx + 3] - s_xz[ty][tx]) +
                                 c1 * (s_yz[ty + 2][tx] - s_yz[ty + 1][tx]) + c2 * (s_yz[ty + 3][tx] - s_yz[ty][tx]) +
                                 c1 * (zq2 - zq1) + c2 * (zq3 - zq0));
    }
}

template <class T>
__global__ void __launch_bounds__(NT) k_str_interior_tiled(Grid g, Fields<T> f, StepConst<T> c, int kchunk) {
    // u, v, w of plane k with a 2-cell halo on every side: rows j0-2..j0+9, cols i0-2..i0+33
    __shared__ T s_u[TY + 4][36];
    __shared__ T s_v[TY + 4][36];
    __shared__ T s_w[TY + 4][36];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = g.nabc + 1 + blockIdx.x * TX, j0 = g.nabc + 1 + blockIdx.y * TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool act = (i <= g.nxt - g.nabc) && (j <= g.nyt - 2);
    const int kb = g.kin_lo() + blockIdx.z * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const int ic = min(i, g.nxt), jc = min(j, g.nyt);
    const long long sy = g.px, sz = g.plane;
    const long long pc = g.at(ic, jc, kb);
    const T* __restrict__ u = f.u; const T* __restrict__ v = f.v; const T* __restrict__ w = f.w;
    const T* __restrict__ mu = f.mu;
    // z queues: u(k-1..k+2), v(k-1..k+2), w(k-2..k+1), mu(k..k+1)
    T uq0, uq1 = u[pc - sz], uq2 = u[pc], uq3 = u[pc + sz];
    T vq0, vq1 = v[pc - sz], vq2 = v[pc], vq3 = v[pc + sz];
    T wq0, wq1 = w[pc - 2 * sz], wq2 = w[pc - sz], wq3 = w[pc];
    T mq0, mq1 = mu[pc];
    const T c1 = c.c1, c2 = c.c2, dth = c.dth;
    const int X = tx + 2, Y = ty + 2;
    for (int k = kb; k <= ke; ++k) {
        const long long pk = pc + (long long)(k - kb) * sz;
        __syncthreads();
        stage<T, TY + 4, 36>(&s_u[0][0], u, g, i0, j0, 2, 2, k, tid);
        stage<T, TY + 4, 36>(&s_v[0][0], v, g, i0, j0, 2, 2, k, tid);
        stage<T, TY + 4, 36>(&s_w[0][0], w, g, i0, j0, 2, 2, k, tid);
        uq0 = uq1; uq1 = uq2; uq2 = uq3; uq3 = u[pk + 2 * sz];
        vq0 = vq1; vq1 = vq2; vq2 = vq3; vq3 = v[pk + 2 * sz];
        wq0 = wq1; wq1 = wq2; wq2 = wq3; wq3 = w[pk + sz];
        mq0 = mq1; mq1 = mu[pk + sz];
        __syncthreads();
        if (!act) continue;
        const T xl = f.lam[pk], xm = mq0;
        const T a = xl + (T)2 * xm, b = xl;
        const T dxu1 = c1 * (s_u[Y][X + 1] - s_u[Y][X]), dxu2 = c2 * (s_u[Y][X + 2] - s_u[Y][X - 1]);
        const T dyv1 = c1 * (s_v[Y][X] - s_v[Y - 1][X]), dyv2 = c2 * (s_v[Y + 1][X] - s_v[Y - 2][X]);
        const T dzw1 = c1 * (wq2 - wq1), dzw2 = c2 * (wq3 - wq0);
        f.xx[pk] = f.xx[pk] + dth * a * (dxu1 + dxu2) + dth * b * (dyv1 + dyv2 + dzw1 + dzw2);
        f.yy[pk] = f.yy[pk] + dth * a * (dyv1 + dyv2) + dth * b * (dxu1 + dxu2 + dzw1 + dzw2);
        f.zz[pk] = f.zz[pk] + dth * a * (dzw1 + dzw2) + dth * b * (dxu1 + dxu2 + dyv1 + dyv2);
        T xmu = (T)0.5 * (xm + mu[pk + sy]);
        f.xy[pk] = f.xy[pk] + dth * xmu * (c1 * (s_u[Y + 1][X] - s_u[Y][X]) + c2 * (s_u[Y + 2][X] - s_u[Y - 1][X]) +
                                           c1 * (s_v[Y][X] - s_v[Y][X - 1]) + c2 * (s_v[Y][X + 1] - s_v[Y][X - 2]));
        xmu = (T)0.5 * (xm + mq1);
        f.xz[pk] = f.xz[pk] + dth * xmu * (c1 * (uq2 - uq1) + c2 * (uq3 - uq0) +
                                           c1 * (s_w[Y][X] - s_w[Y][X - 1]) + c2 * (s_w[Y][X + 1] - s_w[Y][X - 2]));
        xmu = (T)0.5 * (xm + mu[pk + 1 + sy + sz]);
        f.yz[pk] = f.yz[pk] + dth * xmu * (c1 * (vq2 - vq1) + c2 * (vq3 - vq0) +
                                           c1 * (s_w[Y + 1][X] - s_w[Y][X]) + c2 * (s_w[Y + 2][X] - s_w[Y - 1][X]));
    }
}

// Per-thread share of an (H x W) staging window: elements tid, tid+NT, ...  Loads go to
// registers first so that plane k+1 is in flight while plane k is computed.
template <class T, int H, int W>
struct Prefetch {
    static constexpr int N = (H * W + NT - 1) / NT;
    T r[N];
    __device__ __forceinline__ void load(const T* __restrict__ a, const Grid& g, int i0, int j0, int ox, int oy,
                                         int k, int tid) {
        const long long base = g.at(1, 1, k);
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const int e = tid + n * NT;
            T v = (T)0;
            if (e < H * W) {
                const int rr = e / W, cc = e - rr * W;
                const int gi = i0 - ox + cc, gj = j0 - oy + rr;
                if (gi <= g.nxt && gj <= g.nyt) v = a[base + (gi - 1) + (long long)g.px * (gj - 1)];
            }
            r[n] = v;
        }
    }
    __device__ __forceinline__ void store(T* s, int tid) const {
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const int e = tid + n * NT;
            if (e < H * W) s[e] = r[n];
        }
    }
};

// Velocity sweep, software-pipelined: the staged windows, the z-queue fronts and the
// own-point operands of plane k+1 are loaded while plane k is computed.
template <class T>
__device__ __forceinline__ void vel_interior_pipe_body(Grid g, Fields<T> f, StepConst<T> c, int kchunk, int bx_, int by_, int bz_) {
    __shared__ T s_xx[TY][36];
    __shared__ T s_xy[TY + 3][36];
    __shared__ T s_yy[TY + 3][TX];
    __shared__ T s_xz[TY][36];
    __shared__ T s_yz[TY + 3][TX];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = g.nabc + 1 + bx_ * TX, j0 = g.nabc + 1 + by_ * TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool act = (i <= g.nxt - g.nabc) && (j <= g.nyt - 2);
    const int kb = g.kin_lo() + bz_ * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const int ic = min(i, g.nxt), jc = min(j, g.nyt);
    const long long sz = g.plane;
    const long long pc = g.at(ic, jc, kb);
    const T* __restrict__ zz = f.zz; const T* __restrict__ xz = f.xz; const T* __restrict__ yz = f.yz;
    Prefetch<T, TY, 36> pxx; Prefetch<T, TY + 3, 36> pxy; Prefetch<T, TY + 3, TX> pyy;
    Prefetch<T, TY, 36> pxz; Prefetch<T, TY + 3, TX> pyz;
    pxx.load(f.xx, g, i0, j0, 2, 0, kb, tid);
    pxy.load(f.xy, g, i0, j0, 1, 2, kb, tid);
    pyy.load(f.yy, g, i0, j0, 0, 1, kb, tid);
    pxz.load(f.xz, g, i0, j0, 1, 0, kb, tid);
    pyz.load(f.yz, g, i0, j0, 0, 2, kb, tid);
    T zq0, zq1 = zz[pc - sz], zq2 = zz[pc], zq3 = zz[pc + sz], nz = zz[pc + 2 * sz];
    T xq0, xq1 = xz[pc - 2 * sz], xq2 = xz[pc - sz], xq3 = xz[pc], nx = xz[pc + sz];
    T yq0, yq1 = yz[pc - 2 * sz], yq2 = yz[pc - sz], yq3 = yz[pc], ny = yz[pc + sz];
    T pd = f.d[pc], pu = f.u[pc], pv = f.v[pc], pw = f.w[pc];
    const T c1 = c.c1, c2 = c.c2, dth = c.dth;
    for (int k = kb; k <= ke; ++k) {
        const long long pk = pc + (long long)(k - kb) * sz;
        __syncthreads();
        pxx.store(&s_xx[0][0], tid); pxy.store(&s_xy[0][0], tid); pyy.store(&s_yy[0][0], tid);
        pxz.store(&s_xz[0][0], tid); pyz.store(&s_yz[0][0], tid);
        zq0 = zq1; zq1 = zq2; zq2 = zq3; zq3 = nz;
        xq0 = xq1; xq1 = xq2; xq2 = xq3; xq3 = nx;
        yq0 = yq1; yq1 = yq2; yq2 = yq3; yq3 = ny;
        const T cd = pd, cu = pu, cv = pv, cw = pw;
        if (k < ke) {
            pxx.load(f.xx, g, i0, j0, 2, 0, k + 1, tid);
            pxy.load(f.xy, g, i0, j0, 1, 2, k + 1, tid);
            pyy.load(f.yy, g, i0, j0, 0, 1, k + 1, tid);
            pxz.load(f.xz, g, i0, j0, 1, 0, k + 1, tid);
            pyz.load(f.yz, g, i0, j0, 0, 2, k + 1, tid);
            nz = zz[pk + 3 * sz]; nx = xz[pk + 2 * sz]; ny = yz[pk + 2 * sz];
            pd = f.d[pk + sz]; pu = f.u[pk + sz]; pv = f.v[pk + sz]; pw = f.w[pk + sz];
        }
        __syncthreads();
        if (!act) continue;
        const T r = dth / cd;
        f.u[pk] = cu + r * (c1 * (s_xx[ty][tx + 2] - s_xx[ty][tx + 1]) + c2 * (s_xx[ty][tx + 3] - s_xx[ty][tx]) +
                            c1 * (s_xy[ty + 2][tx + 1] - s_xy[ty + 1][tx + 1]) + c2 * (s_xy[ty + 3][tx + 1] - s_xy[ty][tx + 1]) +
                            c1 * (xq2 - xq1) + c2 * (xq3 - xq0));
        f.v[pk] = cv + r * (c1 * (s_xy[ty + 2][tx + 2] - s_xy[ty + 2][tx + 1]) + c2 * (s_xy[ty + 2][tx + 3] - s_xy[ty + 2][tx]) +
                            c1 * (s_yy[ty + 2][tx] - s_yy[ty + 1][tx]) + c2 * (s_yy[ty + 3][tx] - s_yy[ty][tx]) +
                            c1 * (yq2 - yq1) + c2 * (yq3 - yq0));
        f.w[pk] = cw + r * (c1 * (s_xz[ty][tx + 2] - s_xz[ty][tx + 1]) + c2 * (s_xz[ty][tx + 3] - s_xz[ty][tx]) +
                            c1 * (s_yz[ty + 2][tx] - s_yz[ty + 1][tx]) + c2 * (s_yz[ty + 3][tx] - s_yz[ty][tx]) +
                            c1 * (zq2 - zq1) + c2 * (zq3 - zq0));
    }
}

// Stress sweep, software-pipelined like k_vel_interior_pipe.
template <class T>
__device__ __forceinline__ void str_interior_pipe_body(Grid g, Fields<T> f, StepConst<T> c, int kchunk, int bx_, int by_, int bz_) {
    __shared__ T s_u[TY + 4][36];
    __shared__ T s_v[TY + 4][36];
    __shared__ T s_w[TY + 4][36];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = g.nabc + 1 + bx_ * TX, j0 = g.nabc + 1 + by_ * TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool act = (i <= g.nxt - g.nabc) && (j <= g.nyt - 2);
    const int kb = g.kin_lo() + bz_ * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const int ic = min(i, g.nxt - 1), jc = min(j, g.nyt - 1);  // keeps the (i+1,j+1) taps in range
    const long long sy = g.px, sz = g.plane;
    const long long pc = g.at(ic, jc, kb);
    const T* __restrict__ u = f.u; const T* __restrict__ v = f.v; const T* __restrict__ w = f.w;
    const T* __restrict__ mu = f.mu;
    Prefetch<T, TY + 4, 36> pu_, pv_, pw_;
    pu_.load(u, g, i0, j0, 2, 2, kb, tid);
    pv_.load(v, g, i0, j0, 2, 2, kb, tid);
    pw_.load(w, g, i0, j0, 2, 2, kb, tid);
    T uq0, uq1 = u[pc - sz], uq2 = u[pc], uq3 = u[pc + sz], nu = u[pc + 2 * sz];
    T vq0, vq1 = v[pc - sz], vq2 = v[pc], vq3 = v[pc + sz], nv = v[pc + 2 * sz];
    T wq0, wq1 = w[pc - 2 * sz], wq2 = w[pc - sz], wq3 = w[pc], nw = w[pc + sz];
    T mq0, mq1 = mu[pc], nm = mu[pc + sz];
    T pl = f.lam[pc], pmy = mu[pc + sy], pmd = mu[pc + 1 + sy + sz];
    T pxx = f.xx[pc], pyy = f.yy[pc], pzz = f.zz[pc], pxy = f.xy[pc], pxz = f.xz[pc], pyz = f.yz[pc];
    const T c1 = c.c1, c2 = c.c2, dth = c.dth;
    const int X = tx + 2, Y = ty + 2;
    for (int k = kb; k <= ke; ++k) {
        const long long pk = pc + (long long)(k - kb) * sz;
        __syncthreads();
        pu_.store(&s_u[0][0], tid); pv_.store(&s_v[0][0], tid); pw_.store(&s_w[0][0], tid);
        uq0 = uq1; uq1 = uq2; uq2 = uq3; uq3 = nu;
        vq0 = vq1; vq1 = vq2; vq2 = vq3; vq3 = nv;
        wq0 = wq1; wq1 = wq2; wq2 = wq3; wq3 = nw;
        mq0 = mq1; mq1 = nm;
        const T cl = pl, cmy = pmy, cmd = pmd;
        const T cxx = pxx, cyy = pyy, czz = pzz, cxy = pxy, cxz = pxz, cyz = pyz;
        if (k < ke) {
            pu_.load(u, g, i0, j0, 2, 2, k + 1, tid);
            pv_.load(v, g, i0, j0, 2, 2, k + 1, tid);
            pw_.load(w, g, i0, j0, 2, 2, k + 1, tid);
            const long long pn = pk + sz;
            nu = u[pn + 2 * sz]; nv = v[pn + 2 * sz]; nw = w[pn + sz]; nm = mu[pn + sz];
            pl = f.lam[pn]; pmy = mu[pn + sy]; pmd = mu[pn + 1 + sy + sz];
            pxx = f.xx[pn]; pyy = f.yy[pn]; pzz = f.zz[pn]; pxy = f.xy[pn]; pxz = f.xz[pn]; pyz = f.yz[pn];
        }
        __syncthreads();
        if (!act) continue;
        const T xl = cl, xm = mq0;
        const T a = xl + (T)2 * xm, b = xl;
        const T dxu1 = c1 * (s_u[Y][X + 1] - s_u[Y][X]), dxu2 = c2 * (s_u[Y][X + 2] - s_u[Y][X - 1]);
        const T dyv1 = c1 * (s_v[Y][X] - s_v[Y - 1][X]), dyv2 = c2 * (s_v[Y + 1][X] - s_v[Y - 2][X]);
        const T dzw1 = c1 * (wq2 - wq1), dzw2 = c2 * (wq3 - wq0);
        f.xx[pk] = cxx + dth * a * (dxu1 + dxu2) + dth * b * (dyv1 + dyv2 + dzw1 + dzw2);
        f.yy[pk] = cyy + dth * a * (dyv1 + dyv2) + dth * b * (dxu1 + dxu2 + dzw1 + dzw2);
        f.zz[pk] = czz + dth * a * (dzw1 + dzw2) + dth * b * (dxu1 + dxu2 + dyv1 + dyv2);
        T xmu = (T)0.5 * (xm + cmy);
        f.xy[pk] = cxy + dth * xmu * (c1 * (s_u[Y + 1][X] - s_u[Y][X]) + c2 * (s_u[Y + 2][X] - s_u[Y - 1][X]) +
                                      c1 * (s_v[Y][X] - s_v[Y][X - 1]) + c2 * (s_v[Y][X + 1] - s_v[Y][X - 2]));
        xmu = (T)0.5 * (xm + mq1);
        f.xz[pk] = cxz + dth * xmu * (c1 * (uq2 - uq1) + c2 * (uq3 - uq0) +
                                      c1 * (s_w[Y][X] - s_w[Y][X - 1]) + c2 * (s_w[Y][X + 1] - s_w[Y][X - 2]));
        xmu = (T)0.5 * (xm + cmd);
        f.yz[pk] = cyz + dth * xmu * (c1 * (vq2 - vq1) + c2 * (vq3 - vq0) +
                                      c1 * (s_w[Y + 1][X] - s_w[Y][X]) + c2 * (s_w[Y + 2][X] - s_w[Y - 1][X]));
    }
}

// ---------------------------------------------------------------- launch wrappers
template <class T>
__global__ void __launch_bounds__(NT) k_vel_interior_pipe(Grid g, Fields<T> f, StepConst<T> c, int kchunk) {
    vel_interior_pipe_body<T>(g, f, c, kchunk, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class T>
__global__ void __launch_bounds__(NT) k_str_interior_pipe(Grid g, Fields<T> f, StepConst<T> c, int kchunk) {
    str_interior_pipe_body<T>(g, f, c, kchunk, blockIdx.x, blockIdx.y, blockIdx.z);
}


// Interior sweep variants (chosen per context; the default is the fastest measured on B200)
enum InteriorVariant { IV_POINT = 0, IV_TILED = 1, IV_PIPE = 2, IV_TMA = 3 };

struct InteriorCfg {
    // measured on B200 at 1020x410x512 (fraction of the measured HBM copy bandwidth):
    // TMA ring 97% (velocity) and 92% (stress); register-prefetch pipe 66%/67%;
    // per-point 61%/53%; tiled without prefetch 22%/26%.  With the layered medium
    // (no media windows) 32 planes per CTA beat 16 / 8 by 2-4%.
    int variant = IV_TMA;
    int kchunk = 32;      // z-planes per CTA of the velocity sweep
    int kchunk_str = 32;  // z-planes per CTA of the stress sweep
    int by = 8;          // CTA rows (IV_POINT: block = 32 x by)
    // a grid too small to give every SM two CTAs at kchunk planes each gets fewer planes
    // per CTA (halved down to 4); off when FD3D_KCHUNK sets the depth
    bool kchunk_auto = true;
    int nsm = 148;        // SMs of the context's device
};

inline int interior_nz(const Grid& g) { return std::max(0, g.kin_hi() - g.kin_lo() + 1); }  // planes updated

// planes per CTA of an interior sweep of columns x nzT planes
inline int interior_kchunk(const InteriorCfg& cfg, int k, long long columns, int nzT) {
    k = std::max(1, std::min(k, nzT));
    if (cfg.kchunk_auto)
        while (k > 4 && columns * ((nzT + k - 1) / k) < 2LL * cfg.nsm) k = (k + 1) / 2;
    return k;
}

template <class T>
void launch_vel_interior(const InteriorCfg& cfg, const Grid& g, const Fields<T>& f, const StepConst<T>& c,
                         cudaStream_t st) {
    const int nxT = g.nxt - 2 * g.nabc, nyI = g.nyt - 2 - g.nabc, nzT = interior_nz(g);
    if (nzT <= 0) return;  // a z-slab without interior planes
    const int kch = interior_kchunk(cfg, cfg.kchunk, (long long)((nxT + 31) / 32) * ((nyI + 7) / 8), nzT);
    if (cfg.variant == IV_POINT) {
        const int by = cfg.by;
        dim3 grid((nxT + 31) / 32, (nyI + by - 1) / by, (nzT + kch - 1) / kch);
        k_vel_interior<T><<<grid, dim3(32, by), 0, st>>>(g, f, c, kch);
        return;
    }
    dim3 grid((nxT + TX - 1) / TX, (nyI + TY - 1) / TY, (nzT + kch - 1) / kch);
    if (cfg.variant == IV_TILED) k_vel_interior_tiled<T><<<grid, dim3(TX, TY), 0, st>>>(g, f, c, kch);
    else k_vel_interior_pipe<T><<<grid, dim3(TX, TY), 0, st>>>(g, f, c, kch);
}

template <class T>
void launch_str_interior(const InteriorCfg& cfg, const Grid& g, const Fields<T>& f, const StepConst<T>& c,
                         cudaStream_t st) {
    const int nxT = g.nxt - 2 * g.nabc, nyI = g.nyt - 2 - g.nabc, nzT = interior_nz(g);
    if (nzT <= 0) return;  // a z-slab without interior planes
    const int kch = interior_kchunk(cfg, cfg.kchunk_str, (long long)((nxT + 31) / 32) * ((nyI + 7) / 8), nzT);
    if (cfg.variant == IV_POINT) {
        const int by = cfg.by;
        dim3 grid((nxT + 31) / 32, (nyI + by - 1) / by, (nzT + kch - 1) / kch);
        k_str_interior<T><<<grid, dim3(32, by), 0, st>>>(g, f, c, kch);
        return;
    }
    dim3 grid((nxT + TX - 1) / TX, (nyI + TY - 1) / TY, (nzT + kch - 1) / kch);
    if (cfg.variant == IV_TILED) k_str_interior_tiled<T><<<grid, dim3(TX, TY), 0, st>>>(g, f, c, kch);
    else k_str_interior_pipe<T><<<grid, dim3(TX, TY), 0, st>>>(g, f, c, kch);
}

}  // namespace fd3d

#include "fd3d_tma.cuh"
#include <cudaTypedefs.h>

namespace fd3d {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// 3-D tiled map over one padded field array (x = row element incl. offset, y = j-1, z = k-1)
template <class T>
bool encode_field_map(CUtensorMap* m, const T* base, const Grid& g, int box_x, int box_y) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    // the stored planes only (a z-slab holds kofs+1 .. kofs+nzl); z = k - 1 - kofs
    cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.nyt, (cuuint64_t)g.nzl};
    cuuint64_t strides[2] = {(cuuint64_t)g.px * sizeof(T), (cuuint64_t)g.plane * sizeof(T)};
    cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                     (void*)(base + g.plane * g.kofs), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <class T>
bool make_interior_maps(const Grid& g, const Fields<T>& f, VelMaps& V, StrMaps& S) {
    bool ok = true;
    ok &= encode_field_map<T>(&V.xx, f.xx, g, 40, 8);
    ok &= encode_field_map<T>(&V.xy, f.xy, g, 40, 11);
    ok &= encode_field_map<T>(&V.yy, f.yy, g, 32, 11);
    ok &= encode_field_map<T>(&V.xz, f.xz, g, 40, 8);
    ok &= encode_field_map<T>(&V.yz, f.yz, g, 32, 11);
    ok &= encode_field_map<T>(&V.d, f.d, g, 32, 8);
    ok &= encode_field_map<T>(&V.u, f.u, g, 32, 8);
    ok &= encode_field_map<T>(&V.v, f.v, g, 32, 8);
    ok &= encode_field_map<T>(&V.w, f.w, g, 32, 8);
    ok &= encode_field_map<T>(&S.u, f.u, g, 40, 12);
    ok &= encode_field_map<T>(&S.v, f.v, g, 40, 12);
    ok &= encode_field_map<T>(&S.w, f.w, g, 40, 12);
    ok &= encode_field_map<T>(&S.lam, f.lam, g, 32, 8);
    ok &= encode_field_map<T>(&S.mu, f.mu, g, 32, 9);
    ok &= encode_field_map<T>(&S.xx, f.xx, g, 32, 8);
    ok &= encode_field_map<T>(&S.yy, f.yy, g, 32, 8);
    ok &= encode_field_map<T>(&S.zz, f.zz, g, 32, 8);
    ok &= encode_field_map<T>(&S.xy, f.xy, g, 32, 8);
    ok &= encode_field_map<T>(&S.xz, f.xz, g, 32, 8);
    ok &= encode_field_map<T>(&S.yz, f.yz, g, 32, 8);
    return ok;
}

template <class T>
bool prepare_tma_kernels() {
    const int vs = TMA_NS * VelSlot::ELEMS * (int)sizeof(T) + TMA_SMEM_PAD, ss = str_ring_bytes<T, false>(),
              ssl = str_ring_bytes<T, true>();
    bool ok = cudaFuncSetAttribute(k_vel_interior_tma<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, vs) == cudaSuccess;
    ok &= cudaFuncSetAttribute(k_str_interior_tma<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss) == cudaSuccess;
    ok &= cudaFuncSetAttribute(k_vel_interior_tma<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, vs) == cudaSuccess;
    ok &= cudaFuncSetAttribute(k_str_interior_tma<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ssl) == cudaSuccess;
    if (!ok) cudaGetLastError();
    return ok;
}

template <class T>
void launch_vel_interior_tma(const VelMaps& M, const InteriorCfg& cfg, const Grid& g, const Fields<T>& f,
                             const StepConst<T>& c, int* status, cudaStream_t st) {
    const int nxT = g.nxt - 2 * g.nabc, nyI = g.nyt - 2 - g.nabc, nzT = interior_nz(g);
    if (nzT <= 0) return;  // a z-slab without interior planes
    const int kch = interior_kchunk(cfg, cfg.kchunk, (long long)((nxT + 31) / 32) * ((nyI + 7) / 8), nzT);
    dim3 grid((nxT + 31) / 32, (nyI + 7) / 8, (nzT + kch - 1) / kch);
    const size_t sm = TMA_NS * VelSlot::ELEMS * sizeof(T) + TMA_SMEM_PAD;
    if (f.lay) k_vel_interior_tma<T, true><<<grid, dim3(32, 8), sm, st>>>(M, g, f, c, kch, status);
    else k_vel_interior_tma<T, false><<<grid, dim3(32, 8), sm, st>>>(M, g, f, c, kch, status);
}

template <class T>
void launch_str_interior_tma(const StrMaps& M, const InteriorCfg& cfg, const Grid& g, const Fields<T>& f,
                             const StepConst<T>& c, int* status, cudaStream_t st) {
    const int nxT = g.nxt - 2 * g.nabc, nyI = g.nyt - 2 - g.nabc, nzT = interior_nz(g);
    if (nzT <= 0) return;  // a z-slab without interior planes
    const int kch = interior_kchunk(cfg, cfg.kchunk_str, (long long)((nxT + 31) / 32) * ((nyI + 7) / 8), nzT);
    dim3 grid((nxT + 31) / 32, (nyI + 7) / 8, (nzT + kch - 1) / kch);
    if (f.lay) k_str_interior_tma<T, true><<<grid, dim3(32, 8), str_ring_bytes<T, true>(), st>>>(M, g, f, c, kch, status);
    else k_str_interior_tma<T, false><<<grid, dim3(32, 8), str_ring_bytes<T, false>(), st>>>(M, g, f, c, kch, status);
}

}  // namespace fd3d
