// fd3d_tma.cuh -- interior sweeps fed by the Tensor Memory Accelerator (sm_100a).
//
// A CTA owns a 32 x 8 (x,y) column of the interior box and marches a chunk of z.  For
// every z-plane one elected thread issues one cp.async.bulk.tensor (3-D tile) per
// array window -- the x/y halo windows of the differentiated fields and the CTA's own
// tile of every read-modify-write operand -- into a 3-slot shared-memory ring whose
// completion is tracked by an mbarrier per slot (transaction bytes).  Planes k+1 and
// k+2 are in flight while plane k is computed, and the threads issue no address
// arithmetic for the staged data, which is what limited the register-prefetch kernels.
// The z-neighbours of the own column stay in register queues fed by plain loads one
// plane ahead.  Arithmetic and its order are those of uxx1/vyy1/wzz1 and dstres
// (src/fd3d_deriv.f90:50-193, 513-622), as in k_vel_interior / k_str_interior.
//
// All TMA loads read this GPU's own memory; no multicast is used.  Every mbarrier wait
// is bounded: on time-out the kernel records ST_TIMEOUT, waits (bounded) for its own
// copies still in flight and returns.
#pragma once
#include <cuda.h>
#include "fd3d_async.cuh"
#include "fd3d_common.cuh"

namespace fd3d {

struct VelMaps { CUtensorMap xx, xy, yy, xz, yz, d, u, v, w; };
struct StrMaps { CUtensorMap u, v, w, lam, mu, xx, yy, zz, xy, xz, yz; };

#ifndef FD3D_TMA_NS
#define FD3D_TMA_NS 3
#endif
constexpr int TMA_NS = FD3D_TMA_NS;  // ring slots: plane k computed, the next ones in flight
constexpr int TMA_SMEM_PAD = 128;  // alignment slack of the dynamic ring

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(dst), "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}
// Velocity slot layout (elements; every window starts on 128 bytes)
//   xx [8][40]  x i0-4..i0+35, y j0..j0+7
//   xy [11][40] x i0-4..,      y j0-2..j0+8
//   yy [11][32] x i0..i0+31,   y j0-1..j0+9
//   xz [8][40]  x i0-4..,      y j0..j0+7
//   yz [11][32] x i0..,        y j0-2..j0+8
//   d, u, v, w [8][32] own tile
struct VelSlot {
    static constexpr int XX = 0, XY = 320, YY = 768, XZ = 1120, YZ = 1440, D = 1792, U = 2048, V = 2304, W = 2560;
    static constexpr int ELEMS = 2816;                 // padded slot size
    static constexpr int LOADED = 320 + 440 + 352 + 320 + 352 + 4 * 256;  // elements the 9 tiles bring
};

template <class T, bool LAYERED>
__device__ __forceinline__ void vel_issue(const VelMaps& M, T* slot, uint32_t bar, int x0, int y0, int k) {
    mbar_expect_tx(bar, (VelSlot::LOADED - (LAYERED ? 256 : 0)) * sizeof(T));
    const int z = k - 1;  // k counts the stored planes (global plane - kofs)
    tma_load_3d(smem_addr(slot + VelSlot::XX), &M.xx, x0 - 4, y0, z, bar);
    tma_load_3d(smem_addr(slot + VelSlot::XY), &M.xy, x0 - 4, y0 - 2, z, bar);
    tma_load_3d(smem_addr(slot + VelSlot::YY), &M.yy, x0, y0 - 1, z, bar);
    tma_load_3d(smem_addr(slot + VelSlot::XZ), &M.xz, x0 - 4, y0, z, bar);
    tma_load_3d(smem_addr(slot + VelSlot::YZ), &M.yz, x0, y0 - 2, z, bar);
    if (!LAYERED) tma_load_3d(smem_addr(slot + VelSlot::D), &M.d, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + VelSlot::U), &M.u, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + VelSlot::V), &M.v, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + VelSlot::W), &M.w, x0, y0, z, bar);
}

// Ring bookkeeping across the tiles one CTA processes: the n-th plane a CTA ever puts
// through its ring uses slot n % TMA_NS and mbarrier phase (n / TMA_NS) & 1.  A tile
// consumes every plane it issued, so `pc` (planes issued so far) is all that carries over.
__device__ __forceinline__ int ring_slot(unsigned n) { return (int)(n % TMA_NS); }
__device__ __forceinline__ uint32_t ring_parity(unsigned n) { return (n / TMA_NS) & 1u; }

__device__ __forceinline__ void tma_ring_init(uint64_t* bars) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < TMA_NS; ++s) mbar_init(smem_addr(&bars[s]), 1);
        fence_mbar_init();
    }
    __syncthreads();
}

// wait (bounded) for every plane in [k0, ke] of the current tile that was issued, then return
__device__ __forceinline__ void tma_drain_pc(const uint64_t* bars, unsigned pc, int k0, int ke, int kb) {
    for (int k = k0; k <= ke && k < k0 + TMA_NS; ++k) {
        const unsigned n = pc + (unsigned)(k - kb);
        mbar_wait(smem_addr(&bars[ring_slot(n)]), ring_parity(n));
    }
}

// One 32 x 8 x kchunk tile of the velocity sweep through the ring.  Returns false if a
// wait timed out (ST_TIMEOUT is recorded; the caller stops).
template <class T, bool LAYERED = false>
__device__ __forceinline__ bool vel_interior_tma_body(const VelMaps& M, const Grid& g, const Fields<T>& f,
                                                      const StepConst<T>& c, int kchunk, int bx_, int by_, int bz_,
                                                      T* ring, uint64_t* bars, unsigned& pc, int* status) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = g.nabc + 1 + bx_ * 32, j0 = g.nabc + 1 + by_ * 8;
    const int i = i0 + tx, j = j0 + ty;
    const bool act = (i <= g.nxt - g.nabc) && (j <= g.nyt - 2);
    const int kb = g.kin_lo() + bz_ * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const int x0 = g.off + i0 - 1, y0 = j0 - 1;  // tensor coordinates of the tile origin
    const bool leader = (tx == 0 && ty == 0);
    const unsigned p0 = pc;
    if (leader)
        for (int k = kb; k <= min(ke, kb + TMA_NS - 1); ++k) {
            const unsigned n = p0 + (unsigned)(k - kb);
            vel_issue<T, LAYERED>(M, ring + (size_t)ring_slot(n) * VelSlot::ELEMS, smem_addr(&bars[ring_slot(n)]), x0, y0, k - g.kofs);
        }
    // z queues of the own column (plain loads, one plane ahead)
    const int ic = min(i, g.nxt), jc = min(j, g.nyt);
    const long long sz = g.plane;
    const long long pcol = g.at(ic, jc, kb);
    const T* __restrict__ zz = f.zz; const T* __restrict__ xz = f.xz; const T* __restrict__ yz = f.yz;
    T zq0, zq1 = zz[pcol - sz], zq2 = zz[pcol], zq3 = zz[pcol + sz], nz = zz[pcol + 2 * sz];
    T xq0, xq1 = xz[pcol - 2 * sz], xq2 = xz[pcol - sz], xq3 = xz[pcol], nx = xz[pcol + sz];
    T yq0, yq1 = yz[pcol - 2 * sz], yq2 = yz[pcol - sz], yq3 = yz[pcol], ny = yz[pcol + sz];
    const T c1 = c.c1, c2 = c.c2, dth = c.dth;
    for (int k = kb; k <= ke; ++k) {
        const int n = k - kb;
        const unsigned gn = p0 + (unsigned)n;
        const int s = ring_slot(gn);
        const long long pk = pcol + (long long)n * sz;
        zq0 = zq1; zq1 = zq2; zq2 = zq3; zq3 = nz;
        xq0 = xq1; xq1 = xq2; xq2 = xq3; xq3 = nx;
        yq0 = yq1; yq1 = yq2; yq2 = yq3; yq3 = ny;
        if (k < ke) { nz = zz[pk + 3 * sz]; nx = xz[pk + 2 * sz]; ny = yz[pk + 2 * sz]; }
        const T rk = LAYERED ? f.lay[3 * g.nzt + k - 1] : (T)0;  // dth / density of plane k (1-D medium)
        if (!mbar_wait(smem_addr(&bars[s]), ring_parity(gn))) {
            atomicOr(status, ST_TIMEOUT);
            tma_drain_pc(bars, p0, k, ke, kb);
            return false;
        }
        const T* sl = ring + (size_t)s * VelSlot::ELEMS;
        if (act) {
            const T* sxx = sl + VelSlot::XX + ty * 40 + tx;        // column tx+4 is i
            const T* sxy = sl + VelSlot::XY + (ty + 2) * 40 + tx;  // row ty+2 is j
            const T* syy = sl + VelSlot::YY + (ty + 1) * 32 + tx;  // row ty+1 is j
            const T* sxz = sl + VelSlot::XZ + ty * 40 + tx;
            const T* syz = sl + VelSlot::YZ + (ty + 2) * 32 + tx;
            const int o = ty * 32 + tx;
            const T r = LAYERED ? rk : dth / sl[VelSlot::D + o];
            f.u[pk] = sl[VelSlot::U + o] +
                      r * (c1 * (sxx[4] - sxx[3]) + c2 * (sxx[5] - sxx[2]) + c1 * (sxy[4] - sxy[-40 + 4]) +
                           c2 * (sxy[40 + 4] - sxy[-80 + 4]) + c1 * (xq2 - xq1) + c2 * (xq3 - xq0));
            f.v[pk] = sl[VelSlot::V + o] +
                      r * (c1 * (sxy[5] - sxy[4]) + c2 * (sxy[6] - sxy[3]) + c1 * (syy[32] - syy[0]) +
                           c2 * (syy[64] - syy[-32]) + c1 * (yq2 - yq1) + c2 * (yq3 - yq0));
            f.w[pk] = sl[VelSlot::W + o] +
                      r * (c1 * (sxz[5] - sxz[4]) + c2 * (sxz[6] - sxz[3]) + c1 * (syz[0] - syz[-32]) +
                           c2 * (syz[32] - syz[-64]) + c1 * (zq2 - zq1) + c2 * (zq3 - zq0));
        }
        __syncthreads();  // every thread is done with slot s
        if (leader && k + TMA_NS <= ke) {
            fence_proxy_async_smem();
            vel_issue<T, LAYERED>(M, ring + (size_t)s * VelSlot::ELEMS, smem_addr(&bars[s]), x0, y0, k + TMA_NS - g.kofs);
        }
    }
    pc = p0 + (unsigned)(ke - kb + 1);
    return true;
}

template <class T, bool LAYERED>
__global__ void __launch_bounds__(256) k_vel_interior_tma(const __grid_constant__ VelMaps M, Grid g, Fields<T> f,
                                                           StepConst<T> c, int kchunk, int* status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations must start on 128 bytes: round the dynamic base up (128 spare bytes)
    T* ring = reinterpret_cast<T*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    __shared__ __align__(8) uint64_t bars[TMA_NS];
    tma_ring_init(bars);
    unsigned pc = 0;
    vel_interior_tma_body<T, LAYERED>(M, g, f, c, kchunk, blockIdx.x, blockIdx.y, blockIdx.z, ring, bars, pc, status);
}

// Stress slot layout (elements)
//   u, v, w [12][40]  x i0-4..i0+35, y j0-2..j0+9
//   lam, xx, yy, zz, xy, xz, yz [8][32] own tile
//   mu [9][32]        x i0..,  y j0..j0+8
struct StrSlot {
    static constexpr int U = 0, V = 480, W = 960, LAM = 1440, XX = 1696, YY = 1952, ZZ = 2208, XY = 2464, XZ = 2720,
                         YZ = 2976, MU = 3232;
    static constexpr int ELEMS = 3520;
    static constexpr int LOADED = 3520;
};

// The 1-D-medium stress sweep loads no lam / mu windows: its slot packs the six stress
// tiles right after u, v, w (2976 elements), so the ring takes 36 KB instead of 42 KB in FP32.
struct StrSlotLayered {
    static constexpr int U = 0, V = 480, W = 960, XX = 1440, YY = 1696, ZZ = 1952, XY = 2208, XZ = 2464,
                         YZ = 2720;
    static constexpr int LAM = 0, MU = 0;  // not loaded (the medium comes from the per-plane profile)
    static constexpr int ELEMS = 2976;
    static constexpr int LOADED = 2976;
};
template <bool LAYERED> struct StrSlotOf { using type = StrSlot; };
template <> struct StrSlotOf<true> { using type = StrSlotLayered; };

// dynamic shared memory of the stress sweep's ring
template <class T, bool LAYERED>
constexpr int str_ring_bytes() { return TMA_NS * StrSlotOf<LAYERED>::type::ELEMS * (int)sizeof(T) + TMA_SMEM_PAD; }

template <class T, bool LAYERED>
__device__ __forceinline__ void str_issue(const StrMaps& M, T* slot, uint32_t bar, int x0, int y0, int k) {
    using StrSlot = typename StrSlotOf<LAYERED>::type;
    mbar_expect_tx(bar, StrSlot::LOADED * sizeof(T));
    const int z = k - 1;  // k counts the stored planes (global plane - kofs)
    tma_load_3d(smem_addr(slot + StrSlot::U), &M.u, x0 - 4, y0 - 2, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::V), &M.v, x0 - 4, y0 - 2, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::W), &M.w, x0 - 4, y0 - 2, z, bar);
    if (!LAYERED) tma_load_3d(smem_addr(slot + StrSlot::LAM), &M.lam, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::XX), &M.xx, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::YY), &M.yy, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::ZZ), &M.zz, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::XY), &M.xy, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::XZ), &M.xz, x0, y0, z, bar);
    tma_load_3d(smem_addr(slot + StrSlot::YZ), &M.yz, x0, y0, z, bar);
    if (!LAYERED) tma_load_3d(smem_addr(slot + StrSlot::MU), &M.mu, x0, y0, z, bar);
}

template <class T, bool LAYERED = false>
__device__ __forceinline__ bool str_interior_tma_body(const StrMaps& M, const Grid& g, const Fields<T>& f,
                                                      const StepConst<T>& c, int kchunk, int bx_, int by_, int bz_,
                                                      T* ring, uint64_t* bars, unsigned& pc, int* status) {
    using StrSlot = typename StrSlotOf<LAYERED>::type;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i0 = g.nabc + 1 + bx_ * 32, j0 = g.nabc + 1 + by_ * 8;
    const int i = i0 + tx, j = j0 + ty;
    const bool act = (i <= g.nxt - g.nabc) && (j <= g.nyt - 2);
    const int kb = g.kin_lo() + bz_ * kchunk;
    const int ke = min(kb + kchunk - 1, g.kin_hi());
    const int x0 = g.off + i0 - 1, y0 = j0 - 1;
    const bool leader = (tx == 0 && ty == 0);
    const unsigned p0 = pc;
    if (leader)
        for (int k = kb; k <= min(ke, kb + TMA_NS - 1); ++k) {
            const unsigned n = p0 + (unsigned)(k - kb);
            str_issue<T, LAYERED>(M, ring + (size_t)ring_slot(n) * StrSlot::ELEMS, smem_addr(&bars[ring_slot(n)]), x0, y0, k - g.kofs);
        }
    const int ic = min(i, g.nxt - 1), jc = min(j, g.nyt - 1);  // keeps the (i+1,j+1) tap in range
    const long long sy = g.px, sz = g.plane;
    const long long pcol = g.at(ic, jc, kb);
    const T* __restrict__ u = f.u; const T* __restrict__ v = f.v; const T* __restrict__ w = f.w;
    const T* __restrict__ mu = f.mu;
    T uq0, uq1 = u[pcol - sz], uq2 = u[pcol], uq3 = u[pcol + sz], nu = u[pcol + 2 * sz];
    T vq0, vq1 = v[pcol - sz], vq2 = v[pcol], vq3 = v[pcol + sz], nv = v[pcol + 2 * sz];
    T wq0, wq1 = w[pcol - 2 * sz], wq2 = w[pcol - sz], wq3 = w[pcol], nw = w[pcol + sz];
    T mq1 = LAYERED ? (T)0 : mu[pcol + sz], pmd = LAYERED ? (T)0 : mu[pcol + 1 + sy + sz];
    const T c1 = c.c1, c2 = c.c2, dth = c.dth;
    for (int k = kb; k <= ke; ++k) {
        const int n = k - kb;
        const unsigned gn = p0 + (unsigned)n;
        const int s = ring_slot(gn);
        const long long pk = pcol + (long long)n * sz;
        uq0 = uq1; uq1 = uq2; uq2 = uq3; uq3 = nu;
        vq0 = vq1; vq1 = vq2; vq2 = vq3; vq3 = nv;
        wq0 = wq1; wq1 = wq2; wq2 = wq3; wq3 = nw;
        const T cm1 = mq1, cmd = pmd;  // mu(i,j,k+1), mu(i+1,j+1,k+1)
        if (k < ke) {
            const long long pn = pk + sz;
            nu = u[pn + 2 * sz]; nv = v[pn + 2 * sz]; nw = w[pn + sz];
            if (!LAYERED) { mq1 = mu[pn + sz]; pmd = mu[pn + 1 + sy + sz]; }
        }
        // 1-D medium: lam, mu of plane k and mu of plane k+1 (every (i,j) of a plane is equal)
        const T lk = LAYERED ? f.lay[k - 1] : (T)0, mk = LAYERED ? f.lay[g.nzt + k - 1] : (T)0;
        const T mk1 = LAYERED ? f.lay[g.nzt + k] : (T)0;
        if (!mbar_wait(smem_addr(&bars[s]), ring_parity(gn))) {
            atomicOr(status, ST_TIMEOUT);
            tma_drain_pc(bars, p0, k, ke, kb);
            return false;
        }
        const T* sl = ring + (size_t)s * StrSlot::ELEMS;
        if (act) {
            const T* su = sl + StrSlot::U + (ty + 2) * 40 + tx + 4;  // u(i,j)
            const T* sv = sl + StrSlot::V + (ty + 2) * 40 + tx + 4;
            const T* sw = sl + StrSlot::W + (ty + 2) * 40 + tx + 4;
            const int o = ty * 32 + tx;
            const T xl = LAYERED ? lk : sl[StrSlot::LAM + o], xm = LAYERED ? mk : sl[StrSlot::MU + o];
            const T a = xl + (T)2 * xm, b = xl;
            const T dxu1 = c1 * (su[1] - su[0]), dxu2 = c2 * (su[2] - su[-1]);
            const T dyv1 = c1 * (sv[0] - sv[-40]), dyv2 = c2 * (sv[40] - sv[-80]);
            const T dzw1 = c1 * (wq2 - wq1), dzw2 = c2 * (wq3 - wq0);
            f.xx[pk] = sl[StrSlot::XX + o] + dth * a * (dxu1 + dxu2) + dth * b * (dyv1 + dyv2 + dzw1 + dzw2);
            f.yy[pk] = sl[StrSlot::YY + o] + dth * a * (dyv1 + dyv2) + dth * b * (dxu1 + dxu2 + dzw1 + dzw2);
            f.zz[pk] = sl[StrSlot::ZZ + o] + dth * a * (dzw1 + dzw2) + dth * b * (dxu1 + dxu2 + dyv1 + dyv2);
            T xmu = (T)0.5 * (xm + (LAYERED ? mk : sl[StrSlot::MU + o + 32]));
            f.xy[pk] = sl[StrSlot::XY + o] + dth * xmu * (c1 * (su[40] - su[0]) + c2 * (su[80] - su[-40]) +
                                                          c1 * (sv[0] - sv[-1]) + c2 * (sv[1] - sv[-2]));
            xmu = (T)0.5 * (xm + (LAYERED ? mk1 : cm1));
            f.xz[pk] = sl[StrSlot::XZ + o] + dth * xmu * (c1 * (uq2 - uq1) + c2 * (uq3 - uq0) +
                                                          c1 * (sw[0] - sw[-1]) + c2 * (sw[1] - sw[-2]));
            xmu = (T)0.5 * (xm + (LAYERED ? mk1 : cmd));
            f.yz[pk] = sl[StrSlot::YZ + o] + dth * xmu * (c1 * (vq2 - vq1) + c2 * (vq3 - vq0) +
                                                          c1 * (sw[40] - sw[0]) + c2 * (sw[80] - sw[-40]));
        }
        __syncthreads();
        if (leader && k + TMA_NS <= ke) {
            fence_proxy_async_smem();
            str_issue<T, LAYERED>(M, ring + (size_t)s * StrSlot::ELEMS, smem_addr(&bars[s]), x0, y0, k + TMA_NS - g.kofs);
        }
    }
    pc = p0 + (unsigned)(ke - kb + 1);
    return true;
}

template <class T, bool LAYERED>
__global__ void __launch_bounds__(256) k_str_interior_tma(const __grid_constant__ StrMaps M, Grid g, Fields<T> f,
                                                           StepConst<T> c, int kchunk, int* status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations must start on 128 bytes: round the dynamic base up (128 spare bytes)
    T* ring = reinterpret_cast<T*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    __shared__ __align__(8) uint64_t bars[TMA_NS];
    tma_ring_init(bars);
    unsigned pc = 0;
    str_interior_tma_body<T, LAYERED>(M, g, f, c, kchunk, blockIdx.x, blockIdx.y, blockIdx.z, ring, bars, pc, status);
}

// dynamic shared memory of a CTA that runs both sweeps through one ring
template <class T>
constexpr int tma_ring_bytes() {
    return TMA_NS * (VelSlot::ELEMS > StrSlot::ELEMS ? VelSlot::ELEMS : StrSlot::ELEMS) * (int)sizeof(T) + TMA_SMEM_PAD;
}

}  // namespace fd3d
