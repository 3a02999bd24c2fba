// fd3d_post.cuh -- fault-plane observables reduced on the device.
//
//   k_moment_rate   moment rate of history records: sum over the interior fault plane
//                   of |slip rate| * mu(i,nyt,k) * dh^2 (fd3d_theo.f90:574-578 with the
//                   seismogram step equal to the time step), one record per CTA
//   k_post          after the loop (fd3d_theo.f90:604-605, 660-686, 710-749): rupture
//                   velocity and cohesive-zone planes, and per-CTA partial sums of the
//                   seismic moment, the stress-drop numerator / denominator and the
//                   slip-weighted rupture speed
//   k_post_sum      the partial sums added in a fixed order
//
// Every sum is FP64 and reduced in a fixed tree order, so the results do not depend on
// scheduling; against the reference's sequential loops they differ only by the
// summation order (relative ~1e-14).
#pragma once
#include "fd3d_common.cuh"

namespace fd3d {

constexpr int POST_THREADS = 256;
constexpr int POST_NSUM = 5;  // m0, numer, denom, tint, tint2

// fixed-order tree sum of one double per thread of a POST_THREADS block
__device__ __forceinline__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = POST_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// mu at the fault plane (i, nyt, k): the 1-D profile when the medium is layered
template <class T>
__device__ __forceinline__ double fault_mu(const Grid& g, const Fields<T>& f, int i, int k) {
    return f.lay ? (double)f.lay[g.nzt + k - 1] : (double)f.mu[g.at(i, g.nyt, k)];
}

template <class T>
__global__ void __launch_bounds__(POST_THREADS) k_moment_rate(Grid g, Fields<T> f, const T* ring, int cap, int nf,
                                                              int rec0, double dh, double* out) {
    __shared__ double sh[POST_THREADS];
    const int nxT = g.nxt - 2 * g.nabc, nzT = g.ks() - g.nabc;
    const long long plane = (long long)nxT * nzT;
    const long long slot = (long long)((rec0 + (int)blockIdx.x) % cap);
    const T* sx = ring + (slot * nf + 0) * plane;  // sliprateX, then sliprateZ
    const T* sz = sx + plane;
    double acc = 0.0;
    for (long long q = threadIdx.x; q < plane; q += POST_THREADS) {
        const int i = g.nabc + 1 + (int)(q % nxT), k = g.nabc + 1 + (int)(q / nxT);
        const double a = (double)sx[q], b = (double)sz[q];
        acc += sqrt(a * a + b * b) * fault_mu(g, f, i, k) * dh * dh;
    }
    const double r = block_sum(acc, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = r;
}

template <class T>
__global__ void __launch_bounds__(POST_THREADS) k_post(Grid g, Fields<T> f, Fault<T> q, double dh, double dh2,
                                                       double* rvel, double* czone, double* part) {
    __shared__ double sh[POST_THREADS];
    const int nxT = g.nxt - 2 * g.nabc, nzT = g.ks() - g.nabc;
    const long long n = (long long)nxT * nzT;
    const double none = 1.e4;  // ruptime / sliptime of a node that never ruptured
    double s[POST_NSUM] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long t = (long long)blockIdx.x * POST_THREADS + threadIdx.x; t < n;
         t += (long long)gridDim.x * POST_THREADS) {
        const int i = g.nabc + 1 + (int)(t % nxT), k = g.nabc + 1 + (int)(t / nxT);
        const int p = g.at2(i, k);
        const double sx = q.slipX[p], sz = q.slipZ[p];
        const double slip = sqrt(sx * sx + sz * sz);
        s[0] += slip * fault_mu(g, f, i, k) * dh2;  // seismic moment (dh2 = dh*dh in the field type)
        const double dzs = (double)(T)(q.schangeZ[p] - q.T0Z[p]);       // stress drop in `real`
        const double dxs = (double)(T)(q.schangeX[p] - q.T0X[p]);
        s[1] += dzs * sz + dxs * sx;
        s[2] += slip;
        double rv = 0.0, cz = 0.0;
        const double r0 = q.ruptime[p], rxp = q.ruptime[g.at2(i + 1, k)], rzp = q.ruptime[g.at2(i, k + 1)];
        const double rxm = q.ruptime[g.at2(i - 1, k)], rzm = q.ruptime[g.at2(i, k - 1)];
        if (r0 != none && rxp != none && rzp != none && rxm != none && rzm != none && q.sliptime[p] != none) {
            const double den = sqrt((rxp - r0) * (rxp - r0) + (rzp - r0) * (rzp - r0)) +
                               sqrt((r0 - rxm) * (r0 - rxm) + (r0 - rzm) * (r0 - rzm));
            if (den != 0.0) {
                rv = 2.0 * dh / den;
                s[3] += rv * slip;
                s[4] += slip;
            }
            cz = rv * (q.sliptime[p] - r0);
        }
        rvel[p] = rv;
        czone[p] = cz;
    }
    for (int c = 0; c < POST_NSUM; ++c) {
        const double r = block_sum(s[c], sh);
        if (threadIdx.x == 0) part[(long long)blockIdx.x * POST_NSUM + c] = r;
    }
}

__global__ void __launch_bounds__(POST_THREADS) k_post_sum(const double* part, int nblk, double* out) {
    __shared__ double sh[POST_THREADS];
    for (int c = 0; c < POST_NSUM; ++c) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblk; b += POST_THREADS) v += part[(long long)b * POST_NSUM + c];
        const double r = block_sum(v, sh);
        if (threadIdx.x == 0) out[c] = r;
    }
}

}  // namespace fd3d
