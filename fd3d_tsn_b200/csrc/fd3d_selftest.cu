// fd3d_selftest.cu -- exhaustive device check of div_pre against the IEEE division.
//
// The PML updates divide by dh and by 1 + omega, divisors known before the launch;
// div_pre (fd3d_common.cuh) forms those quotients from a host-computed reciprocal.
// fd3d_check_division runs div_pre and __fdiv_rn on every one of the 2^32 float bit
// patterns for each divisor given and counts the dividends whose results differ in
// any bit (two NaNs count as equal).
#include <cuda_runtime.h>
#include <cstdint>
#include "../../include/fd3d_gpu.h"
#include "fd3d_common.cuh"

using namespace fd3d;

namespace {

__global__ void k_check_division(float b, float y, unsigned long long* bad, unsigned* first) {
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long local = 0;
    unsigned ex = 0;
    for (uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; n < (1ull << 32); n += nthreads) {
        const unsigned bits = (unsigned)n;
        const float x = __uint_as_float(bits);
        const float q = div_pre(x, b, y);
        const float r = __fdiv_rn(x, b);
        const bool same = (__float_as_uint(q) == __float_as_uint(r)) || (q != q && r != r);
        if (!same) {
            if (local == 0) ex = bits;
            ++local;
        }
    }
    if (local) {
        atomicAdd(bad, local);
        atomicCAS(first, 0xffffffffu, ex);
    }
}

}  // namespace

extern "C" int fd3d_check_division(const float* divisors, int n, unsigned long long* mismatches,
                                   unsigned* first_bad) {
    if (!divisors || n < 0 || !mismatches) return FD3D_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return FD3D_ERR_NODEV; }
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FD3D_ERR_CUDA;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return FD3D_ERR_CUDA;
    unsigned long long* dbad = nullptr;
    unsigned* dfirst = nullptr;
    if (cudaMalloc(&dbad, sizeof(unsigned long long)) != cudaSuccess) return FD3D_ERR_NOMEM;
    if (cudaMalloc(&dfirst, sizeof(unsigned)) != cudaSuccess) { cudaFree(dbad); return FD3D_ERR_NOMEM; }
    int rc = FD3D_OK;
    for (int i = 0; i < n && rc == FD3D_OK; ++i) {
        const float b = divisors[i];
        const float y = div_pre_recip(b);
        const unsigned none = 0xffffffffu;
        if (cudaMemset(dbad, 0, sizeof(unsigned long long)) != cudaSuccess ||
            cudaMemcpy(dfirst, &none, sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess) {
            rc = FD3D_ERR_CUDA;
            break;
        }
        k_check_division<<<nsm * 8, 256>>>(b, y, dbad, dfirst);
        unsigned long long hb = 0;
        unsigned hf = none;
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(&hb, dbad, sizeof(hb), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(&hf, dfirst, sizeof(hf), cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = FD3D_ERR_CUDA;
            break;
        }
        mismatches[i] = hb;
        if (first_bad) first_bad[i] = hf;
    }
    cudaFree(dbad);
    cudaFree(dfirst);
    return rc;
}
