// fd3d_ctx.cu -- C ABI of the single-model B200 path (include/fd3d_gpu.h).
//
// Owns the device state of one forward model, enqueues the eight launches of a
// time step on the context's stream, captures chunks of steps in a CUDA graph,
// and drains the device history ring into the reference's result files.  A context
// can also own a z-slab of a model (a range of planes) that steps with the model's other
// slabs, in one process or over NCCL, exchanging halos between the phases of a step.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "fd3d_nccl.h"
#include "../../include/fd3d_gpu.h"
#include "fd3d_common.cuh"
#include "fd3d_kernels.cuh"
#include "fd3d_opt.cuh"
#include "fd3d_post.cuh"
#include "fd3d_setup.h"
#include "fd3d_host.h"
#include "fd3d_trace.h"

using namespace fd3d;

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            std::fprintf(stderr, "fd3d: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_),  \
                         __FILE__, __LINE__);                                                  \
            return FD3D_ERR_CUDA;                                                              \
        }                                                                                      \
    } while (0)

namespace fd3d {

// Whether the uploaded medium varies with k only: every (i,j) of a plane k equals
// (1,1,k) in all three arrays (sets *nonuniform otherwise); the profile of column (1,1)
// goes to tab (lam, mu, d and dth/d, nzt values each).
template <class T>
__global__ void k_layer_check(Grid g, const T* lam, const T* mu, const T* d, T dth, T dt, T* tab, int* nonuniform) {
    const int nrows = g.nyt * g.nzl;  // rows (j,k) of the stored planes, from kofs+1; a CTA per row
    int bad = 0;
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int j = 1 + r % g.nyt, k = g.kofs + 1 + r / g.nyt;
        const long long p0 = g.at(1, 1, k), row = g.at(1, j, k);
        const T l0 = lam[p0], m0 = mu[p0], d0 = d[p0];
        for (int i = threadIdx.x; i < g.nxt; i += blockDim.x)
            bad |= (lam[row + i] != l0) | (mu[row + i] != m0) | (d[row + i] != d0);
        if (j == 1 && threadIdx.x == 0) {
            tab[k - 1] = l0;
            tab[g.nzt + k - 1] = m0;
            tab[2 * g.nzt + k - 1] = d0;
            tab[3 * g.nzt + k - 1] = dth / d0;
            tab[4 * g.nzt + k - 1] = dt / d0;
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(nonuniform, 1);
}

// inversion_modeltofd3d (fd3d_init.f90:806-835) on the device: control points (nli x
// nwi, Fortran order) bilinearly interpolated onto the interior fault plane in the
// field type, in the reference's operation order; striniX goes to T0Xb for the next pass
template <class T>
__global__ void k_model_to_fd3d(Grid g, int nli, const T* T0I, const T* TsI, const T* DcI, const T* ns, T DL, T DW,
                                T dh, int dipslip, Fault<T> q) {
    const int i = g.nabc + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = g.nabc + 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nxt - g.nabc || k > g.ks()) return;
    const T ZS = dh * (T)(k - 1 - g.nabc);
    const int kk = (int)(ZS / DW) + 1;
    const T u = (ZS - DW * (T)(kk - 1)) / DW;
    const T XS = dh * (T)(i - 1 - g.nabc);
    const int ii = (int)(XS / DL) + 1;
    const T t = (XS - DL * (T)(ii - 1)) / DL;
    auto C2 = [&](const T* a, int x, int z) { return a[(x - 1) + nli * (z - 1)]; };
    auto bil = [&](const T* a) {
        return ((T)1 - t) * ((T)1 - u) * C2(a, ii, kk) + t * ((T)1 - u) * C2(a, ii + 1, kk) +
               t * u * C2(a, ii + 1, kk + 1) + ((T)1 - t) * u * C2(a, ii, kk + 1);
    };
    const int p = g.at2(i, k);
    const T t0 = bil(T0I);
    if (dipslip) q.T0Z[p] = t0; else q.T0Xb[p] = t0;
    q.peakZ[p] = bil(TsI) * ns[k - 1];
    const T dc = bil(DcI);
    q.Dc[p] = dc;
    q.DcZ[p] = dc;
}

// A contiguous Fortran-order (nxt,nyt,nzt) array, staged on the device, into the padded
// layout (element type converted when the host's real kind differs from the field type)
template <class T, class S>
__global__ void k_repack(Grid g, const S* __restrict__ src, T* __restrict__ dst) {
    const int nrows = g.nyt * g.nzl;  // rows (j,k) of the stored planes, from kofs+1; a CTA per row
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int j = 1 + r % g.nyt, k = g.kofs + 1 + r / g.nyt;
        const S* s = src + (long long)r * g.nxt;
        T* o = dst + g.at(1, j, k);
        for (int i = threadIdx.x; i < g.nxt; i += blockDim.x) o[i] = (T)s[i];
    }
}

// n copies of v (the reset values of the fault planes)
template <class U>
__global__ void k_fill(U* a, size_t n, U v) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) a[q] = v;
}

// interp_fric (fd3d_deriv.f90:3174-3189): X-node values are 4-point averages
template <class T>
__global__ void k_interp_fric(Grid g, Fault<T> q) {
    const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 2 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.nxt - 1 || k > g.nzt - 1) return;
    const int a = g.at2(i, k), b = g.at2(i - 1, k), c = g.at2(i, k - 1), d = g.at2(i - 1, k - 1);
    q.peakX[a] = (q.peakZ[a] + q.peakZ[b] + q.peakZ[c] + q.peakZ[d]) / (T)4;
    q.dynX[a] = (q.dynZ[a] + q.dynZ[b] + q.dynZ[c] + q.dynZ[d]) / (T)4;
    q.DcX[a] = (q.DcZ[a] + q.DcZ[b] + q.DcZ[c] + q.DcZ[d]) / (T)4;
    q.T0X[a] = (q.T0Xb[a] + q.T0Xb[b] + q.T0Xb[c] + q.T0Xb[d]) / (T)4;
}

// Makes `dev` the calling thread's current device for the scope of a call and puts the
// previous one back on exit (a host thread may have another device current).
struct DeviceGuard {
    int prev = -1;
    bool changed = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev && cudaSetDevice(dev) == cudaSuccess) changed = true;
    }
    ~DeviceGuard() {
        if (changed) cudaSetDevice(prev);
    }
};

// A step in phases, and what a z-slab's neighbours need after each: the velocities
// after phase 0, the stresses after phase 1, the trial tractions and their damped parts
// after phase 2 (the friction law averages neighbouring nodes), the tractions after phase 3
// (the output averages them).
enum { STEP_PHASES = 5 };
enum HaloSet { HALO_NONE = -1, HALO_VEL = 0, HALO_STR = 1, HALO_TRIAL = 2, HALO_TRACTION = 3 };
inline int halo_after_phase(int ph) { return ph <= 3 ? ph : HALO_NONE; }
struct HaloArray {
    void* base;           // element of global plane / row 1 sits at base (index unit*(k-1))
    size_t elem, unit;    // bytes per element, elements per plane or row
};

struct CtxBase {
    fd3d_params p;
    Grid g;
    int device = 0;        // the device the context's memory and streams live on
    cudaStream_t st = nullptr;
    int law = 0;
    int nf = 4;            // history planes per record
    int steps_done = 0;    // host mirror of the device counter
    int rec_written = 0;   // history records already written to files
    bool medium_ok = false, fault_ok = false;
    int* it_dev = nullptr;
    int* status = nullptr;
    int hist_cap = 0;
    void* ring = nullptr;
    void* seis = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Side stream of the step: the fault-band and PML sweeps of each half-step run beside
    // the interior sweep (disjoint cells, both read only the other half-step's fields), so
    // the latency-bound PML tiles can take SM slots the interior sweep leaves free
    // (FD3D_OVERLAP=0 puts everything on one stream).
    cudaStream_t st2 = nullptr;
    cudaEvent_t evf[4] = {};
    // Completion marks of the last runs: a history or station read waits for the run that
    // made its records only, so the runs enqueued after it keep the GPU busy meanwhile.
    static constexpr int NMARK = 8;
    cudaEvent_t mark_ev[NMARK] = {};
    int mark_steps[NMARK] = {};
    int nmark = 0, next_mark = 0;
    void mark_run() {
        if (cudaEventRecord(mark_ev[next_mark], st) != cudaSuccess) { cudaGetLastError(); return; }
        mark_steps[next_mark] = steps_done;
        next_mark = (next_mark + 1) % NMARK;
        nmark = std::min(nmark + 1, NMARK);
    }
    // wait until the first `steps` steps have completed
    cudaError_t wait_steps(int steps) {
        int best = -1;
        for (int m = 0; m < nmark; ++m)
            if (mark_steps[m] >= steps && (best < 0 || mark_steps[m] < mark_steps[best])) best = m;
        return best < 0 ? cudaStreamSynchronize(st) : cudaEventSynchronize(mark_ev[best]);
    }
    int overlap = 1;
    // the fault boundary condition as separate launches (fres, traction, friction, output)
    // with the trial tractions in q.txt / q.tzt instead of the fused kernel
    bool split_bc = false;
    // z-slab of a model decomposed over several contexts (fd3d_ctx_create_slab): the
    // planes it updates; it steps only inside a slab group, which exchanges the halos
    bool slab = false;
    int slab_lo = 0, slab_hi = 0;
    // a slab in its own process (fd3d_slab_connect): the NCCL communicator of the model's
    // slabs, this slab's rank (from the bottom) and their number
    ncclComm_t comm = nullptr;
    int slab_rank = -1, slab_nranks = 0;
    float last_ms = 0.f;
    bool profiling = false;
    int pml_minb_vel = 1, pml_minb_str = 4;  // register caps of the PML sweeps (CTAs per SM; 1: none), measured fastest
    std::vector<cudaEvent_t> kev;   // 2 per kernel id
    float ktimes[FD3D_NKERNELS] = {0};
    int klaunch[FD3D_NKERNELS] = {0};
    static constexpr int NGRAPH = 6;          // graphs of 32, 16, 8, 4, 2 and 1 steps
    cudaGraphExec_t gexec[NGRAPH] = {};
    InteriorCfg icfg;       // interior sweep variant and CTA shape
    virtual ~CtxBase() {}
    virtual int alloc() = 0;
    virtual int upload_medium(const void*, const void*, const void*, int) = 0;
    virtual int upload_medium_layers(const double*, const double*, const double*) = 0;
    virtual int upload_fault(const fd3d_fault*) = 0;
    virtual int upload_fault_model(int, int, const double*, const double*, const double*, double, int) = 0;
    virtual int reset() = 0;
    virtual int enqueue_step() = 0;
    // one of the STEP_PHASES parts of a step (enqueue_step runs them in order)
    virtual int enqueue_phase(int ph) = 0;
    // the arrays of halo set `set` (HaloSet) with their element size and elements per
    // plane (3-D fields) or row (fault planes); base pointers take the global index
    virtual int halo_arrays(int set, std::vector<HaloArray>& out) = 0;
    virtual int fetch_field(int, void*, int) = 0;
    virtual int fetch_plane(int, double*) = 0;
    virtual int moment_rate(int rec0, int nrec, double* host) = 0;
    virtual int post(double* out4) = 0;
    virtual size_t elem() const = 0;
    virtual int save_state(std::FILE* fp) = 0;
    virtual int load_state(std::FILE* fp) = 0;
    virtual bool layered() const = 0;
};

template <class T>
struct Ctx : CtxBase {
    Fields<T> f{};
    Fault<T> q{};
    FvwScalars fs{};
    StepConst<T> c{};
    PmlDesc D{};
    PmlAux<T> X{};
    VelMaps vmaps{};        // TMA descriptors of the interior sweeps
    StrMaps smaps{};
    bool tma_ok = false;
    std::vector<void*> allocs;
    T* fieldpool = nullptr;
    std::vector<double> psiX0, psiZ0;  // initial FVW state, restored by reset
    size_t elem() const override { return sizeof(T); }
    bool layered() const override { return f.lay != nullptr; }

    // Device memory of the context: one allocation (zeroed once) carved into 256-byte
    // aligned arrays; a request beyond it gets its own allocation.
    char* block = nullptr;
    size_t block_bytes = 0, block_used = 0;
    T* dlay = nullptr;      // 1-D medium profile (Fields::lay) when the medium is layered
    int* lflag = nullptr;   // result word of the layered-medium check
    // fault-plane observables (fd3d_post.cuh): rupture velocity and cohesive-zone planes,
    // partial and final sums of the post-loop quantities, moment rate of ring records
    static constexpr int POST_BLOCKS = 148;
    double *rvel_d = nullptr, *czone_d = nullptr, *part_d = nullptr, *sums_d = nullptr, *mrate_d = nullptr;
    static size_t carve(size_t bytes) { return (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255; }
    template <class U> int dalloc(U** ptr, size_t n) {
        const size_t bytes = carve(n * sizeof(U));
        if (block && block_used + bytes <= block_bytes) {
            *ptr = (U*)(block + block_used);
            block_used += bytes;
            return 0;
        }
        void* v = nullptr;
        CK(cudaMalloc(&v, bytes));
        CK(cudaMemsetAsync(v, 0, bytes, st));
        allocs.push_back(v);
        *ptr = (U*)v;
        return 0;
    }

    ~Ctx() override {
        if (comm) nccl().CommDestroy(comm);
        for (cudaGraphExec_t& gx : gexec) if (gx) cudaGraphExecDestroy(gx);
        for (void* v : allocs) cudaFree(v);
        if (block) cudaFree(block);
        for (auto e : kev) cudaEventDestroy(e);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto e : evf) if (e) cudaEventDestroy(e);
        for (auto e : mark_ev) if (e) cudaEventDestroy(e);
        if (st2) cudaStreamDestroy(st2);
        if (st) cudaStreamDestroy(st);
    }

    int alloc() override {
        CK(cudaGetDevice(&device));
        CK(cudaDeviceGetAttribute(&icfg.nsm, cudaDevAttrMultiProcessorCount, device));
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        if (const char* e = std::getenv("FD3D_OVERLAP")) overlap = std::atoi(e);
        CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
        for (auto& e : evf) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto& e : mark_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        kev.resize(2 * FD3D_NKERNELS);
        for (auto& e : kev) CK(cudaEventCreate(&e));
        g = slab ? make_slab_grid(p, slab_lo, slab_hi) : make_grid(p);
        if (slab) { split_bc = true; overlap = 0; }
        c = make_const<T>(p);
        law = p.law;
        nf = (law == FD3D_LAW_FVW) ? 5 : 4;
        std::vector<Damp<T>> prof;
        make_pml<T>(p, D, prof);
        if (!pml_modes_hold(D, prof)) return FD3D_ERR_ARG;
        D.klo = g.klo;
        D.khi = g.khi;
        const int stride = std::max(1, p.history_stride);
        p.history_stride = stride;
        const long long plane = (long long)(p.nxt - 2 * p.nabc) * (p.nzt - p.nfs - p.nabc);
        int cap = p.history_capacity;
        if (cap <= 0) {
            // default: a ring of ~256 MB, at least 8 and at most 4096 records
            long long rec = plane * nf * (long long)sizeof(T);
            cap = (int)std::min<long long>(4096, std::max<long long>(8, (256ll << 20) / std::max<long long>(rec, 1)));
        }
        hist_cap = cap;
        {   // size of everything below, in the order it is carved
            const size_t n2 = (size_t)p.nxt * p.nzt;
            block_bytes = carve((size_t)g.n3 * 12 * sizeof(T)) + 37 * carve(n2 * sizeof(T)) +
                          10 * carve(n2 * sizeof(double)) + carve(pml_aux_elems(D) * sizeof(T)) +
                          carve(prof.size() * sizeof(Damp<T>)) + 2 * carve(sizeof(int)) +
                          carve((size_t)cap * nf * plane * sizeof(T)) +
                          carve((size_t)cap * std::max(1, p.nstations) * 3 * sizeof(T)) +
                          carve((size_t)LAY_N * p.nzt * sizeof(T)) + carve(sizeof(int)) + 2 * carve(n2 * sizeof(double)) +
                          carve((size_t)POST_BLOCKS * POST_NSUM * sizeof(double)) + carve(POST_NSUM * sizeof(double)) +
                          carve((size_t)cap * sizeof(double)) + (slab ? 2 * carve(n2 * sizeof(T)) : 0);
            void* v = nullptr;
            if (cudaMalloc(&v, block_bytes) != cudaSuccess) { cudaGetLastError(); return FD3D_ERR_NOMEM; }
            block = (char*)v;
            CK(cudaMemsetAsync(block, 0, block_bytes, st));
        }
        // 12 arrays of the 3-D grid in one pool
        if (dalloc(&fieldpool, (size_t)g.n3 * 12)) return FD3D_ERR_NOMEM;
        T* b = fieldpool - g.plane * g.kofs;  // a z-slab: global plane k at b + plane*(k-1)
        T** outs[9] = {&f.u, &f.v, &f.w, &f.xx, &f.yy, &f.zz, &f.xy, &f.yz, &f.xz};
        for (int a = 0; a < 9; ++a) *outs[a] = b + (size_t)a * g.n3;
        f.lam = b + 9 * (size_t)g.n3;
        f.mu = b + 10 * (size_t)g.n3;
        f.d = b + 11 * (size_t)g.n3;
        const size_t n2 = (size_t)p.nxt * p.nzt;
        T** tp[] = {&q.tx, &q.tz, &q.RFx, &q.RFz, &q.v1t, &q.au1, &q.av1, &q.aw1,
                    &q.uZ, &q.wX, &q.tabsX, &q.tabsZ, &q.T0X, &q.T0Z, &q.T0Xb, &q.Dc, &q.peakX, &q.dynX, &q.DcX, &q.peakZ,
                    &q.dynZ, &q.DcZ, &q.coh, &q.aX, &q.bX, &q.vwX, &q.fwX, &q.aZ, &q.bZ, &q.vwZ, &q.fwZ,
                    &q.schangeX, &q.schangeZ};
        for (T** a : tp) if (dalloc(a, n2)) return FD3D_ERR_NOMEM;
        // two-plane state (Fault): damping memory and X-node slip path
        if (dalloc(&q.avdx, 2 * n2) || dalloc(&q.avdz, 2 * n2)) return FD3D_ERR_NOMEM;
        double** dp[] = {&q.psiX, &q.psiZ, &q.distZ, &q.slipX, &q.slipZ, &q.ruptime, &q.rise, &q.sliptime};
        for (double** a : dp) if (dalloc(a, n2)) return FD3D_ERR_NOMEM;
        if (dalloc(&q.distX, 2 * n2)) return FD3D_ERR_NOMEM;
        q.n2 = (int)n2;
        q.txt = q.tzt = nullptr;  // trial tractions live in shared memory (fault_bc_body)
        if (slab && (dalloc(&q.txt, n2) || dalloc(&q.tzt, n2))) return FD3D_ERR_NOMEM;  // separate-launch fault BC
        T* pool = nullptr;
        if (dalloc(&pool, pml_aux_elems(D))) return FD3D_ERR_NOMEM;
        pml_aux_bind(X, pool, D);
        Damp<T>* dprof = nullptr;
        if (dalloc(&dprof, prof.size())) return FD3D_ERR_NOMEM;
        CK(cudaMemcpyAsync(dprof, prof.data(), prof.size() * sizeof(Damp<T>), cudaMemcpyHostToDevice, st));
        X.prof = dprof;
        tma_ok = make_interior_maps<T>(g, f, vmaps, smaps) && prepare_tma_kernels<T>();
        if (slab && !tma_ok) return FD3D_ERR_CUDA;
        if (!tma_ok && icfg.variant == IV_TMA) {
            std::fprintf(stderr, "fd3d: tensor maps of the interior sweeps could not be encoded for this grid; "
                                 "the interior sweeps fall back to plain loads (fd3d_ctx_info reports it)\n");
            icfg.variant = IV_PIPE;
        }
        if (dalloc(&it_dev, 1)) return FD3D_ERR_NOMEM;
        if (dalloc(&status, 1)) return FD3D_ERR_NOMEM;
        T* r = nullptr;
        if (dalloc(&r, (size_t)cap * nf * plane)) return FD3D_ERR_NOMEM;
        ring = r;
        T* sg = nullptr;
        if (dalloc(&sg, (size_t)cap * std::max(1, p.nstations) * 3)) return FD3D_ERR_NOMEM;
        seis = sg;
        if (dalloc(&dlay, (size_t)LAY_N * p.nzt)) return FD3D_ERR_NOMEM;
        if (dalloc(&lflag, 1)) return FD3D_ERR_NOMEM;
        if (dalloc(&rvel_d, n2) || dalloc(&czone_d, n2) || dalloc(&part_d, (size_t)POST_BLOCKS * POST_NSUM) ||
            dalloc(&sums_d, POST_NSUM) || dalloc(&mrate_d, (size_t)cap))
            return FD3D_ERR_NOMEM;
        CK(cudaStreamSynchronize(st));
        return FD3D_OK;
    }

    // After a medium upload: the kernels read the 1-D profile when the medium is layered
    // (checked on the device), and graphs captured with the old medium are dropped.
    int medium_uploaded() {
        int nonuni = 0;
        CK(cudaMemsetAsync(lflag, 0, sizeof(int), st));
        k_layer_check<T><<<1024, 256, 0, st>>>(g, f.lam, f.mu, f.d, c.dth, c.dt, dlay, lflag);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&nonuni, lflag, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        f.lay = nonuni ? nullptr : dlay;
        for (cudaGraphExec_t& gx : gexec)
            if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
        medium_ok = true;
        return FD3D_OK;
    }

    int upload_medium(const void* l, const void* m, const void* d, int rk) override {
        if (rk != 4 && rk != 8) return FD3D_ERR_ARG;
        // the planes this context stores: all of them, or a z-slab's own and halo planes
        const size_t nrow = (size_t)p.nxt * p.nyt;
        const size_t n = nrow * g.nzl, src0 = nrow * g.kofs;
        const void* src[3] = {l, m, d};
        T* dst[3] = {(T*)f.lam + g.plane * g.kofs, (T*)f.mu + g.plane * g.kofs, (T*)f.d + g.plane * g.kofs};
        for (int a = 0; a < 3; ++a)
            if (!src[a]) return FD3D_ERR_ARG;
        if (steps_done == 0 && n * (size_t)rk <= (size_t)g.n3 * 9 * sizeof(T)) {
            // The wave field is still zero: use it as the staging buffer of one contiguous
            // copy per array (the host array as it lies), repack on the device, zero it again.
            for (int a = 0; a < 3; ++a) {
                CK(cudaMemcpyAsync(fieldpool, (const char*)src[a] + src0 * rk, n * (size_t)rk, cudaMemcpyHostToDevice, st));
                T* at_k = dst[a] - g.plane * g.kofs;  // indexed by the global plane
                if (rk == 8) k_repack<T, double><<<1184, 256, 0, st>>>(g, (const double*)fieldpool, at_k);
                else k_repack<T, float><<<1184, 256, 0, st>>>(g, (const float*)fieldpool, at_k);
                CK(cudaGetLastError());
            }
            CK(cudaMemsetAsync(fieldpool, 0, n * (size_t)rk, st));
            CK(cudaStreamSynchronize(st));
            return medium_uploaded();
        }
        if ((size_t)rk == sizeof(T)) {
            // same element type: one pitched copy per array straight into the padded rows
            for (int a = 0; a < 3; ++a) {
                CK(cudaMemcpy2DAsync(dst[a] + g.off, (size_t)g.px * sizeof(T), (const char*)src[a] + src0 * rk,
                                     (size_t)p.nxt * sizeof(T), (size_t)p.nxt * sizeof(T), (size_t)p.nyt * g.nzl,
                                     cudaMemcpyHostToDevice, st));
            }
            CK(cudaStreamSynchronize(st));
            return medium_uploaded();
        }
        std::vector<T> row((size_t)g.px * p.nyt * 16);
        for (int a = 0; a < 3; ++a) {
            // pack k-slabs into the padded layout on the host, one copy per slab
            const int kb = 16;
            for (int k0 = 0; k0 < g.nzl; k0 += kb) {
                const int nk = std::min(kb, g.nzl - k0);
                std::fill(row.begin(), row.end(), (T)0);
                for (int kk = 0; kk < nk; ++kk)
                    for (int j = 0; j < p.nyt; ++j) {
                        const size_t so = src0 + (size_t)p.nxt * ((size_t)j + (size_t)p.nyt * (k0 + kk));
                        T* o = row.data() + (size_t)g.px * ((size_t)j + (size_t)p.nyt * kk) + g.off;
                        if (rk == 8) { const double* s = (const double*)src[a] + so; for (int i = 0; i < p.nxt; ++i) o[i] = (T)s[i]; }
                        else         { const float* s = (const float*)src[a] + so;  for (int i = 0; i < p.nxt; ++i) o[i] = (T)s[i]; }
                    }
                CK(cudaMemcpyAsync(dst[a] + (size_t)g.plane * k0, row.data(), (size_t)g.plane * nk * sizeof(T),
                                   cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
            }
        }
        return medium_uploaded();
    }

    int upload_medium_layers(const double* l, const double* m, const double* d) override {
        if (!l || !m || !d) return FD3D_ERR_ARG;
        std::vector<T> slab_((size_t)g.plane);
        T* dst[3] = {(T*)f.lam, (T*)f.mu, (T*)f.d};
        const double* src[3] = {l, m, d};
        for (int a = 0; a < 3; ++a)
            for (int k = g.kofs; k < g.kofs + g.nzl; ++k) {
                std::fill(slab_.begin(), slab_.end(), (T)0);
                const T v = (T)src[a][k];
                for (int j = 0; j < p.nyt; ++j)
                    for (int i = 0; i < p.nxt; ++i) slab_[(size_t)g.px * j + g.off + i] = v;
                CK(cudaMemcpyAsync(dst[a] + (size_t)g.plane * k, slab_.data(), (size_t)g.plane * sizeof(T),
                                   cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
            }
        return medium_uploaded();
    }

    int up2(T* dst, const std::vector<T>& v) {
        CK(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        return 0;
    }
    int up2d(double* dst, const std::vector<double>& v) {
        CK(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        return 0;
    }

    // friction arrays + interp_fric (fd3d_deriv.f90:3150-3190)
    int upload_fault(const fd3d_fault* fl) override {
        if (!fl) return FD3D_ERR_ARG;
        const int nxt = p.nxt, nzt = p.nzt;
        const size_t n2 = (size_t)nxt * nzt;
        auto cp = [&](const double* s, double dflt) {
            std::vector<T> v(n2);
            for (size_t k = 0; k < n2; ++k) v[k] = (T)(s ? s[k] : dflt);
            return v;
        };
        if (!fl->striniX || !fl->Dc) return FD3D_ERR_ARG;
        std::vector<T> sX = cp(fl->striniX, 0), sZ = cp(fl->striniZ, 0), Dc = cp(fl->Dc, 0);
        std::vector<T> zero(n2, (T)0);
        std::vector<T> pkZ = zero, dyZ = zero, DcZ = zero, T0Z = sZ, coh = zero;
        int rc = 0;
        if (law == FD3D_LAW_FVW) {
            if (!fl->a || !fl->b || !fl->psi || !fl->vw || !fl->aX || !fl->bX || !fl->psiX || !fl->vwX) return FD3D_ERR_ARG;
            rc |= up2(q.aZ, cp(fl->a, 0)); rc |= up2(q.bZ, cp(fl->b, 0)); rc |= up2(q.vwZ, cp(fl->vw, 0));
            rc |= up2(q.aX, cp(fl->aX, 0)); rc |= up2(q.bX, cp(fl->bX, 0)); rc |= up2(q.vwX, cp(fl->vwX, 0));
            rc |= up2(q.fwZ, cp(fl->fwZ, fl->fw)); rc |= up2(q.fwX, cp(fl->fwX, fl->fw));
            psiZ0.assign(fl->psi, fl->psi + n2);
            psiX0.assign(fl->psiX, fl->psiX + n2);
            fs.Sn = fl->Sn; fs.v0 = fl->v0; fs.f0 = fl->f0; fs.fw = fl->fw; fs.uini = fl->uini; fs.wini = fl->wini;
            fs.nucleation = fl->nucleation;
            fs.hx0 = fl->hx0; fs.hz0 = fl->hz0; fs.perturb = fl->perturb; fs.RR2 = fl->RR2; fs.TT2 = fl->TT2;
            fs.strinixI = fl->strinixI;
        } else {
            if (!fl->peak_xz || !fl->dyn_xz) return FD3D_ERR_ARG;
            pkZ = cp(fl->peak_xz, 0); dyZ = cp(fl->dyn_xz, 0); DcZ = Dc; coh = cp(fl->coh, 0);
            fs = FvwScalars{};
        }
        // Z-node planes up; X-node planes (4-point averages, zero on the border) by
        // k_interp_fric on the device, T0X from striniX staged in T0Xb
        rc |= up2(q.Dc, Dc); rc |= up2(q.T0Xb, sX); rc |= up2(q.T0Z, T0Z);
        rc |= up2(q.peakZ, pkZ); rc |= up2(q.dynZ, dyZ); rc |= up2(q.DcZ, DcZ); rc |= up2(q.coh, coh);
        if (rc) return FD3D_ERR_CUDA;
        T* xnodes[] = {q.peakX, q.dynX, q.DcX, q.T0X};
        for (T* a : xnodes) CK(cudaMemsetAsync(a, 0, n2 * sizeof(T), st));
        k_interp_fric<T><<<dim3((p.nxt + 31) / 32, (p.nzt + 7) / 8), dim3(32, 8), 0, st>>>(g, q);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(q.T0Xb, q.T0X, n2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
        CK(cudaStreamSynchronize(st));
        fault_ok = true;
        return reset_state(false);
    }

    int upload_fault_model(int nli, int nwi, const double* T0I, const double* TsI, const double* DcI, double dip,
                           int dipslip) override {
        if (law != FD3D_LAW_SW || nli < 2 || nwi < 2 || !T0I || !TsI || !DcI) return FD3D_ERR_ARG;
        const size_t nc = (size_t)nli * nwi, n2 = (size_t)p.nxt * p.nzt;
        // control points and the normal-stress profile (fd3d_init.f90:77-86) in the field type
        std::vector<T> ctl(3 * nc + (size_t)p.nzt);
        for (size_t q2 = 0; q2 < nc; ++q2) {
            ctl[q2] = (T)T0I[q2]; ctl[nc + q2] = (T)TsI[q2]; ctl[2 * nc + q2] = (T)DcI[q2];
        }
        const T pi = (T)3.1415926535, dh = c.dh;
        for (int k = 1; k <= p.nzt; ++k) {
            const T cns = dipslip ? (T)8520. : (T)16200.;
            ctl[3 * nc + k - 1] = std::max((T)1.e5, cns * dh * (T)(p.nzt - p.nfs - k) * (T)std::sin((T)dip / (T)180. * pi));
        }
        const T DL = dh * (T)(p.nxt - 2 * p.nabc) / (T)(nli - 1);
        const T DW = dh * (T)(p.nzt - p.nfs - p.nabc) / (T)(nwi - 1);
        T* dctl = nullptr;  // set-up scratch, released before returning
        CK(cudaMalloc(&dctl, ctl.size() * sizeof(T)));
        CK(cudaMemcpyAsync(dctl, ctl.data(), ctl.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        T* zero[] = {q.T0Xb, q.T0Z, q.peakZ, q.Dc, q.DcZ, q.dynZ, q.coh, q.peakX, q.dynX, q.DcX, q.T0X};
        for (T* a : zero) CK(cudaMemsetAsync(a, 0, n2 * sizeof(T), st));
        const dim3 b2(32, 8);
        const int nxT = p.nxt - 2 * p.nabc, nzT = g.ks() - p.nabc;
        k_model_to_fd3d<T><<<dim3((nxT + 31) / 32, (nzT + 7) / 8), b2, 0, st>>>(
            g, nli, dctl, dctl + nc, dctl + 2 * nc, dctl + 3 * nc, DL, DW, dh, dipslip, q);
        k_interp_fric<T><<<dim3((p.nxt + 31) / 32, (p.nzt + 7) / 8), b2, 0, st>>>(g, q);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(q.T0Xb, q.T0X, n2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
        CK(cudaStreamSynchronize(st));
        CK(cudaFree(dctl));
        fs = FvwScalars{};
        fault_ok = true;
        return reset_state(false);
    }

    // Checkpoint: the whole device state of the context is its one allocation (wave field,
    // medium, PML split components, fault planes, step counter, history and station rings),
    // written as it lies, after the host-side state a run depends on.
    struct SavedHost {
        unsigned long long block_bytes;
        int steps_done, rec_written, medium_ok, fault_ok, layered;
        FvwScalars fs;
        unsigned long long npsi;
    };
    static constexpr size_t CKPT_CHUNK = 64ull << 20;
    int save_state(std::FILE* fp) override {
        if (slab) return FD3D_ERR_STATE;  // the slab range is not part of the file
        if (!allocs.empty()) return FD3D_ERR_STATE;  // state outside the block: not restorable
        CK(cudaStreamSynchronize(st));
        SavedHost h{};
        h.block_bytes = block_bytes; h.steps_done = steps_done; h.rec_written = rec_written;
        h.medium_ok = medium_ok; h.fault_ok = fault_ok; h.layered = f.lay != nullptr; h.fs = fs;
        h.npsi = psiZ0.size();
        if (std::fwrite(&h, sizeof h, 1, fp) != 1) return FD3D_ERR_IO;
        if (h.npsi && (std::fwrite(psiZ0.data(), sizeof(double), h.npsi, fp) != h.npsi ||
                       std::fwrite(psiX0.data(), sizeof(double), h.npsi, fp) != h.npsi))
            return FD3D_ERR_IO;
        std::vector<char> buf(std::min(CKPT_CHUNK, block_bytes));
        for (size_t off = 0; off < block_bytes; off += buf.size()) {
            const size_t n = std::min(buf.size(), block_bytes - off);
            CK(cudaMemcpy(buf.data(), block + off, n, cudaMemcpyDeviceToHost));
            if (std::fwrite(buf.data(), 1, n, fp) != n) return FD3D_ERR_IO;
        }
        return FD3D_OK;
    }
    int load_state(std::FILE* fp) override {
        SavedHost h{};
        if (std::fread(&h, sizeof h, 1, fp) != 1) return FD3D_ERR_IO;
        if (h.block_bytes != block_bytes || !allocs.empty()) return FD3D_ERR_ARG;  // another layout
        std::vector<double> pz(h.npsi), px(h.npsi);
        if (h.npsi && (std::fread(pz.data(), sizeof(double), h.npsi, fp) != h.npsi ||
                       std::fread(px.data(), sizeof(double), h.npsi, fp) != h.npsi))
            return FD3D_ERR_IO;
        CK(cudaStreamSynchronize(st));
        std::vector<char> buf(std::min(CKPT_CHUNK, block_bytes));
        for (size_t off = 0; off < block_bytes; off += buf.size()) {
            const size_t n = std::min(buf.size(), block_bytes - off);
            if (std::fread(buf.data(), 1, n, fp) != n) return FD3D_ERR_IO;
            CK(cudaMemcpy(block + off, buf.data(), n, cudaMemcpyHostToDevice));
        }
        steps_done = h.steps_done; rec_written = h.rec_written;
        medium_ok = h.medium_ok != 0; fault_ok = h.fault_ok != 0;
        f.lay = h.layered ? dlay : nullptr;
        fs = h.fs;
        psiZ0 = std::move(pz); psiX0 = std::move(px);
        for (cudaGraphExec_t& gx : gexec)
            if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
        nmark = 0;
        return FD3D_OK;
    }

    // zeroing of fd3d_theo.f90:59-88 and of the PML aux (fd3d_deriv.f90:1342-1410)
    int reset_state(bool keep_psi) {
        (void)keep_psi;
        CK(cudaMemsetAsync(fieldpool, 0, (size_t)g.n3 * 9 * sizeof(T), st));
        const size_t n2 = (size_t)p.nxt * p.nzt;
        T* zt[] = {q.tx, q.tz, q.RFx, q.RFz, q.v1t, q.au1, q.av1, q.aw1, q.uZ, q.wX, q.schangeX, q.schangeZ};
        for (T* a : zt) CK(cudaMemsetAsync(a, 0, n2 * sizeof(T), st));
        CK(cudaMemsetAsync(q.avdx, 0, 2 * n2 * sizeof(T), st));
        CK(cudaMemsetAsync(q.avdz, 0, 2 * n2 * sizeof(T), st));
        double* zd[] = {q.distZ, q.slipX, q.slipZ, q.rise};
        for (double* a : zd) CK(cudaMemsetAsync(a, 0, n2 * sizeof(double), st));
        CK(cudaMemsetAsync(q.distX, 0, 2 * n2 * sizeof(double), st));
        const unsigned fb = (unsigned)std::min<size_t>(1184, (n2 + 255) / 256);
        k_fill<double><<<fb, 256, 0, st>>>(q.ruptime, n2, 1.e4);
        k_fill<double><<<fb, 256, 0, st>>>(q.sliptime, n2, 1.e4);
        const T t0 = law == FD3D_LAW_FVW ? (T)1 : (T)0;
        k_fill<T><<<fb, 256, 0, st>>>(q.tabsX, n2, t0);
        k_fill<T><<<fb, 256, 0, st>>>(q.tabsZ, n2, t0);
        CK(cudaGetLastError());
        // initial state variable and prestress (the nucleation ramp rewrites T0X)
        CK(cudaMemcpyAsync(q.T0X, q.T0Xb, n2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
        if (law == FD3D_LAW_FVW) {
            CK(cudaMemcpyAsync(q.psiZ, psiZ0.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(q.psiX, psiX0.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        CK(cudaMemsetAsync(X.vel, 0, pml_aux_elems(D) * sizeof(T), st));
        CK(cudaMemsetAsync(it_dev, 0, sizeof(int), st));
        CK(cudaMemsetAsync(status, 0, sizeof(int), st));
        CK(cudaStreamSynchronize(st));
        steps_done = 0;
        rec_written = 0;
        nmark = 0;
        return FD3D_OK;
    }

    int reset() override {
        if (!fault_ok) return FD3D_ERR_STATE;
        return reset_state(false);
    }

    void kbeg(int id) { if (profiling) cudaEventRecord(kev[2 * id], st); }
    void kend(int id) {
        if (!profiling) return;
        cudaEventRecord(kev[2 * id + 1], st);
        cudaEventSynchronize(kev[2 * id + 1]);
        float ms = 0;
        cudaEventElapsedTime(&ms, kev[2 * id], kev[2 * id + 1]);
        ktimes[id] += ms;
        klaunch[id] += 1;
    }

    int enqueue_step() override {
        for (int ph = 0; ph < STEP_PHASES; ++ph) {
            const int rc = enqueue_phase(ph);
            if (rc) return rc;
        }
        return FD3D_OK;
    }

    // Phase 0 the velocity half-step, 1 the stress sweeps, 2-4 the fault boundary
    // condition (fused into phase 2 for a whole model; fres + traction, friction, output
    // as separate launches for a z-slab or when split_bc is set) and the nucleation ramp.
    int enqueue_phase(int ph) override {
        const int nxT = p.nxt - 2 * p.nabc;
        const int nzT = std::max(1, g.kin_hi() - g.kin_lo() + 1);  // fault rows updated (a launch has one at least)
        const dim3 b2(32, 8);
        const bool ov = overlap > 0 && !profiling;
        const bool top = g.owns(g.ks());  // the free-surface rows are this context's
        cudaStream_t sp = ov ? st2 : st;  // fault band and PML
        auto fork = [&](int e) { cudaEventRecord(evf[e], st); cudaStreamWaitEvent(st2, evf[e], 0); };
        auto join = [&](int e) { cudaEventRecord(evf[e], st2); cudaStreamWaitEvent(st, evf[e], 0); };
        HistDesc h;
        if (ph >= 2) {
            h.ring = ring; h.cap = hist_cap; h.stride = p.history_stride; h.nf = nf; h.nst = p.nstations;
            for (int s = 0; s < p.nstations; ++s) { h.sta[3 * s] = p.staX[s]; h.sta[3 * s + 1] = p.staY[s]; h.sta[3 * s + 2] = p.staZ[s]; }
            h.seis = seis;
        }
        switch (ph) {
        case 0:  // velocity half-step
            if (ov) fork(0);
            kbeg(0);
            if (icfg.variant == IV_TMA) launch_vel_interior_tma<T>(vmaps, icfg, g, f, c, status, st);
            else launch_vel_interior<T>(icfg, g, f, c, st);
            kend(0);
            kbeg(1);
            k_vel_fault<T><<<dim3((std::max(nxT, p.nxt) + 31) / 32, (nzT + 7) / 8), b2, 0, sp>>>(g, f, q, c, law, fs, it_dev, status);
            kend(1);
            kbeg(2);
            launch_pml<T>(false, pml_minb_vel, sp, g, f, D, X, c, status);
            kend(2);
            if (ov) join(1);
            kbeg(3);
            if (!p.fspace && top) k_vel_fs<T><<<dim3((p.nxt + 31) / 32, (p.nyt + 7) / 8), b2, 0, st>>>(g, f);  // fuvw
            kend(3);
            break;
        case 1:  // stress sweeps
            if (ov) fork(2);
            kbeg(4);
            if (icfg.variant == IV_TMA) launch_str_interior_tma<T>(smaps, icfg, g, f, c, status, st);
            else launch_str_interior<T>(icfg, g, f, c, st);
            kend(4);
            kbeg(5);
            k_str_fault<T><<<dim3((nxT + 31) / 32, (nzT + 7) / 8), b2, 0, sp>>>(g, f, q, c);
            kend(5);
            kbeg(6);
            launch_pml<T>(true, pml_minb_str, sp, g, f, D, X, c, status);
            kend(6);
            if (ov) join(3);
            break;
        case 2:  // fault boundary condition
            kbeg(7);
            if (!split_bc) {   // fres and the fused trial traction, friction and output tiles in one launch
                int nfres, tiles_x, tiles;
                fault_bc_grid(g, nfres, tiles_x, tiles);
                k_fault_bc<T><<<nfres + tiles, b2, 0, st>>>(g, f, q, c, law, fs, it_dev, h, status, nfres, tiles_x);
            } else {           // the same as separate launches, trial tractions in q.txt / q.tzt
                if (!p.fspace && top) k_str_fs<T><<<dim3((p.nxt + 31) / 32, (p.nyt + 7) / 8), b2, 0, st>>>(g, f);  // fres
                k_traction<T><<<dim3((nxT + 31) / 32, (nzT + 7) / 8), b2, 0, st>>>(g, f, q, c, it_dev);
            }
            break;
        case 3:
            if (split_bc) k_friction<T><<<dim3((nxT + 31) / 32, (nzT + 7) / 8), b2, 0, st>>>(g, f, q, c, law, fs, it_dev);
            break;
        default:
            if (split_bc) k_output<T><<<dim3((nxT + 31) / 32, (nzT + 7) / 8), b2, 0, st>>>(g, f, q, law, it_dev, h, status);
            if (law == FD3D_LAW_FVW && fs.nucleation) {  // every node of the plane (a z-slab too: no halo needed)
                const int ni = (p.nxt - p.nabc) - (p.nabc - 1) + 1, nk = g.ks() - (p.nabc - 1) + 1;
                k_nucleation<T><<<dim3((ni + 31) / 32, (nk + 7) / 8), b2, 0, st>>>(g, q, c, fs, it_dev);
            }
            kend(7);
            break;
        }
        return FD3D_OK;
    }

    int halo_arrays(int set, std::vector<HaloArray>& out) override {
        out.clear();
        const size_t e = sizeof(T), pl = (size_t)g.plane, row = (size_t)p.nxt;
        T* vel[] = {f.u, f.v, f.w};
        T* str[] = {f.xx, f.yy, f.zz, f.xy, f.yz, f.xz};
        T* trial[] = {q.txt, q.tzt, q.RFx, q.RFz};
        T* trac[] = {q.tx, q.tz};
        T** a = nullptr;
        size_t na = 0, unit = pl;
        switch (set) {
            case HALO_VEL: a = vel; na = 3; break;
            case HALO_STR: a = str; na = 6; break;
            case HALO_TRIAL: a = trial; na = 4; unit = row; break;
            case HALO_TRACTION: a = trac; na = 2; unit = row; break;
            default: return FD3D_ERR_ARG;
        }
        for (size_t k = 0; k < na; ++k) out.push_back(HaloArray{a[k], e, unit});
        return FD3D_OK;
    }

    int fetch_field(int which, void* host, int rk) override {
        if (rk != 4 && rk != 8) return FD3D_ERR_ARG;
        const T* src;
        switch (which) {
            case FD3D_FIELD_U: src = f.u; break;   case FD3D_FIELD_V: src = f.v; break;
            case FD3D_FIELD_W: src = f.w; break;   case FD3D_FIELD_XX: src = f.xx; break;
            case FD3D_FIELD_YY: src = f.yy; break; case FD3D_FIELD_ZZ: src = f.zz; break;
            case FD3D_FIELD_XY: src = f.xy; break; case FD3D_FIELD_YZ: src = f.yz; break;
            case FD3D_FIELD_XZ: src = f.xz; break;
            default: return FD3D_ERR_ARG;
        }
        // the planes this context owns (all of them for a whole model); the host array
        // keeps its other planes, so the z-slabs of a model fill one array between them
        std::vector<T> slab((size_t)g.plane);
        for (int k = g.klo - 1; k < g.khi; ++k) {
            CK(cudaMemcpyAsync(slab.data(), src + (size_t)g.plane * k, (size_t)g.plane * sizeof(T), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int j = 0; j < p.nyt; ++j) {
                const size_t o = (size_t)p.nxt * ((size_t)j + (size_t)p.nyt * k);
                const T* s = slab.data() + (size_t)g.px * j + g.off;
                if (rk == 8) { double* d = (double*)host + o; for (int i = 0; i < p.nxt; ++i) d[i] = (double)s[i]; }
                else         { float* d = (float*)host + o;  for (int i = 0; i < p.nxt; ++i) d[i] = (float)s[i]; }
            }
        }
        return FD3D_OK;
    }

    int fetch_plane(int which, double* host) override {
        const size_t n2 = (size_t)p.nxt * p.nzt;
        const T* ts = nullptr;
        const double* ds = nullptr;
        switch (which) {
            case FD3D_PLANE_TX: ts = q.tx; break;            case FD3D_PLANE_TZ: ts = q.tz; break;
            case FD3D_PLANE_SLIPX: ds = q.slipX; break;      case FD3D_PLANE_SLIPZ: ds = q.slipZ; break;
            case FD3D_PLANE_RUPTIME: ds = q.ruptime; break;  case FD3D_PLANE_RISE: ds = q.rise; break;
            case FD3D_PLANE_SLIPTIME: ds = q.sliptime; break;
            case FD3D_PLANE_DISTX: ds = pp_wr(q.distX, steps_done, (int)n2); break;  // the last step's plane
            case FD3D_PLANE_DISTZ: ds = q.distZ; break;
            case FD3D_PLANE_PSIX: ds = q.psiX; break;        case FD3D_PLANE_PSIZ: ds = q.psiZ; break;
            case FD3D_PLANE_T0X: ts = q.T0X; break;          case FD3D_PLANE_T0Z: ts = q.T0Z; break;
            case FD3D_PLANE_SCHANGEX: ts = q.schangeX; break; case FD3D_PLANE_SCHANGEZ: ts = q.schangeZ; break;
            case FD3D_PLANE_RVEL: ds = rvel_d; break;        case FD3D_PLANE_CZONE: ds = czone_d; break;
            default: return FD3D_ERR_ARG;
        }
        if (ds) {
            CK(cudaMemcpyAsync(host, ds, n2 * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        } else {
            std::vector<T> v(n2);
            CK(cudaMemcpyAsync(v.data(), ts, n2 * sizeof(T), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (size_t k = 0; k < n2; ++k) host[k] = (double)v[k];
        }
        return FD3D_OK;
    }

    int moment_rate(int rec0, int nrec, double* host) override {
        if (slab) return FD3D_ERR_STATE;  // a sum over the whole fault plane
        for (int r0 = 0; r0 < nrec; r0 += hist_cap) {  // at most one ring of records per pass
            const int n = std::min(hist_cap, nrec - r0);
            k_moment_rate<T><<<n, POST_THREADS, 0, st>>>(g, f, (const T*)ring, hist_cap, nf, rec0 + r0, (double)c.dh,
                                                         mrate_d);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(host + r0, mrate_d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        return FD3D_OK;
    }

    int post(double* out4) override {
        if (slab) return FD3D_ERR_STATE;  // sums over the whole fault plane
        const double dh2 = (double)(c.dh * c.dh);  // dh*dh in the field type, as the reference
        k_post<T><<<POST_BLOCKS, POST_THREADS, 0, st>>>(g, f, q, (double)c.dh, dh2, rvel_d, czone_d, part_d);
        k_post_sum<<<1, POST_THREADS, 0, st>>>(part_d, POST_BLOCKS, sums_d);
        CK(cudaGetLastError());
        double s[POST_NSUM];
        CK(cudaMemcpyAsync(s, sums_d, sizeof(s), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        out4[0] = s[3] / s[4];                          // average rupture speed (tint / tint2)
        out4[1] = s[0];                                 // seismic moment M0
        out4[2] = 0.0;                                  // rupture area: never set by the reference
        out4[3] = s[2] != 0.0 ? -(s[1] / s[2]) : 0.0;   // average stress drop
        return FD3D_OK;
    }
};

}  // namespace fd3d

struct fd3d_ctx {
    CtxBase* impl;
};

extern "C" {

const char* fd3d_version(void) { return "fd3d-b200 0.1 (sm_100a)"; }

int fd3d_struct_sizes(size_t* params_bytes, size_t* fault_bytes) {
    if (!params_bytes || !fault_bytes) return FD3D_ERR_ARG;
    *params_bytes = sizeof(fd3d_params);
    *fault_bytes = sizeof(fd3d_fault);
    return FD3D_OK;
}

const char* fd3d_status_string(int s) {
    switch (s) {
        case FD3D_OK: return "ok";
        case FD3D_ERR_ARG: return "bad argument";
        case FD3D_ERR_CFL: return "CFL > 0.25: simulation would be numerically unstable";
        case FD3D_ERR_CUDA: return "CUDA runtime error";
        case FD3D_ERR_NOMEM: return "out of device memory / HBM budget";
        case FD3D_ERR_NEWTON: return "FVW Newton solve did not converge";
        case FD3D_ERR_NONFINITE: return "non-finite value on the fault plane";
        case FD3D_ERR_STATE: return "call out of order";
        case FD3D_ERR_IO: return "file I/O error";
        case FD3D_ERR_NODEV: return "no CUDA device";
        case FD3D_ERR_BUSY: return "no free slot";
        case FD3D_ERR_TIMEOUT: return "a bounded device-side wait timed out";
        default: return "unknown status";
    }
}

int fd3d_device_count(int* count) {
    if (!count) return FD3D_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); *count = 0; return FD3D_OK; }
    *count = n;
    return FD3D_OK;
}

int fd3d_set_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return FD3D_ERR_NODEV; }
    if (dev < 0 || dev >= n) return FD3D_ERR_ARG;
    CK(cudaSetDevice(dev));
    return FD3D_OK;
}

static int create_ctx(const fd3d_params* p, int slab_lo, int slab_hi, fd3d_ctx** out) {
    if (!out) return FD3D_ERR_ARG;
    *out = nullptr;
    int rc = validate_params(p);
    if (rc) return rc;
    const bool slab = slab_lo > 0;
    if (slab && !slab_range_ok(*p, slab_lo, slab_hi)) return FD3D_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return FD3D_ERR_NODEV; }
    CtxBase* c = (p->precision == FD3D_PREC_F64) ? (CtxBase*)new Ctx<double>() : (CtxBase*)new Ctx<float>();
    c->p = *p;
    c->slab = slab;
    c->slab_lo = slab_lo;
    c->slab_hi = slab_hi;
    // manual override of the interior sweep variant: FD3D_INTERIOR=point|tiled|pipe,
    // FD3D_KCHUNK=<planes per CTA>, FD3D_BY=<CTA rows of the point kernel>
    if (const char* e = std::getenv("FD3D_INTERIOR")) {
        if (!std::strcmp(e, "point")) c->icfg.variant = IV_POINT;
        else if (!std::strcmp(e, "tiled")) c->icfg.variant = IV_TILED;
        else if (!std::strcmp(e, "pipe")) c->icfg.variant = IV_PIPE;
        else if (!std::strcmp(e, "tma")) c->icfg.variant = IV_TMA;
    }
    if (const char* e = std::getenv("FD3D_KCHUNK")) {
        c->icfg.kchunk = c->icfg.kchunk_str = std::max(1, std::atoi(e));
        c->icfg.kchunk_auto = false;
    }
    if (const char* e = std::getenv("FD3D_KCHUNK_STR")) {
        c->icfg.kchunk_str = std::max(1, std::atoi(e));
        c->icfg.kchunk_auto = false;
    }
    if (const char* e = std::getenv("FD3D_BY")) c->icfg.by = std::min(32, std::max(1, std::atoi(e)));
    // FD3D_PML_MINB=<v>[,<s>]: CTAs per SM the velocity / stress PML sweeps are compiled for
    if (const char* e = std::getenv("FD3D_PML_MINB")) {
        int v = 1, s = 0;
        const int n = std::sscanf(e, "%d,%d", &v, &s);
        c->pml_minb_vel = std::min(4, std::max(1, v));
        c->pml_minb_str = n == 2 ? std::min(4, std::max(1, s)) : c->pml_minb_vel;
    }
    if (slab && c->icfg.variant != IV_TMA) { delete c; return FD3D_ERR_ARG; }  // z-slabs: the TMA sweeps only
    rc = c->alloc();
    if (rc) {
        delete c;
        return rc == FD3D_ERR_CUDA ? FD3D_ERR_NOMEM : rc;
    }
    *out = new fd3d_ctx{c};
    return FD3D_OK;
}

int fd3d_ctx_create(const fd3d_params* p, fd3d_ctx** out) { return create_ctx(p, 0, 0, out); }

int fd3d_ctx_create_slab(const fd3d_params* p, int k_lo, int k_hi, fd3d_ctx** out) {
    if (k_lo < 1) return FD3D_ERR_ARG;
    return create_ctx(p, k_lo, k_hi, out);
}

int fd3d_slab_range(fd3d_ctx* ctx, int* k_lo, int* k_hi) {
    if (!ctx || !k_lo || !k_hi) return FD3D_ERR_ARG;
    *k_lo = ctx->impl->g.klo;
    *k_hi = ctx->impl->g.khi;
    return FD3D_OK;
}

int fd3d_ctx_destroy(fd3d_ctx* ctx) {
    if (!ctx) return FD3D_ERR_ARG;
    if (ctx->impl->st) cudaStreamSynchronize(ctx->impl->st);
    delete ctx->impl;
    delete ctx;
    return FD3D_OK;
}

// file layout: magic, sizeof(fd3d_params), the parameters, then the context's state
static const char CKPT_MAGIC[8] = {'F', 'D', '3', 'D', 'C', 'K', 'P', '1'};

int fd3d_checkpoint(fd3d_ctx* ctx, const char* path) {
    fd3d::TraceRange trace_("fd3d_checkpoint");
    if (!ctx || !path) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    std::FILE* fp = std::fopen(path, "wb");
    if (!fp) return FD3D_ERR_IO;
    const unsigned psz = sizeof(fd3d_params);
    int rc = (std::fwrite(CKPT_MAGIC, 1, 8, fp) == 8 && std::fwrite(&psz, sizeof psz, 1, fp) == 1 &&
              std::fwrite(&c->p, sizeof(fd3d_params), 1, fp) == 1)
                 ? c->save_state(fp) : FD3D_ERR_IO;
    if (std::fclose(fp) != 0 && rc == FD3D_OK) rc = FD3D_ERR_IO;
    return rc;
}

int fd3d_restore(const char* path, fd3d_ctx** out) {
    fd3d::TraceRange trace_("fd3d_restore");
    if (!path || !out) return FD3D_ERR_ARG;
    *out = nullptr;
    std::FILE* fp = std::fopen(path, "rb");
    if (!fp) return FD3D_ERR_IO;
    char magic[8];
    unsigned psz = 0;
    fd3d_params p{};
    int rc = FD3D_OK;
    if (std::fread(magic, 1, 8, fp) != 8 || std::memcmp(magic, CKPT_MAGIC, 8) != 0 ||
        std::fread(&psz, sizeof psz, 1, fp) != 1 || psz != sizeof(fd3d_params) ||
        std::fread(&p, sizeof p, 1, fp) != 1)
        rc = FD3D_ERR_IO;
    if (rc == FD3D_OK) rc = fd3d_ctx_create(&p, out);
    if (rc == FD3D_OK) {
        rc = (*out)->impl->load_state(fp);
        if (rc != FD3D_OK) { fd3d_ctx_destroy(*out); *out = nullptr; }
    }
    std::fclose(fp);
    return rc;
}

int fd3d_upload_medium(fd3d_ctx* ctx, const void* l, const void* m, const void* d, int rk) {
    fd3d::TraceRange trace_("fd3d_upload_medium");
    if (!ctx) return FD3D_ERR_ARG;
    return ctx->impl->upload_medium(l, m, d, rk);
}

int fd3d_upload_medium_layers(fd3d_ctx* ctx, const double* l, const double* m, const double* d) {
    fd3d::TraceRange trace_("fd3d_upload_medium_layers");
    if (!ctx) return FD3D_ERR_ARG;
    return ctx->impl->upload_medium_layers(l, m, d);
}

int fd3d_upload_fault(fd3d_ctx* ctx, const fd3d_fault* f) {
    fd3d::TraceRange trace_("fd3d_upload_fault");
    if (!ctx) return FD3D_ERR_ARG;
    return ctx->impl->upload_fault(f);
}

int fd3d_reset(fd3d_ctx* ctx) {
    if (!ctx) return FD3D_ERR_ARG;
    return ctx->impl->reset();
}

// graph g of the context holds 32 >> g time steps (captured on first use)
static int get_graph(CtxBase* c, int g, cudaGraphExec_t* out) {
    if (!c->gexec[g]) {
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < (32 >> g); ++s) c->enqueue_step();
        CK(cudaStreamEndCapture(c->st, &gr));
        cudaError_t e = cudaGraphInstantiate(&c->gexec[g], gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) { c->gexec[g] = nullptr; return FD3D_ERR_CUDA; }
    }
    *out = c->gexec[g];
    return FD3D_OK;
}

int fd3d_run(fd3d_ctx* ctx, int nsteps) {
    fd3d::TraceRange trace_("fd3d_run");
    if (!ctx || nsteps < 0) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    DeviceGuard dg(c->device);
    if (!c->medium_ok || !c->fault_ok || c->slab) return FD3D_ERR_STATE;  // a z-slab steps in its group
    CK(cudaEventRecord(c->ev0, c->st));
    int left = nsteps;
    if (!c->profiling) {
        // the whole run as graph launches: chunks of 32 steps, the rest by its binary digits
        for (int g = 0; g < CtxBase::NGRAPH && left > 0; ++g) {
            const int n = 32 >> g;
            if (left < n) continue;
            cudaGraphExec_t gx;
            int rc = get_graph(c, g, &gx);
            if (rc) return rc;
            while (left >= n) {
                CK(cudaGraphLaunch(gx, c->st));
                left -= n;
            }
        }
    }
    for (int s = 0; s < left; ++s) c->enqueue_step();
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, c->st));
    c->steps_done += nsteps;
    c->mark_run();
    return FD3D_OK;
}

int fd3d_sync(fd3d_ctx* ctx) {
    if (!ctx) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    CK(cudaStreamSynchronize(c->st));
    CK(cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
    int st = 0;
    CK(cudaMemcpy(&st, c->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st & ST_TIMEOUT) return FD3D_ERR_TIMEOUT;
    if (st & ST_NONFINITE) return FD3D_ERR_NONFINITE;
    if (st & ST_NEWTON) return FD3D_ERR_NEWTON;
    return FD3D_OK;
}

int fd3d_steps_done(fd3d_ctx* ctx, int* it) {
    if (!ctx || !it) return FD3D_ERR_ARG;
    *it = ctx->impl->steps_done;
    return FD3D_OK;
}

int fd3d_last_run_ms(fd3d_ctx* ctx, float* ms) {
    if (!ctx || !ms) return FD3D_ERR_ARG;
    *ms = ctx->impl->last_ms;
    return FD3D_OK;
}

int fd3d_set_profiling(fd3d_ctx* ctx, int on) {
    if (!ctx) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    c->profiling = on != 0;
    for (int k = 0; k < FD3D_NKERNELS; ++k) { c->ktimes[k] = 0; c->klaunch[k] = 0; }
    return FD3D_OK;
}

int fd3d_kernel_times(fd3d_ctx* ctx, float* ms, int* launches) {
    if (!ctx || !ms) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    for (int k = 0; k < FD3D_NKERNELS; ++k) {
        ms[k] = c->ktimes[k];
        if (launches) launches[k] = c->klaunch[k];
    }
    return FD3D_OK;
}

int fd3d_ctx_info(fd3d_ctx* ctx, int* interior_variant, int* layered_medium) {
    if (!ctx) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    if (interior_variant) *interior_variant = c->icfg.variant;
    if (layered_medium) *layered_medium = c->layered() ? 1 : 0;
    return FD3D_OK;
}

int fd3d_history_records(fd3d_ctx* ctx, int* nrec) {
    if (!ctx || !nrec) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    *nrec = c->steps_done / c->p.history_stride;
    return FD3D_OK;
}

int fd3d_fetch_history(fd3d_ctx* ctx, int field, int rec0, int nrec, void* host, int rk) {
    fd3d::TraceRange trace_("fd3d_fetch_history");
    if (!ctx || !host || nrec < 0 || rec0 < 0 || (rk != 4 && rk != 8)) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    if (field < 0 || field >= c->nf) return FD3D_ERR_ARG;
    const int have = c->steps_done / c->p.history_stride;
    if (rec0 + nrec > have || rec0 < have - c->hist_cap) return FD3D_ERR_ARG;  // overwritten or not yet made
    CK(c->wait_steps((rec0 + nrec) * c->p.history_stride));
    const size_t plane = (size_t)(c->p.nxt - 2 * c->p.nabc) * (c->p.nzt - c->p.nfs - c->p.nabc);
    const size_t es = c->elem();
    if ((size_t)rk == es) {
        // same element type: the records go straight to the caller's buffer, one strided
        // copy per contiguous run of ring slots (a page-locked buffer makes it one DMA)
        for (int r = 0; r < nrec;) {
            const int slot = (rec0 + r) % c->hist_cap;
            const int run = std::min(nrec - r, c->hist_cap - slot);
            const char* src = (const char*)c->ring + ((size_t)slot * c->nf + field) * plane * es;
            CK(cudaMemcpy2D((char*)host + (size_t)r * plane * es, plane * es, src, (size_t)c->nf * plane * es,
                            plane * es, (size_t)run, cudaMemcpyDeviceToHost));
            r += run;
        }
        return FD3D_OK;
    }
    std::vector<char> buf(plane * es);
    for (int r = 0; r < nrec; ++r) {
        const size_t slot = (size_t)((rec0 + r) % c->hist_cap);
        const char* src = (const char*)c->ring + (slot * c->nf + field) * plane * es;
        CK(cudaMemcpy(buf.data(), src, plane * es, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < plane; ++k) {
            double v = es == 4 ? (double)((float*)buf.data())[k] : ((double*)buf.data())[k];
            if (rk == 8) ((double*)host)[(size_t)r * plane + k] = v;
            else ((float*)host)[(size_t)r * plane + k] = (float)v;
        }
    }
    return FD3D_OK;
}

int fd3d_fetch_stations(fd3d_ctx* ctx, int rec0, int nrec, double* host) {
    if (!ctx || !host || nrec < 0 || rec0 < 0) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    const int have = c->steps_done / c->p.history_stride;
    if (rec0 + nrec > have || rec0 < have - c->hist_cap) return FD3D_ERR_ARG;
    CK(c->wait_steps((rec0 + nrec) * c->p.history_stride));
    const int ns = c->p.nstations;
    if (ns == 0) return FD3D_OK;
    const size_t es = c->elem();
    // the records are contiguous in the ring apart from its wrap: at most two copies
    std::vector<char> buf((size_t)nrec * 3 * ns * es);
    for (int r = 0; r < nrec;) {
        const int slot = (rec0 + r) % c->hist_cap;
        const int run = std::min(nrec - r, c->hist_cap - slot);
        CK(cudaMemcpy(buf.data() + (size_t)r * 3 * ns * es, (const char*)c->seis + (size_t)slot * 3 * ns * es,
                      (size_t)run * 3 * ns * es, cudaMemcpyDeviceToHost));
        r += run;
    }
    for (size_t q = 0; q < (size_t)nrec * 3 * ns; ++q)
        host[q] = es == 4 ? (double)((const float*)buf.data())[q] : ((const double*)buf.data())[q];
    return FD3D_OK;
}

int fd3d_fetch_field(fd3d_ctx* ctx, int field, void* host, int rk) {
    if (!ctx || !host) return FD3D_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->impl->st));
    return ctx->impl->fetch_field(field, host, rk);
}

int fd3d_fetch_plane(fd3d_ctx* ctx, int plane, double* host) {
    if (!ctx || !host) return FD3D_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->impl->st));
    return ctx->impl->fetch_plane(plane, host);
}

int fd3d_upload_fault_model(fd3d_ctx* ctx, int nli, int nwi, const double* T0I, const double* TsI, const double* DcI,
                            double dip, int dipslip) {
    fd3d::TraceRange trace_("fd3d_upload_fault_model");
    if (!ctx) return FD3D_ERR_ARG;
    return ctx->impl->upload_fault_model(nli, nwi, T0I, TsI, DcI, dip, dipslip);
}

int fd3d_fetch_moment_rate(fd3d_ctx* ctx, int rec0, int nrec, double* host) {
    if (!ctx || !host || nrec < 0 || rec0 < 0) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    const int have = c->steps_done / c->p.history_stride;
    if (rec0 + nrec > have || rec0 < have - c->hist_cap) return FD3D_ERR_ARG;  // overwritten or not yet made
    return c->moment_rate(rec0, nrec, host);
}

int fd3d_post_process(fd3d_ctx* ctx, double* out4) {
    if (!ctx || !out4) return FD3D_ERR_ARG;
    return ctx->impl->post(out4);
}

int fd3d_fetch_final(fd3d_ctx* ctx, double* slipX, double* slipZ, double* ruptime, double* rise, double* sliptime) {
    if (!ctx) return FD3D_ERR_ARG;
    int rc = 0;
    CtxBase* c = ctx->impl;
    const size_t n2 = (size_t)c->p.nxt * c->p.nzt;
    if (slipX) rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_SLIPX, slipX);
    if (slipZ) rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_SLIPZ, slipZ);
    std::vector<double> rt(n2);
    rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_RUPTIME, rt.data());
    if (ruptime) std::memcpy(ruptime, rt.data(), n2 * sizeof(double));
    if (rise) {  // rise = rise - ruptime (fd3d_theo.f90:658)
        rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_RISE, rise);
        for (size_t k = 0; k < n2; ++k) rise[k] = rise[k] - rt[k];
    }
    if (sliptime) rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_SLIPTIME, sliptime);
    return rc ? FD3D_ERR_CUDA : FD3D_OK;
}

int fd3d_write_results(fd3d_ctx* ctx, const char* dir, int rk) {
    fd3d::TraceRange trace_("fd3d_write_results");
    if (!ctx || !dir || (rk != 4 && rk != 8)) return FD3D_ERR_ARG;
    if (ctx->impl->slab) return FD3D_ERR_STATE;  // a z-slab holds part of the planes
    return fd3d::write_results(ctx, ctx->impl->p, ctx->impl->nf, ctx->impl->rec_written, dir, rk);
}


// ---------------------------------------------------------------- z-slab groups
// One model over several contexts (GPUs), each owning a range of planes.  A step runs in
// STEP_PHASES phases; after phases 0-3 every slab pulls the halo planes (or fault-plane
// rows) of the arrays its neighbours just updated, two on each side, into its own memory:
// one contiguous copy per array and side, since planes are the slowest index.  Each pull
// waits (cudaStreamWaitEvent) for the neighbour's phase; what a neighbour writes next is
// never what was just pulled from it until the next exchange of the same set, which in
// turn waits for this slab, so no slab overwrites data another is still copying.

// The two planes (or fault-plane rows) a slab owning k_lo..k_hi exchanges with its
// neighbour below (side 0) or above (side 1): it sends its own first / last two and receives
// the neighbour's into its halo.  Both transports use it; a slab's receive on one side is
// its neighbour's send on the other.
int fd3d_slab_halo_plan(int k_lo, int k_hi, int side, int* send_k0, int* recv_k0) {
    if (!send_k0 || !recv_k0 || (side != 0 && side != 1) || k_hi - k_lo + 1 < SLAB_MIN) return FD3D_ERR_ARG;
    *send_k0 = side == 0 ? k_lo : k_hi - 1;
    *recv_k0 = side == 0 ? k_lo - 2 : k_hi + 1;
    return FD3D_OK;
}

// Planes 1..nzt in n slabs of about equal cost (a PML cell moves about 2.2 times the
// bytes of an interior cell), every slab valid for slab_range_ok.
int fd3d_slab_plan(const fd3d_params* p, int n, int* k_lo, int* k_hi) {
    if (!p || n < 1 || !k_lo || !k_hi) return FD3D_ERR_ARG;
    int rc = validate_params(p);
    if (rc) return rc;
    const int nzt = p->nzt, nab = p->nabc, ks = nzt - p->nfs;
    std::vector<double> w(nzt + 1, 0.0), cum(nzt + 1, 0.0);
    const double plane = (double)p->nxt * p->nyt;
    const double pml_cols = 2.0 * nab * p->nyt + (double)nab * (p->nxt - 2 * nab);
    for (int k = 1; k <= nzt; ++k) {
        const bool zpml = k <= nab || (p->fspace && k > ks);
        w[k] = zpml ? 2.2 * plane : (plane - pml_cols) + 2.2 * pml_cols;
        cum[k] = cum[k - 1] + w[k];
    }
    int k = 0;
    for (int r = 0; r < n; ++r) {
        k_lo[r] = k + 1;
        if (r == n - 1) { k_hi[r] = nzt; break; }
        const double target = cum[nzt] * (r + 1) / n;
        int e = k + SLAB_MIN;
        while (e < nzt && cum[e] < target) ++e;
        e = std::min(e, ks - 3);                                  // the top slab owns ks-2 .. nzt
        e = std::min(e, ks - 3 - SLAB_MIN * (n - 2 - r));         // room for the slabs still to come
        k_hi[r] = e;
        k = e;
    }
    for (int r = 0; r < n; ++r)
        if (!slab_range_ok(*p, k_lo[r], k_hi[r]) || (r > 0 && k_lo[r] != k_hi[r - 1] + 1)) return FD3D_ERR_ARG;
    return FD3D_OK;
}

struct fd3d_slab_group {
    std::vector<fd3d::CtxBase*> r;
    std::vector<cudaEvent_t> ev;   // per slab: its last phase is enqueued up to here
};

int fd3d_slab_group_create(fd3d_ctx* const* ctxs, int n, fd3d_slab_group** out) {
    if (!ctxs || n < 1 || !out) return FD3D_ERR_ARG;
    *out = nullptr;
    std::vector<CtxBase*> r(n);
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i] || !ctxs[i]->impl->slab) return FD3D_ERR_ARG;
        r[i] = ctxs[i]->impl;
    }
    // one model: same parameters, same field type, planes 1..nzt covered in order
    for (int i = 0; i < n; ++i) {
        const fd3d_params &a = r[i]->p, &b = r[0]->p;
        if (a.nxt != b.nxt || a.nyt != b.nyt || a.nzt != b.nzt || a.nabc != b.nabc || a.fspace != b.fspace ||
            a.law != b.law || a.precision != b.precision || a.dt != b.dt || a.dh != b.dh)
            return FD3D_ERR_ARG;
        if (r[i]->g.klo != (i == 0 ? 1 : r[i - 1]->g.khi + 1)) return FD3D_ERR_ARG;
    }
    if (r[n - 1]->g.khi != r[0]->p.nzt) return FD3D_ERR_ARG;
    auto* G = new fd3d_slab_group;
    G->r = r;
    G->ev.assign(n, nullptr);
    for (int i = 0; i < n; ++i) {
        DeviceGuard dg(r[i]->device);
        if (cudaEventCreateWithFlags(&G->ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            for (auto e : G->ev) if (e) cudaEventDestroy(e);
            delete G;
            return FD3D_ERR_CUDA;
        }
        // neighbours on other devices: peer access for the pulls (a copy still works without)
        for (int nb : {i - 1, i + 1})
            if (nb >= 0 && nb < n && r[nb]->device != r[i]->device) {
                int can = 0;
                if (cudaDeviceCanAccessPeer(&can, r[i]->device, r[nb]->device) == cudaSuccess && can)
                    cudaDeviceEnablePeerAccess(r[nb]->device, 0);
                cudaGetLastError();  // already enabled is fine
            }
    }
    *out = G;
    return FD3D_OK;
}

int fd3d_slab_group_destroy(fd3d_slab_group* G) {
    if (!G) return FD3D_ERR_ARG;
    for (size_t i = 0; i < G->r.size(); ++i) {
        DeviceGuard dg(G->r[i]->device);
        cudaStreamSynchronize(G->r[i]->st);
        if (G->ev[i]) cudaEventDestroy(G->ev[i]);
    }
    delete G;
    return FD3D_OK;
}

// pull two planes / rows of every array of the set from the slab below (its top two) and
// from the slab above (its bottom two) into slab i's halo
static int slab_exchange(fd3d_slab_group* G, int set) {
    const int n = (int)G->r.size();
    std::vector<std::vector<HaloArray>> arr(n);
    for (int i = 0; i < n; ++i) {
        DeviceGuard dg(G->r[i]->device);
        int rc = G->r[i]->halo_arrays(set, arr[i]);
        if (rc) return rc;
        CK(cudaEventRecord(G->ev[i], G->r[i]->st));
    }
    for (int i = 0; i < n; ++i) {
        CtxBase* c = G->r[i];
        DeviceGuard dg(c->device);
        for (int side = 0; side < 2; ++side) {
            const int nb = side == 0 ? i - 1 : i + 1;
            if (nb < 0 || nb >= n) continue;
            CK(cudaStreamWaitEvent(c->st, G->ev[nb], 0));
            int send_k0 = 0, recv_k0 = 0;  // pull into the halo: the neighbour's send planes
            fd3d_slab_halo_plan(c->g.klo, c->g.khi, side, &send_k0, &recv_k0);
            const long long k0 = recv_k0;
            for (size_t a = 0; a < arr[i].size(); ++a) {
                const HaloArray &d = arr[i][a], &s = arr[nb][a];
                const size_t off = d.unit * (size_t)(k0 - 1) * d.elem, bytes = 2 * d.unit * d.elem;
                CK(cudaMemcpyAsync((char*)d.base + off, (const char*)s.base + off, bytes, cudaMemcpyDefault, c->st));
            }
        }
    }
    return FD3D_OK;
}

int fd3d_slab_group_run(fd3d_slab_group* G, int nsteps) {
    fd3d::TraceRange trace_("fd3d_slab_group_run");
    if (!G || nsteps < 0) return FD3D_ERR_ARG;
    for (CtxBase* c : G->r)
        if (!c->medium_ok || !c->fault_ok) return FD3D_ERR_STATE;
    for (CtxBase* c : G->r) {
        DeviceGuard dg(c->device);
        CK(cudaEventRecord(c->ev0, c->st));
    }
    for (int s = 0; s < nsteps; ++s)
        for (int ph = 0; ph < STEP_PHASES; ++ph) {
            for (CtxBase* c : G->r) {
                DeviceGuard dg(c->device);
                int rc = c->enqueue_phase(ph);
                if (rc) return rc;
            }
            const int set = halo_after_phase(ph);
            if (set != HALO_NONE && G->r.size() > 1) {
                int rc = slab_exchange(G, set);
                if (rc) return rc;
            }
        }
    for (CtxBase* c : G->r) {
        DeviceGuard dg(c->device);
        CK(cudaGetLastError());
        CK(cudaEventRecord(c->ev1, c->st));
        c->steps_done += nsteps;
        c->mark_run();
    }
    return FD3D_OK;
}

// wait for every slab; the run time is the longest slab's; the first error status of any
int fd3d_slab_group_sync(fd3d_slab_group* G, float* ms) {
    if (!G) return FD3D_ERR_ARG;
    int first = FD3D_OK;
    float worst = 0.f;
    for (size_t i = 0; i < G->r.size(); ++i) {
        DeviceGuard dg(G->r[i]->device);
        fd3d_ctx tmp{G->r[i]};
        const int rc = fd3d_sync(&tmp);
        if (rc && !first) first = rc;
        worst = std::max(worst, G->r[i]->last_ms);
    }
    if (ms) *ms = worst;
    return first;
}


// ---- z-slabs in separate processes (one GPU each): the halo exchange over NCCL --------
int fd3d_nccl_unique_id(unsigned char* id) {
    if (!id) return FD3D_ERR_ARG;
    const NcclApi& n = nccl();
    if (!n.ok) return FD3D_ERR_NODEV;
    ncclUniqueId u;
    if (n.GetUniqueId(&u) != ncclSuccess) return FD3D_ERR_CUDA;
    std::memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
    return FD3D_OK;
}

int fd3d_slab_connect(fd3d_ctx* ctx, const unsigned char* id, int rank, int nranks) {
    if (!ctx || !id || nranks < 1 || rank < 0 || rank >= nranks) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    if (!c->slab || c->comm) return FD3D_ERR_STATE;
    const NcclApi& n = nccl();
    if (!n.ok) return FD3D_ERR_NODEV;
    DeviceGuard dg(c->device);
    ncclUniqueId u;
    std::memcpy(u.internal, id, NCCL_UNIQUE_ID_BYTES);
    ncclComm_t comm = nullptr;
    if (n.CommInitRank(&comm, nranks, u, rank) != ncclSuccess) return FD3D_ERR_CUDA;
    // every rank's plane range: rank r must hold the r-th slab from the bottom
    int* d = nullptr;
    std::vector<int> all(2 * (size_t)nranks);
    const int mine[2] = {c->g.klo, c->g.khi};
    bool ok = cudaMalloc(&d, sizeof(int) * 2 * (nranks + 1)) == cudaSuccess &&
              cudaMemcpyAsync(d, mine, sizeof mine, cudaMemcpyHostToDevice, c->st) == cudaSuccess &&
              n.AllGather(d, d + 2, 2, ncclInt, comm, c->st) == ncclSuccess &&
              cudaMemcpyAsync(all.data(), d + 2, sizeof(int) * 2 * nranks, cudaMemcpyDeviceToHost, c->st) == cudaSuccess &&
              cudaStreamSynchronize(c->st) == cudaSuccess;
    if (d) cudaFree(d);
    cudaGetLastError();
    for (int r = 0; ok && r < nranks; ++r)
        ok = all[2 * r] == (r == 0 ? 1 : all[2 * r - 1] + 1) && (r < nranks - 1 || all[2 * r + 1] == c->p.nzt);
    if (!ok) { n.CommDestroy(comm); return FD3D_ERR_ARG; }
    c->comm = comm;
    c->slab_rank = rank;
    c->slab_nranks = nranks;
    return FD3D_OK;
}

// the exchange of one halo set with the ranks below and above: the same planes / rows as
// slab_exchange, each sent as two contiguous planes / rows and received into the halo
static int nccl_exchange(CtxBase* c, int set) {
    std::vector<HaloArray> arr;
    int rc = c->halo_arrays(set, arr);
    if (rc) return rc;
    const NcclApi& n = nccl();
    if (n.GroupStart() != ncclSuccess) return FD3D_ERR_CUDA;
    bool ok = true;
    for (int side = 0; side < 2; ++side) {
        const int nb = side == 0 ? c->slab_rank - 1 : c->slab_rank + 1;
        if (nb < 0 || nb >= c->slab_nranks) continue;
        int send_k0 = 0, recv_k0 = 0;
        fd3d_slab_halo_plan(c->g.klo, c->g.khi, side, &send_k0, &recv_k0);
        for (const HaloArray& a : arr) {
            const size_t bytes = 2 * a.unit * a.elem;
            ok &= n.Send((const char*)a.base + a.unit * (size_t)(send_k0 - 1) * a.elem, bytes, ncclChar, nb, c->comm,
                         c->st) == ncclSuccess;
            ok &= n.Recv((char*)a.base + a.unit * (size_t)(recv_k0 - 1) * a.elem, bytes, ncclChar, nb, c->comm,
                         c->st) == ncclSuccess;
        }
    }
    ok &= n.GroupEnd() == ncclSuccess;
    return ok ? FD3D_OK : FD3D_ERR_CUDA;
}

int fd3d_slab_run(fd3d_ctx* ctx, int nsteps) {
    fd3d::TraceRange trace_("fd3d_slab_run");
    if (!ctx || nsteps < 0) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    if (!c->slab || !c->comm || !c->medium_ok || !c->fault_ok) return FD3D_ERR_STATE;
    DeviceGuard dg(c->device);
    CK(cudaEventRecord(c->ev0, c->st));
    for (int s = 0; s < nsteps; ++s)
        for (int ph = 0; ph < STEP_PHASES; ++ph) {
            int rc = c->enqueue_phase(ph);
            if (rc) return rc;
            const int set = halo_after_phase(ph);
            if (set != HALO_NONE && c->slab_nranks > 1) {
                rc = nccl_exchange(c, set);
                if (rc) return rc;
            }
        }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, c->st));
    c->steps_done += nsteps;
    c->mark_run();
    return FD3D_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// fd3d_run_noalloc: the time step with the fault boundary condition as separate launches
// (fres, trial traction, friction, output) whose trial-traction scratch is taken from a
// fixed, file-scope device array instead of memory the library allocates.  Meant for
// hosts that cannot let the library allocate device memory once their run has started
// (their device memory is handed out by another runtime, such as the OpenACC present
// table of a Fortran host, or was reserved up front against a fixed budget).  fd3d_run
// may allocate on its first call (it instantiates a CUDA graph of the step); this entry
// point launches the kernels one by one and calls no cudaMalloc, cudaFree or other
// allocating routine.  The array's device address is looked up once per device and kept
// for the life of the process, so a device reset (cudaDeviceReset) between calls is not
// supported.
//
// Limit: nxt*nzt <= FD3D_NOALLOC_MAX_PLANE fault-plane nodes (the array holds two
// planes of doubles, 16 MiB, on every GPU that loads the library, until exit).
// The array is shared by every call on a device and keeps the last call's contents;
// calls whose work overlaps on a GPU (several contexts on different streams) race on it.
// ---------------------------------------------------------------------------
#include <mutex>

#define FD3D_NOALLOC_MAX_PLANE (1 << 20)

static __device__ __align__(256) unsigned char fd3d_noalloc_scratch[2ull * FD3D_NOALLOC_MAX_PLANE * sizeof(double)];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {};  // device address of fd3d_noalloc_scratch, per device ordinal

// once per device, with that device current: the host-side name of the array is not a
// device address, so the kernels get the address returned by cudaGetSymbolAddress
int noalloc_scratch(int dev, void** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (dev < 0 || dev >= 256) return FD3D_ERR_ARG;
    if (!g_noalloc_addr[dev]) {
        int cur = -1;
        if (cudaGetDevice(&cur) != cudaSuccess) return FD3D_ERR_CUDA;
        if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return FD3D_ERR_CUDA;
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, fd3d_noalloc_scratch);
        if (cur != dev) cudaSetDevice(cur);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "fd3d_run_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return FD3D_ERR_CUDA;
        }
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return FD3D_OK;
}

template <class T>
int run_noalloc_t(Ctx<T>* c, int nsteps, void* scratch) {
    const size_t n2 = (size_t)c->p.nxt * c->p.nzt;
    // cells outside the interior plane are read as zero by the friction launch
    CK(cudaMemsetAsync(scratch, 0, 2 * n2 * sizeof(T), c->st));
    CK(cudaEventRecord(c->ev0, c->st));
    T* const txt0 = c->q.txt;
    T* const tzt0 = c->q.tzt;
    c->q.txt = (T*)scratch;
    c->q.tzt = (T*)scratch + n2;
    c->split_bc = true;
    for (int s = 0; s < nsteps; ++s) c->enqueue_step();
    c->split_bc = false;
    c->q.txt = txt0;
    c->q.tzt = tzt0;
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, c->st));
    c->steps_done += nsteps;
    c->mark_run();
    return FD3D_OK;
}
}  // namespace

extern "C" int fd3d_run_noalloc(fd3d_ctx* ctx, int nsteps) {
    fd3d::TraceRange trace_("fd3d_run_noalloc");
    if (!ctx || nsteps < 0) return FD3D_ERR_ARG;
    CtxBase* c = ctx->impl;
    if (!c->medium_ok || !c->fault_ok || c->slab) return FD3D_ERR_STATE;
    const long long n2 = (long long)c->p.nxt * c->p.nzt;
    if (n2 > FD3D_NOALLOC_MAX_PLANE) {
        std::fprintf(stderr, "fd3d_run_noalloc: fault plane nxt*nzt = %lld nodes exceeds the limit of %d\n", n2,
                     FD3D_NOALLOC_MAX_PLANE);
        return FD3D_ERR_ARG;
    }
    DeviceGuard dg(c->device);  // the memset and the launches go to the context's device
    void* scratch = nullptr;
    int rc = noalloc_scratch(c->device, &scratch);
    if (rc) return rc;
    if (auto* cf = dynamic_cast<Ctx<float>*>(c)) return run_noalloc_t(cf, nsteps, scratch);
    if (auto* cd = dynamic_cast<Ctx<double>*>(c)) return run_noalloc_t(cd, nsteps, scratch);
    return FD3D_ERR_STATE;
}
