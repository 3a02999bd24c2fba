// fd3d_batch.cu -- many independent forward models in one launch schedule.
//
// Models of uneven size live in one device arena (first-fit, 256-byte aligned blocks,
// each with its own padded pitch).  Their work is a host-built list of (model, tile)
// items.  Two schedules run it: the persistent one is one cooperative kernel per run
// whose CTAs walk the items phase by phase and meet at a bounded grid-wide barrier
// between phases; the graph one replays CUDA graphs of per-region kernels over all
// models (see k_bint).  A time step has five phases:
//   0 velocity: interior tiles, fault band + fault plane, PML chunks
//   1 free-surface velocity ghosts
//   2 stress: interior tiles, fault band + fault plane, PML chunks
//   3 fault boundary condition: free-surface stress ghosts and the fused trial traction,
//     friction and output tiles (fault_bc_body)
//   4 nucleation ramp (rate-and-state models that have one; an empty phase is skipped)
// Every item runs the same __device__ body as the single-model launch of that region
// (fd3d_kernels.cuh / fd3d_opt.cuh), so a model's results do not depend on which other
// models share the launch.  The schedule, the z-extent of the interior tiles and (for
// the persistent kernel) the number of CTAs per SM are picked by an autotuner that
// times the candidates on the live batch (and resets the models after).
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>
#include "../../include/fd3d_gpu.h"
#include "fd3d_common.cuh"
#include "fd3d_kernels.cuh"
#include "fd3d_opt.cuh"
#include "fd3d_setup.h"
#include "fd3d_trace.h"

using namespace fd3d;

#define BCK(x)                                                                                  \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            std::fprintf(stderr, "fd3d batch: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                                   \
            return FD3D_ERR_CUDA;                                                               \
        }                                                                                       \
    } while (0)

namespace {

enum WorkType : int {
    W_VEL_INT = 0, W_VEL_FAULT, W_VEL_PML, W_VEL_FS, W_STR_INT, W_STR_FAULT, W_STR_PML, W_STR_FS, W_FBC, W_NUC
};
constexpr int NPHASE = 5;

struct Work {
    int tm;          // type | model << 8
    int bx, by, bz;
};

struct ModelDev {
    Grid g;
    Fields<float> f;
    Fault<float> q;
    StepConst<float> c;
    FvwScalars fs;
    PmlDesc D;
    PmlAux<float> X;
    HistDesc h;
    int law;
    int* it_dev;
    int* status;
    double* psiX0;
    double* psiZ0;
};

struct BatchSync {
    unsigned count;
    unsigned gen;
    int abort;
    int pad;
};

constexpr int BARRIER_SPIN_LIMIT = 1 << 22;

// Sense-counting grid barrier with a bounded spin; false if this CTA gave up (or another did).
__device__ bool grid_barrier(BatchSync* b, unsigned nblocks, int* status) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        ok = 1;
        volatile unsigned* vgen = &b->gen;
        volatile int* vab = &b->abort;
        const unsigned g0 = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&b->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            int n = 0;
            while (*vgen == g0) {
                if (*vab) { ok = 0; break; }
                if (++n > BARRIER_SPIN_LIMIT) {
                    atomicOr(status, ST_TIMEOUT);
                    atomicExch(&b->abort, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

struct ModelMaps {  // TMA descriptors of one model's interior sweeps (global memory, 64-byte aligned)
    VelMaps v;
    StrMaps s;
};

#ifndef FD3D_BATCH_MINB
#define FD3D_BATCH_MINB 3
#endif
constexpr int BATCH_MIN_CTAS = FD3D_BATCH_MINB;  // register cap so that this many CTAs of 256 threads fit an SM

__global__ void __launch_bounds__(256, BATCH_MIN_CTAS)
k_batch(const ModelDev* __restrict__ models, const ModelMaps* __restrict__ maps, const Work* __restrict__ work,
        const int* __restrict__ pbeg, const int* __restrict__ limit, int nsteps, int kchunk, BatchSync* sync,
        int* gstatus) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* ring = reinterpret_cast<float*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    __shared__ __align__(8) uint64_t bars[TMA_NS];
    __shared__ __align__(8) uint64_t pbar;  // PML tiles staged through the ring memory
    if (threadIdx.x == 0 && threadIdx.y == 0) mbar_init(smem_addr(&pbar), 1);
    tma_ring_init(bars);
    unsigned pc = 0;  // planes this CTA has put through its ring
    unsigned pt = 0;  // PML tiles this CTA has staged (mbarrier phase = pt & 1)
    const unsigned nb = gridDim.x;
    for (int s = 0; s < nsteps; ++s) {
        for (int ph = 0; ph < NPHASE; ++ph) {
            const int b0 = pbeg[ph], b1 = pbeg[ph + 1];
            if (b0 == b1) continue;  // an empty phase needs no barrier (uniform over the grid)
            for (int w = b0 + blockIdx.x; w < b1; w += nb) {
                const Work it = work[w];
                const int m = it.tm >> 8, type = it.tm & 255;
                if (s >= limit[m]) continue;  // uniform over the CTA: the item belongs to one model
                const ModelDev& M = models[m];
                bool ok = true;
                switch (type) {
                    case W_VEL_INT:
                        ok = vel_interior_tma_body<float, true>(maps[m].v, M.g, M.f, M.c, kchunk, it.bx, it.by, it.bz,
                                                                ring, bars, pc, gstatus);
                        break;
                    case W_VEL_FAULT:
                        vel_fault_body<float>(M.g, M.f, M.q, M.c, M.law, M.fs, M.it_dev, M.status, it.bx, it.by, 0);
                        break;
                    case W_VEL_PML:
                        ok = vel_pml_tile<float>(M.g, M.f, M.D, M.X, M.c, it.bx, ring, smem_addr(&pbar), pt & 1u,
                                                 gstatus);
                        ++pt;
                        break;
                    case W_VEL_FS: vel_fs_body<float>(M.g, M.f, it.bx, it.by, 0); break;
                    case W_STR_INT:
                        ok = str_interior_tma_body<float, true>(maps[m].s, M.g, M.f, M.c, kchunk, it.bx, it.by, it.bz,
                                                                ring, bars, pc, gstatus);
                        break;
                    case W_STR_FAULT: str_fault_body<float>(M.g, M.f, M.q, M.c, it.bx, it.by, 0); break;
                    case W_STR_PML:
                        ok = str_pml_tile<float>(M.g, M.f, M.D, M.X, M.c, it.bx, ring, smem_addr(&pbar), pt & 1u,
                                                 gstatus);
                        ++pt;
                        break;
                    case W_STR_FS: str_fs_body<float>(M.g, M.f, it.bx, it.by, 0); break;
                    case W_FBC:
                        fault_bc_body<float>(M.g, M.f, M.q, M.c, M.law, M.fs, M.it_dev, M.h, M.status, it.bx, it.by,
                                             ring);
                        break;
                    case W_NUC: nucleation_body<float>(M.g, M.q, M.c, M.fs, M.it_dev, it.bx, it.by, 0); break;
                    default: break;
                }
                if (!ok) {  // a ring wait timed out: make every CTA leave at its next barrier
                    if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(&sync->abort, 1);
                    return;
                }
                __syncthreads();  // the next item may reuse the ring
            }
            if (!grid_barrier(sync, nb, gstatus)) return;
        }
    }
}

// ---------------------------------------------------------------- self-test of the waits
// An mbarrier phase that no copy or arrival completes, and a grid barrier that one CTA
// never reaches: both waits must give up by their bound, record ST_TIMEOUT and return,
// leaving the context usable (failure detection without a hung or faulted GPU).
__global__ void k_check_mbar_wait(int* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) { mbar_init(smem_addr(&bar), 1); fence_mbar_init(); }
    __syncthreads();
    const bool done = mbar_wait(smem_addr(&bar), 0u);  // nothing ever arrives on this phase
    if (__syncthreads_or(!done) && threadIdx.x == 0) atomicOr(status, ST_TIMEOUT);
}

__global__ void k_check_grid_barrier(BatchSync* sync, int* status) {
    if (blockIdx.x == gridDim.x - 1) return;  // this CTA never arrives
    grid_barrier(sync, gridDim.x, status);
}

// ---------------------------------------------------------------- graph schedule
// The same items as k_batch, one kernel per region and step, every CTA one item.
// A CUDA graph holds a chunk of steps: per step the interior, fault-band and PML
// sweeps of a half-step run as three parallel branches, the plane regions follow in
// order, and k_step_end advances the run's step counter (items of a model whose
// step limit is reached return at once).  Each kernel gets its own register and
// shared-memory budget, so each region runs at its own occupancy.
constexpr int NTYPES = 10;

__device__ __forceinline__ bool item_live(const Work& it, const int* limit, const int* run_step, int& m) {
    m = it.tm >> 8;
    return *run_step < limit[m];
}

template <bool STRESS>
__global__ void __launch_bounds__(256) k_bint(const ModelDev* __restrict__ models, const ModelMaps* __restrict__ maps,
                                              const Work* __restrict__ work, int b0, const int* __restrict__ limit,
                                              const int* run_step, int kchunk, int* gstatus) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* ring = reinterpret_cast<float*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    __shared__ __align__(8) uint64_t bars[TMA_NS];
    pdl_wait();
    pdl_launch_dependents();
    const Work it = work[b0 + blockIdx.x];
    int m;
    if (!item_live(it, limit, run_step, m)) return;
    tma_ring_init(bars);
    const ModelDev& M = models[m];
    unsigned pc = 0;
    if (STRESS)
        str_interior_tma_body<float, true>(maps[m].s, M.g, M.f, M.c, kchunk, it.bx, it.by, it.bz, ring, bars, pc,
                                           gstatus);
    else
        vel_interior_tma_body<float, true>(maps[m].v, M.g, M.f, M.c, kchunk, it.bx, it.by, it.bz, ring, bars, pc,
                                           gstatus);
}

template <bool STRESS>
__global__ void __launch_bounds__(PML_TILE, 4) k_bpml(const ModelDev* __restrict__ models,
                                                      const Work* __restrict__ work, int b0,
                                                      const int* __restrict__ limit, const int* run_step,
                                                      int* gstatus) {
    __shared__ __align__(128) float sm[PML_TILE * (STRESS ? AUX_NS : AUX_NV)];
    __shared__ __align__(8) uint64_t bar;
    pdl_wait();
    pdl_launch_dependents();
    const Work it = work[b0 + blockIdx.x];
    int m;
    if (!item_live(it, limit, run_step, m)) return;
    if (threadIdx.x == 0 && threadIdx.y == 0) { mbar_init(smem_addr(&bar), 1); fence_mbar_init(); }
    const ModelDev& M = models[m];
    if (STRESS) str_pml_tile<float>(M.g, M.f, M.D, M.X, M.c, it.bx, sm, smem_addr(&bar), 0u, gstatus);
    else vel_pml_tile<float>(M.g, M.f, M.D, M.X, M.c, it.bx, sm, smem_addr(&bar), 0u, gstatus);
}

// Plane items in three kernels by register need, so that light items are not held to a
// heavy body's register count: KIND 1 the fused fault-BC tiles (and the fres items launched
// with them, 78 registers), KIND 2 the fault-band velocity (its rate-and-state Newton path
// takes 114), KIND 0 the rest (free surface, stress fault band, nucleation ramp).
template <int KIND>
__global__ void __launch_bounds__(256) k_bplane(const ModelDev* __restrict__ models, const Work* __restrict__ work,
                                                int b0, const int* __restrict__ limit, const int* run_step) {
    __shared__ float sm[KIND == 1 ? FBC_SMEM : 1];
    pdl_wait();
    pdl_launch_dependents();
    const Work it = work[b0 + blockIdx.x];
    int m;
    if (!item_live(it, limit, run_step, m)) return;
    const ModelDev& M = models[m];
    if (KIND == 2) {
        if ((it.tm & 255) == W_VEL_FAULT)
            vel_fault_body<float>(M.g, M.f, M.q, M.c, M.law, M.fs, M.it_dev, M.status, it.bx, it.by, 0);
        return;
    }
    if (KIND == 1) {
        if ((it.tm & 255) == W_FBC)
            fault_bc_body<float>(M.g, M.f, M.q, M.c, M.law, M.fs, M.it_dev, M.h, M.status, it.bx, it.by, sm);
        else if ((it.tm & 255) == W_STR_FS)
            str_fs_body<float>(M.g, M.f, it.bx, it.by, 0);
        return;
    }
    switch (it.tm & 255) {
        case W_VEL_FS: vel_fs_body<float>(M.g, M.f, it.bx, it.by, 0); break;
        case W_STR_FAULT: str_fault_body<float>(M.g, M.f, M.q, M.c, it.bx, it.by, 0); break;
        case W_STR_FS: str_fs_body<float>(M.g, M.f, it.bx, it.by, 0); break;
        case W_NUC: nucleation_body<float>(M.g, M.q, M.c, M.fs, M.it_dev, it.bx, it.by, 0); break;
        default: break;
    }
}

__global__ void k_step_end(int* run_step) {
    pdl_wait();
    pdl_launch_dependents();
    *run_step += 1;
}

// A launch of the graph schedule, with programmatic stream serialization when pdl is set:
// the kernel's CTAs may be scheduled while the kernel before it drains, and wait in
// pdl_wait (every kernel of the schedule starts with it) for its completion.
template <class... K, class... A>
static cudaError_t launch_g(bool pdl, void (*kern)(K...), unsigned grid, dim3 blk, size_t smem, cudaStream_t s,
                            A... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = blk;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

// OR of the live models' device status words into out (one read-back per sync)
__global__ void k_or_status(int* const* __restrict__ st, int n, int* out) {
    int v = 0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) v |= *st[q];
    v = __reduce_or_sync(0xffffffffu, v);
    __shared__ int acc;
    if (threadIdx.x == 0) acc = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicOr(&acc, v);
    __syncthreads();
    if (threadIdx.x == 0) *out = acc;
}

// 1-D layered medium -> padded 3-D arrays of one model
__global__ void k_fill_layers(Grid g, float* lam, float* mu, float* d, const float* lk, const float* mk,
                              const float* dk) {
    const long long n = g.plane * g.nzt;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q / g.plane);
        const long long r = q - (long long)k * g.plane;
        const int x = (int)(r % g.px), j = (int)(r / g.px);
        (void)j;
        const bool in = (x >= g.off) && (x < g.off + g.nxt);
        lam[q] = in ? lk[k] : 0.f;
        mu[q] = in ? mk[k] : 0.f;
        d[q] = in ? dk[k] : 0.f;
    }
}

// initial fault state (fd3d_theo.f90:59-88) on top of zeroed arrays
__global__ void k_model_reset(ModelDev M, int n2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q == 0) { *M.it_dev = 0; *M.status = 0; }
    if (q >= n2) return;
    M.q.ruptime[q] = 1.e4;
    M.q.sliptime[q] = 1.e4;
    M.q.tabsX[q] = M.law == 1 ? 1.f : 0.f;
    M.q.tabsZ[q] = M.law == 1 ? 1.f : 0.f;
    M.q.T0X[q] = M.q.T0Xb[q];
    if (M.law == 1) { M.q.psiX[q] = M.psiX0[q]; M.q.psiZ[q] = M.psiZ0[q]; }
}

// ---------------------------------------------------------------- host side
struct Block { size_t off, size; };

struct Arena {  // first-fit allocator over [0, cap)
    size_t cap = 0;
    std::vector<Block> free_;
    void init(size_t c) { cap = c; free_.assign(1, Block{0, c}); }
    bool alloc(size_t n, size_t* off) {
        n = (n + 255) & ~(size_t)255;
        for (size_t b = 0; b < free_.size(); ++b)
            if (free_[b].size >= n) {
                *off = free_[b].off;
                free_[b].off += n;
                free_[b].size -= n;
                if (free_[b].size == 0) free_.erase(free_.begin() + b);
                return true;
            }
        return false;
    }
    void release(size_t off, size_t n) {
        n = (n + 255) & ~(size_t)255;
        free_.push_back(Block{off, n});
        std::sort(free_.begin(), free_.end(), [](const Block& a, const Block& b) { return a.off < b.off; });
        std::vector<Block> m;
        for (const Block& b : free_) {
            if (!m.empty() && m.back().off + m.back().size == b.off) m.back().size += b.size;
            else m.push_back(b);
        }
        free_ = m;
    }
    size_t in_use() const {
        size_t f = 0;
        for (const Block& b : free_) f += b.size;
        return cap - f;
    }
};

struct Bump {  // carve aligned sub-arrays out of one model block
    char* base;
    size_t used = 0;
    template <class U> U* take(size_t n) {
        used = (used + 255) & ~(size_t)255;
        U* p = (U*)(base + used);
        used += n * sizeof(U);
        return p;
    }
};

// fault planes of a model: NF_PLANES single and NF2_PLANES two-plane float arrays, ND_PLANES
// single and ND2_PLANES two-plane double arrays (the two-plane state of Fault)
constexpr int NF_PLANES = 33, NF2_PLANES = 2, ND_PLANES = 10, ND2_PLANES = 1;

size_t model_bytes(const fd3d_params& p, const Grid& g, const PmlDesc& D, int prof_n, int nf, int cap) {
    const size_t n2 = (size_t)p.nxt * p.nzt;
    const size_t plane = (size_t)(p.nxt - 2 * p.nabc) * (p.nzt - p.nfs - p.nabc);
    size_t b = 0;
    auto add = [&](size_t bytes) { b = ((b + 255) & ~(size_t)255) + bytes; };
    add((size_t)g.n3 * 12 * 4);
    for (int k = 0; k < NF_PLANES; ++k) add(n2 * 4);
    for (int k = 0; k < NF2_PLANES; ++k) add(2 * n2 * 4);
    for (int k = 0; k < ND_PLANES; ++k) add(n2 * 8);
    for (int k = 0; k < ND2_PLANES; ++k) add(2 * n2 * 8);
    add(pml_aux_elems(D) * 4);
    add((size_t)prof_n * sizeof(Damp<float>));
    add((size_t)cap * nf * plane * 4);
    add((size_t)cap * std::max(1, p.nstations) * 3 * 4);
    add((size_t)LAY_N * p.nzt * 4);
    add(64);
    return b + 256;
}

struct Model {
    bool live = false;
    fd3d_params p{};
    ModelDev dev{};
    size_t off = 0, bytes = 0;
    int steps = 0;      // steps done
    int nf = 4;
    int cap = 0;
    // this model's work items per phase, for the interior tile depth items_kchunk
    std::vector<Work> items[NPHASE];
    int items_kchunk = -1;
};

enum { MODE_PERSISTENT = FD3D_BATCH_PERSISTENT, MODE_GRAPH = FD3D_BATCH_GRAPH };

struct Tuning {
    int kchunk = 16;
    int per_sm = 0;     // CTAs per SM (0 = occupancy limit), persistent schedule
    int mode = MODE_GRAPH;
};

}  // namespace

struct fd3d_batch {
    int dev = 0;
    cudaStream_t st = nullptr;
    cudaStream_t sst = nullptr;  // set-up of newly added models, concurrent with a run on st
    char* arena_base = nullptr;
    Arena arena;
    std::vector<Model> models;
    ModelDev* d_models = nullptr;
    ModelMaps* d_maps = nullptr;
    int* d_limit = nullptr;
    int* d_pbeg = nullptr;
    Work* d_work = nullptr;
    size_t work_cap = 0;
    BatchSync* d_sync = nullptr;
    int* d_status = nullptr;
    bool dirty = true;           // work list must be rebuilt
    std::vector<Work> work;
    int pbeg[NPHASE + 1] = {0};
    Tuning tun;
    int max_active = 0;          // CTAs per SM at the occupancy limit
    int nsm = 0;
    int built_kchunk = -1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    std::mutex mu;
    // graph schedule: items sorted by type, the run's step counter, branch streams,
    // and graphs of 32, 16, 8, 4, 2 and 1 steps captured for the current work list
    std::vector<Work> work_t;
    int tbeg[NTYPES + 1] = {0};
    Work* d_work_t = nullptr;
    size_t work_t_cap = 0;
    int* d_run_step = nullptr;
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t evf[3] = {nullptr, nullptr, nullptr};
    static constexpr int NGRAPH = 6;
    cudaGraphExec_t gx[NGRAPH] = {};
    int graph_kchunk = -1;
    int pdl = 0;                 // graph schedule: programmatic dependent launch between its kernels
                                 // (measured 2.3-2.5% slower: the early CTAs hold SM slots in the tail)
    int branches = 0;            // graph schedule: fault-band and PML sweeps on side streams (1) or in
                                 // series on the main stream (0, measured 9-11% faster: the branches interfered)
    int** d_stptr = nullptr;     // status words of the live models (k_or_status)
    int n_stptr = 0;
    int* d_status_or = nullptr;
    Work* h_stage = nullptr;     // page-locked staging of the work lists
    size_t stage_cap = 0;
    bool work_t_ok = false;      // the type-sorted list matches the work list
};

namespace {

// the work items of model m for interior tile depth kch, per phase
void build_model_items(Model& M, int m, int kch) {
    std::vector<Work>* per = M.items;
    for (int ph = 0; ph < NPHASE; ++ph) per[ph].clear();
    const fd3d_params& p = M.p;
    const Grid& g = M.dev.g;
    const int tm = m << 8;
    const int nxT = p.nxt - 2 * p.nabc, nyI = p.nyt - 2 - p.nabc, nzT = g.ks() - p.nabc;
    const int kc = std::max(1, std::min(kch, nzT));
    const int gx = (nxT + 31) / 32, gy = (nyI + 7) / 8, gz = (nzT + kc - 1) / kc;
    for (int z = 0; z < gz; ++z)
        for (int y = 0; y < gy; ++y)
            for (int x = 0; x < gx; ++x) {
                per[0].push_back(Work{tm | W_VEL_INT, x, y, z});
                per[2].push_back(Work{tm | W_STR_INT, x, y, z});
            }
    const int fx = (std::max(nxT, p.nxt) + 31) / 32, fz = (nzT + 7) / 8;
    for (int y = 0; y < fz; ++y)
        for (int x = 0; x < fx; ++x) per[0].push_back(Work{tm | W_VEL_FAULT, x, y, 0});
    const int npml = (int)((M.dev.D.cum[PML_MAXS] + PML_TILE - 1) / PML_TILE);
    for (int x = 0; x < npml; ++x) {
        per[0].push_back(Work{tm | W_VEL_PML, x, 0, 0});
        per[2].push_back(Work{tm | W_STR_PML, x, 0, 0});
    }
    const int sx = (p.nxt + 31) / 32, sy = p.fspace ? 0 : (p.nyt + 7) / 8;  // no fuvw/fres under FSPACE
    for (int y = 0; y < sy; ++y)
        for (int x = 0; x < sx; ++x) {
            per[1].push_back(Work{tm | W_VEL_FS, x, y, 0});
            per[3].push_back(Work{tm | W_STR_FS, x, y, 0});
        }
    const int px = (nxT + 31) / 32;
    for (int y = 0; y < fz; ++y)
        for (int x = 0; x < px; ++x) per[2].push_back(Work{tm | W_STR_FAULT, x, y, 0});
    {   // fused fault BC tiles (fault_bc_body)
        int nfres, tx, nt;
        fault_bc_grid(g, nfres, tx, nt);
        for (int t = 0; t < nt; ++t) per[3].push_back(Work{tm | W_FBC, t % tx, t / tx, 0});
    }
    if (M.p.law == FD3D_LAW_FVW && M.dev.fs.nucleation) {
        const int ni = (p.nxt - p.nabc) - (p.nabc - 1) + 1, nk = g.ks() - (p.nabc - 1) + 1;
        for (int y = 0; y < (nk + 7) / 8; ++y)
            for (int x = 0; x < (ni + 31) / 32; ++x) per[4].push_back(Work{tm | W_NUC, x, y, 0});
    }
    M.items_kchunk = kch;
}

// page-locked staging of n items (grown by half again when short)
int stage_items(fd3d_batch* b, size_t n) {
    if (n <= b->stage_cap) return FD3D_OK;
    if (b->h_stage) cudaFreeHost(b->h_stage);
    b->h_stage = nullptr;
    b->stage_cap = n + n / 2 + 1024;
    BCK(cudaHostAlloc((void**)&b->h_stage, b->stage_cap * sizeof(Work), cudaHostAllocDefault));
    return FD3D_OK;
}

// The items of the live models grouped by type, for the graph schedule (built when a
// graph run needs them after the work list changed)
int build_work_t(fd3d_batch* b) {
    std::vector<std::vector<Work>> byt(NTYPES);
    for (const Work& w : b->work) byt[w.tm & 255].push_back(w);
    b->work_t.clear();
    for (int t = 0; t < NTYPES; ++t) {
        b->tbeg[t] = (int)b->work_t.size();
        b->work_t.insert(b->work_t.end(), byt[t].begin(), byt[t].end());
    }
    b->tbeg[NTYPES] = (int)b->work_t.size();
    if (b->work_t.size() > b->work_t_cap) {
        if (b->d_work_t) cudaFree(b->d_work_t);
        b->work_t_cap = b->work_t.size() + b->work_t.size() / 2 + 64;
        BCK(cudaMalloc(&b->d_work_t, b->work_t_cap * sizeof(Work)));
    }
    if (!b->work_t.empty()) {
        if (stage_items(b, b->work_t.size())) return FD3D_ERR_CUDA;
        std::memcpy(b->h_stage, b->work_t.data(), b->work_t.size() * sizeof(Work));
        BCK(cudaMemcpyAsync(b->d_work_t, b->h_stage, b->work_t.size() * sizeof(Work), cudaMemcpyHostToDevice, b->st));
    }
    for (cudaGraphExec_t& g : b->gx)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    BCK(cudaStreamSynchronize(b->st));  // the staging buffer is reused by the next build
    b->work_t_ok = true;
    return FD3D_OK;
}

// The work list of the live models, phase by phase: each model's items are built once
// (and again when the tile depth changes), so a change of the resident set only
// concatenates them.
int build_work(fd3d_batch* b) {
    const int kch = b->tun.kchunk;
    size_t n = 0;
    for (size_t m = 0; m < b->models.size(); ++m) {
        Model& M = b->models[m];
        if (!M.live) continue;
        if (M.items_kchunk != kch) build_model_items(M, (int)m, kch);
        for (int ph = 0; ph < NPHASE; ++ph) n += M.items[ph].size();
    }
    b->work.resize(n);
    size_t at = 0;
    for (int ph = 0; ph < NPHASE; ++ph) {
        b->pbeg[ph] = (int)at;
        for (const Model& M : b->models)
            if (M.live && !M.items[ph].empty()) {
                std::memcpy(b->work.data() + at, M.items[ph].data(), M.items[ph].size() * sizeof(Work));
                at += M.items[ph].size();
            }
    }
    {   // status words of the live models
        std::vector<int*> sp;
        for (const Model& M : b->models)
            if (M.live) sp.push_back(M.dev.status);
        b->n_stptr = (int)sp.size();
        if (!sp.empty())
            BCK(cudaMemcpyAsync(b->d_stptr, sp.data(), sp.size() * sizeof(int*), cudaMemcpyHostToDevice, b->st));
    }
    b->work_t_ok = false;
    b->pbeg[NPHASE] = (int)b->work.size();
    if (b->work.size() > b->work_cap) {
        if (b->d_work) cudaFree(b->d_work);
        b->work_cap = b->work.size() + b->work.size() / 2 + 64;
        BCK(cudaMalloc(&b->d_work, b->work_cap * sizeof(Work)));
    }
    if (!b->work.empty()) {
        if (stage_items(b, b->work.size())) return FD3D_ERR_CUDA;
        std::memcpy(b->h_stage, b->work.data(), b->work.size() * sizeof(Work));
        BCK(cudaMemcpyAsync(b->d_work, b->h_stage, b->work.size() * sizeof(Work), cudaMemcpyHostToDevice, b->st));
    }
    BCK(cudaMemcpyAsync(b->d_pbeg, b->pbeg, sizeof(b->pbeg), cudaMemcpyHostToDevice, b->st));
    BCK(cudaStreamSynchronize(b->st));
    if (b->tun.mode == MODE_GRAPH) {
        int rc = build_work_t(b);
        if (rc) return rc;
    }
    b->dirty = false;
    b->built_kchunk = b->tun.kchunk;
    return FD3D_OK;
}

// one time step of the graph schedule on b->st (fork/join over the side streams)
int enqueue_graph_step(fd3d_batch* b) {
    const dim3 blk(32, 8);
    const int kc = b->tun.kchunk;
    const bool pdl = b->pdl && !b->branches;  // on the one stream only
    cudaError_t err = cudaSuccess;             // the first failed launch
    auto chk = [&](cudaError_t e) { if (err == cudaSuccess) err = e; };
    auto n_of = [&](int t) { return b->tbeg[t + 1] - b->tbeg[t]; };
    auto plane = [&](cudaStream_t s, int t0, int t1) {  // item types [t0, t1) in one launch
        const int n = b->tbeg[t1] - b->tbeg[t0];
        if (n == 0) return;
        const int* lim = b->d_limit;
        const int* rs = b->d_run_step;
        const ModelDev* md = b->d_models;
        const Work* wt = b->d_work_t;
        if (t0 <= W_FBC && W_FBC < t1) chk(launch_g(pdl, k_bplane<1>, n, blk, 0, s, md, wt, b->tbeg[t0], lim, rs));
        else if (t0 == W_VEL_FAULT) chk(launch_g(pdl, k_bplane<2>, n, blk, 0, s, md, wt, b->tbeg[t0], lim, rs));
        else chk(launch_g(pdl, k_bplane<0>, n, blk, 0, s, md, wt, b->tbeg[t0], lim, rs));
    };
    // the fault-band and PML sweeps on side streams beside the interior sweep, or (branches
    // off) all on the main stream one after another
    cudaStream_t s0 = b->branches ? b->side[0] : b->st, s1 = b->branches ? b->side[1] : b->st;
    for (int half = 0; half < 2; ++half) {
        const int ti = half ? W_STR_INT : W_VEL_INT, tf = half ? W_STR_FAULT : W_VEL_FAULT;
        const int tp = half ? W_STR_PML : W_VEL_PML, tfs = half ? W_STR_FS : W_VEL_FS;
        if (b->branches) {
            BCK(cudaEventRecord(b->evf[0], b->st));
            BCK(cudaStreamWaitEvent(b->side[0], b->evf[0], 0));
            BCK(cudaStreamWaitEvent(b->side[1], b->evf[0], 0));
        }
        const ModelDev* md = b->d_models;
        const ModelMaps* mp = b->d_maps;
        const Work* wt = b->d_work_t;
        const int* lim = b->d_limit;
        const int* rs = b->d_run_step;
        if (n_of(ti) > 0) {
            const size_t sm = tma_ring_bytes<float>();
            if (half) chk(launch_g(pdl, k_bint<true>, n_of(ti), blk, sm, b->st, md, mp, wt, b->tbeg[ti], lim, rs, kc, b->d_status));
            else chk(launch_g(pdl, k_bint<false>, n_of(ti), blk, sm, b->st, md, mp, wt, b->tbeg[ti], lim, rs, kc, b->d_status));
        }
        plane(s0, tf, tf + 1);
        if (n_of(tp) > 0) {
            if (half) chk(launch_g(pdl, k_bpml<true>, n_of(tp), blk, 0, s1, md, wt, b->tbeg[tp], lim, rs, b->d_status));
            else chk(launch_g(pdl, k_bpml<false>, n_of(tp), blk, 0, s1, md, wt, b->tbeg[tp], lim, rs, b->d_status));
        }
        if (b->branches) {
            BCK(cudaEventRecord(b->evf[1], b->side[0]));
            BCK(cudaEventRecord(b->evf[2], b->side[1]));
            BCK(cudaStreamWaitEvent(b->st, b->evf[1], 0));
            BCK(cudaStreamWaitEvent(b->st, b->evf[2], 0));
        }
        plane(b->st, tfs, half ? W_FBC + 1 : tfs + 1);  // after the stresses: fres and the fault BC tiles
    }
    plane(b->st, W_NUC, W_NUC + 1);
    chk(launch_g(pdl, k_step_end, 1, dim3(1), 0, b->st, b->d_run_step));
    BCK(err);
    BCK(cudaGetLastError());
    return FD3D_OK;
}

// graph g holds 32 >> g steps of the graph schedule (captured on first use)
int get_batch_graph(fd3d_batch* b, int g, cudaGraphExec_t* out) {
    if (b->graph_kchunk != b->tun.kchunk) {
        for (cudaGraphExec_t& x : b->gx)
            if (x) { cudaGraphExecDestroy(x); x = nullptr; }
        b->graph_kchunk = b->tun.kchunk;
    }
    if (!b->gx[g]) {
        cudaGraph_t gr;
        BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        int rc = FD3D_OK;
        for (int s = 0; s < (32 >> g) && rc == FD3D_OK; ++s) rc = enqueue_graph_step(b);
        cudaError_t e = cudaStreamEndCapture(b->st, &gr);
        if (rc) {
            if (e == cudaSuccess) cudaGraphDestroy(gr);
            return rc;
        }
        BCK(e);
        e = cudaGraphInstantiate(&b->gx[g], gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) { b->gx[g] = nullptr; return FD3D_ERR_CUDA; }
    }
    *out = b->gx[g];
    return FD3D_OK;
}

int launch_graphs(fd3d_batch* b, int nsteps) {
    if (!b->work_t_ok) {
        int rc = build_work_t(b);
        if (rc) return rc;
    }
    BCK(cudaMemsetAsync(b->d_run_step, 0, sizeof(int), b->st));
    int left = nsteps;
    for (int g = 0; g < fd3d_batch::NGRAPH && left > 0; ++g) {
        const int n = 32 >> g;
        if (left < n) continue;
        cudaGraphExec_t x;
        int rc = get_batch_graph(b, g, &x);
        if (rc) return rc;
        while (left >= n) {
            BCK(cudaGraphLaunch(x, b->st));
            left -= n;
        }
    }
    return FD3D_OK;
}

int launch_batch(fd3d_batch* b, int nsteps) {
    if (b->tun.mode == MODE_GRAPH) return launch_graphs(b, nsteps);
    const int per_sm = b->tun.per_sm > 0 ? std::min(b->tun.per_sm, b->max_active) : b->max_active;
    const int grid = std::max(1, per_sm * b->nsm);
    BCK(cudaMemsetAsync(b->d_sync, 0, sizeof(BatchSync), b->st));
    void* args[] = {&b->d_models, &b->d_maps, &b->d_work, &b->d_pbeg, &b->d_limit, &nsteps, &b->tun.kchunk, &b->d_sync,
                    &b->d_status};
    BCK(cudaLaunchCooperativeKernel((void*)k_batch, dim3(grid), dim3(32, 8), args, tma_ring_bytes<float>(), b->st));
    return FD3D_OK;
}

// host-side interp_fric + friction arrays of one model (fd3d_deriv.f90:3150-3190)
void fault_planes(const fd3d_params& p, const fd3d_fault& fl, std::vector<std::vector<float>>& F, std::vector<double>& pz,
                  std::vector<double>& px) {
    const int nxt = p.nxt, nzt = p.nzt;
    const size_t n2 = (size_t)nxt * nzt;
    auto cp = [&](const double* s, double dflt) {
        std::vector<float> v(n2);
        for (size_t k = 0; k < n2; ++k) v[k] = (float)(s ? s[k] : dflt);
        return v;
    };
    auto I2 = [&](int i, int k) { return (size_t)(i - 1) + (size_t)nxt * (k - 1); };
    std::vector<float> zero(n2, 0.f);
    F.assign(18, zero);  // T0X T0Z Dc peakX dynX DcX peakZ dynZ DcZ coh aX bX vwX fwX aZ bZ vwZ fwZ
    std::vector<float> sX = cp(fl.striniX, 0);
    F[1] = cp(fl.striniZ, 0);
    F[2] = cp(fl.Dc, 0);
    const bool fvw = p.law == FD3D_LAW_FVW;
    if (fvw) {
        F[10] = cp(fl.aX, 0); F[11] = cp(fl.bX, 0); F[12] = cp(fl.vwX, 0); F[13] = cp(fl.fwX, fl.fw);
        F[14] = cp(fl.a, 0); F[15] = cp(fl.b, 0); F[16] = cp(fl.vw, 0); F[17] = cp(fl.fwZ, fl.fw);
        pz.assign(fl.psi, fl.psi + n2);
        px.assign(fl.psiX, fl.psiX + n2);
    } else {
        F[6] = cp(fl.peak_xz, 0); F[7] = cp(fl.dyn_xz, 0); F[8] = F[2]; F[9] = cp(fl.coh, 0);
        pz.assign(n2, 0.0);
        px.assign(n2, 0.0);
    }
    for (int i = 2; i <= nxt - 1; ++i)
        for (int k = 2; k <= nzt - 1; ++k) {
            if (!fvw) {
                F[3][I2(i, k)] = (F[6][I2(i, k)] + F[6][I2(i - 1, k)] + F[6][I2(i, k - 1)] + F[6][I2(i - 1, k - 1)]) / 4.f;
                F[4][I2(i, k)] = (F[7][I2(i, k)] + F[7][I2(i - 1, k)] + F[7][I2(i, k - 1)] + F[7][I2(i - 1, k - 1)]) / 4.f;
                F[5][I2(i, k)] = (F[8][I2(i, k)] + F[8][I2(i - 1, k)] + F[8][I2(i, k - 1)] + F[8][I2(i - 1, k - 1)]) / 4.f;
            }
            F[0][I2(i, k)] = (sX[I2(i, k)] + sX[I2(i - 1, k)] + sX[I2(i, k - 1)] + sX[I2(i - 1, k - 1)]) / 4.f;
        }
}

int reset_model(fd3d_batch* b, Model& M, cudaStream_t st) {
    const size_t n2 = (size_t)M.p.nxt * M.p.nzt;
    ModelDev& d = M.dev;
    BCK(cudaMemsetAsync(d.f.u, 0, (size_t)d.g.n3 * 9 * sizeof(float), st));
    float* zt[] = {d.q.tx, d.q.tz, d.q.RFx, d.q.RFz, d.q.v1t, d.q.au1, d.q.av1,
                   d.q.aw1, d.q.uZ, d.q.wX, d.q.schangeX, d.q.schangeZ};
    for (float* a : zt) BCK(cudaMemsetAsync(a, 0, n2 * sizeof(float), st));
    BCK(cudaMemsetAsync(d.q.avdx, 0, 2 * n2 * sizeof(float), st));
    BCK(cudaMemsetAsync(d.q.avdz, 0, 2 * n2 * sizeof(float), st));
    double* zd[] = {d.q.distZ, d.q.slipX, d.q.slipZ, d.q.rise};
    for (double* a : zd) BCK(cudaMemsetAsync(a, 0, n2 * sizeof(double), st));
    BCK(cudaMemsetAsync(d.q.distX, 0, 2 * n2 * sizeof(double), st));
    BCK(cudaMemsetAsync(d.X.vel, 0, pml_aux_elems(d.D) * sizeof(float), st));
    k_model_reset<<<(unsigned)((n2 + 255) / 256), 256, 0, st>>>(d, (int)n2);
    BCK(cudaGetLastError());
    M.steps = 0;
    return FD3D_OK;
}

}  // namespace

extern "C" {

int fd3d_check_waits(int* mbar_status, int* barrier_status) {
    if (!mbar_status || !barrier_status) return FD3D_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return FD3D_ERR_NODEV; }
    int* st = nullptr;
    BatchSync* sync = nullptr;
    if (cudaMalloc(&st, 2 * sizeof(int)) != cudaSuccess) return FD3D_ERR_NOMEM;
    if (cudaMalloc(&sync, sizeof(BatchSync)) != cudaSuccess) { cudaFree(st); return FD3D_ERR_NOMEM; }
    int rc = FD3D_OK, h[2] = {0, 0};
    if (cudaMemset(st, 0, 2 * sizeof(int)) != cudaSuccess || cudaMemset(sync, 0, sizeof(BatchSync)) != cudaSuccess)
        rc = FD3D_ERR_CUDA;
    if (rc == FD3D_OK) {
        k_check_mbar_wait<<<1, 64>>>(st);
        k_check_grid_barrier<<<2, 64>>>(sync, st + 1);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(h, st, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = FD3D_ERR_CUDA;
    }
    cudaFree(st);
    cudaFree(sync);
    *mbar_status = h[0];
    *barrier_status = h[1];
    return rc;
}

int fd3d_batch_create(size_t arena_bytes, int max_models, fd3d_batch** out) {
    if (!out || max_models < 1 || arena_bytes < (1u << 20)) return FD3D_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return FD3D_ERR_NODEV; }
    fd3d_batch* b = new fd3d_batch();
    cudaGetDevice(&b->dev);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->dev);
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev);
    if (!coop) { delete b; return FD3D_ERR_NODEV; }
    auto fail = [&](int rc) { fd3d_batch_destroy(b); return rc; };
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->sst, cudaStreamNonBlocking) != cudaSuccess)
        return fail(FD3D_ERR_CUDA);
    if (cudaMalloc(&b->arena_base, arena_bytes) != cudaSuccess) { cudaGetLastError(); return fail(FD3D_ERR_NOMEM); }
    b->arena.init(arena_bytes);
    b->models.resize(max_models);
    if (cudaMalloc(&b->d_models, sizeof(ModelDev) * max_models) != cudaSuccess ||
        cudaMalloc(&b->d_maps, sizeof(ModelMaps) * max_models) != cudaSuccess ||
        cudaMalloc(&b->d_limit, sizeof(int) * max_models) != cudaSuccess ||
        cudaMalloc(&b->d_pbeg, sizeof(int) * (NPHASE + 1)) != cudaSuccess ||
        cudaMalloc(&b->d_sync, sizeof(BatchSync)) != cudaSuccess || cudaMalloc(&b->d_status, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_run_step, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_stptr, sizeof(int*) * max_models) != cudaSuccess ||
        cudaMalloc(&b->d_status_or, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return fail(FD3D_ERR_NOMEM);
    }
    for (cudaStream_t& s : b->side)
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return fail(FD3D_ERR_CUDA);
    for (cudaEvent_t& e : b->evf)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(FD3D_ERR_CUDA);
    if (cudaFuncSetAttribute(k_bint<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_ring_bytes<float>()) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_bint<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_ring_bytes<float>()) !=
            cudaSuccess) {
        cudaGetLastError();
        return fail(FD3D_ERR_CUDA);
    }
    cudaMemset(b->d_status, 0, sizeof(int));
    cudaEventCreate(&b->ev0);
    cudaEventCreate(&b->ev1);
    if (cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_ring_bytes<float>()) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->max_active, k_batch, 256, tma_ring_bytes<float>()) != cudaSuccess ||
        b->max_active < 1 || !tensor_map_encoder()) {
        cudaGetLastError();
        return fail(FD3D_ERR_CUDA);
    }
    if (const char* e = std::getenv("FD3D_BATCH_KCHUNK")) b->tun.kchunk = std::max(1, std::atoi(e));
    if (const char* e = std::getenv("FD3D_BATCH_PER_SM")) b->tun.per_sm = std::max(0, std::atoi(e));
    // FD3D_BATCH_BRANCHES=1: the graph schedule runs the fault-band and PML sweeps on side streams
    if (const char* e = std::getenv("FD3D_BATCH_BRANCHES")) b->branches = std::atoi(e) != 0;
    // FD3D_BATCH_PDL=1: the graph schedule's kernels with programmatic dependent launch
    if (const char* e = std::getenv("FD3D_BATCH_PDL")) b->pdl = std::atoi(e) != 0;
    // FD3D_BATCH_MODE=persistent|graph
    if (const char* e = std::getenv("FD3D_BATCH_MODE"))
        b->tun.mode = std::strcmp(e, "persistent") == 0 ? MODE_PERSISTENT : MODE_GRAPH;
    *out = b;
    return FD3D_OK;
}

int fd3d_batch_destroy(fd3d_batch* b) {
    if (!b) return FD3D_ERR_ARG;
    if (b->st) cudaStreamSynchronize(b->st);
    if (b->sst) cudaStreamSynchronize(b->sst);
    cudaFree(b->arena_base);
    cudaFree(b->d_models);
    cudaFree(b->d_maps);
    cudaFree(b->d_limit);
    cudaFree(b->d_pbeg);
    cudaFree(b->d_sync);
    cudaFree(b->d_status);
    cudaFree(b->d_work);
    cudaFree(b->d_work_t);
    if (b->h_stage) cudaFreeHost(b->h_stage);
    cudaFree(b->d_run_step);
    cudaFree(b->d_stptr);
    cudaFree(b->d_status_or);
    for (cudaGraphExec_t g : b->gx)
        if (g) cudaGraphExecDestroy(g);
    for (cudaStream_t s : b->side)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->evf)
        if (e) cudaEventDestroy(e);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    if (b->sst) cudaStreamDestroy(b->sst);
    delete b;
    return FD3D_OK;
}

int fd3d_batch_bytes_needed(const fd3d_params* p, size_t* bytes) {
    if (!p || !bytes) return FD3D_ERR_ARG;
    int rc = validate_params(p);
    if (rc) return rc;
    Grid g = make_grid(*p);
    PmlDesc D;
    std::vector<Damp<float>> prof;
    make_pml<float>(*p, D, prof);
    const int nf = p->law == FD3D_LAW_FVW ? 5 : 4;
    const int cap = p->history_capacity > 0 ? p->history_capacity : 16;
    *bytes = model_bytes(*p, g, D, (int)prof.size(), nf, cap);
    return FD3D_OK;
}

int fd3d_batch_add(fd3d_batch* b, const fd3d_params* pin, const double* lam_k, const double* mu_k, const double* d_k,
                   const fd3d_fault* fl, int* slot) {
    if (!b || !pin || !lam_k || !mu_k || !d_k || !fl || !slot) return FD3D_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    int rc = validate_params(pin);
    if (rc) return rc;
    if (pin->precision != FD3D_PREC_F32) return FD3D_ERR_ARG;  // the batch runs the FP32 build
    if (!fl->striniX || !fl->Dc) return FD3D_ERR_ARG;
    if (pin->law == FD3D_LAW_SW && (!fl->peak_xz || !fl->dyn_xz)) return FD3D_ERR_ARG;
    if (pin->law == FD3D_LAW_FVW && (!fl->a || !fl->b || !fl->psi || !fl->vw || !fl->aX || !fl->bX || !fl->psiX || !fl->vwX))
        return FD3D_ERR_ARG;
    int m = -1;
    for (size_t q = 0; q < b->models.size(); ++q)
        if (!b->models[q].live) { m = (int)q; break; }
    if (m < 0) return FD3D_ERR_BUSY;
    Model M;
    M.p = *pin;
    M.p.history_stride = std::max(1, M.p.history_stride);
    M.nf = M.p.law == FD3D_LAW_FVW ? 5 : 4;
    M.cap = M.p.history_capacity > 0 ? M.p.history_capacity : 16;
    ModelDev& d = M.dev;
    d.g = make_grid(M.p);
    d.c = make_const<float>(M.p);
    d.law = M.p.law;
    std::vector<Damp<float>> prof;
    make_pml<float>(M.p, d.D, prof);
    if (!pml_modes_hold(d.D, prof)) return FD3D_ERR_ARG;
    M.bytes = model_bytes(M.p, d.g, d.D, (int)prof.size(), M.nf, M.cap);
    if (!b->arena.alloc(M.bytes, &M.off)) return FD3D_ERR_NOMEM;
    Bump bp{b->arena_base + M.off};
    const fd3d_params& p = M.p;
    const size_t n2 = (size_t)p.nxt * p.nzt;
    float* fp = bp.take<float>((size_t)d.g.n3 * 12);
    float** outs[9] = {&d.f.u, &d.f.v, &d.f.w, &d.f.xx, &d.f.yy, &d.f.zz, &d.f.xy, &d.f.yz, &d.f.xz};
    for (int a = 0; a < 9; ++a) *outs[a] = fp + (size_t)a * d.g.n3;
    float* lam = fp + 9 * (size_t)d.g.n3;
    float* mu = fp + 10 * (size_t)d.g.n3;
    float* dd = fp + 11 * (size_t)d.g.n3;
    d.f.lam = lam; d.f.mu = mu; d.f.d = dd;  // d.f.lay: the layer table, set below
    float** fq[NF_PLANES] = {&d.q.tx, &d.q.tz, &d.q.RFx, &d.q.RFz, &d.q.v1t,
                             &d.q.au1, &d.q.av1, &d.q.aw1, &d.q.uZ, &d.q.wX, &d.q.tabsX, &d.q.tabsZ, &d.q.T0X,
                             &d.q.T0Z, &d.q.T0Xb, &d.q.Dc, &d.q.peakX, &d.q.dynX, &d.q.DcX, &d.q.peakZ, &d.q.dynZ,
                             &d.q.DcZ, &d.q.coh, &d.q.aX, &d.q.bX, &d.q.vwX, &d.q.fwX, &d.q.aZ, &d.q.bZ, &d.q.vwZ,
                             &d.q.fwZ, &d.q.schangeX, &d.q.schangeZ};
    for (float** a : fq) *a = bp.take<float>(n2);
    float** fq2[NF2_PLANES] = {&d.q.avdx, &d.q.avdz};
    for (float** a : fq2) *a = bp.take<float>(2 * n2);
    d.q.txt = d.q.tzt = nullptr;  // the fused fault BC keeps the trial tractions in shared memory
    double** dq[ND_PLANES] = {&d.q.psiX, &d.q.psiZ, &d.q.distZ, &d.q.slipX, &d.q.slipZ, &d.q.ruptime,
                              &d.q.rise, &d.q.sliptime, &d.psiX0, &d.psiZ0};
    for (double** a : dq) *a = bp.take<double>(n2);
    d.q.distX = bp.take<double>(2 * n2);
    d.q.n2 = (int)n2;
    float* aux = bp.take<float>(pml_aux_elems(d.D));
    pml_aux_bind(d.X, aux, d.D);
    Damp<float>* dprof = bp.take<Damp<float>>(prof.size());
    d.X.prof = dprof;
    const size_t plane = (size_t)(p.nxt - 2 * p.nabc) * (p.nzt - p.nfs - p.nabc);
    float* ring = bp.take<float>((size_t)M.cap * M.nf * plane);
    float* seis = bp.take<float>((size_t)M.cap * std::max(1, p.nstations) * 3);
    float* layers = bp.take<float>((size_t)LAY_N * p.nzt);
    d.f.lay = layers;  // batch models always carry a 1-D medium
    d.it_dev = bp.take<int>(1);
    d.status = bp.take<int>(1);
    d.h.ring = ring; d.h.cap = M.cap; d.h.stride = p.history_stride; d.h.nf = M.nf; d.h.nst = p.nstations;
    for (int s = 0; s < p.nstations; ++s) { d.h.sta[3 * s] = p.staX[s]; d.h.sta[3 * s + 1] = p.staY[s]; d.h.sta[3 * s + 2] = p.staZ[s]; }
    d.h.seis = seis;
    if (p.law == FD3D_LAW_FVW) {
        d.fs.Sn = fl->Sn; d.fs.v0 = fl->v0; d.fs.f0 = fl->f0; d.fs.fw = fl->fw; d.fs.uini = fl->uini; d.fs.wini = fl->wini;
        d.fs.nucleation = fl->nucleation;
        d.fs.hx0 = fl->hx0; d.fs.hz0 = fl->hz0; d.fs.perturb = fl->perturb; d.fs.RR2 = fl->RR2; d.fs.TT2 = fl->TT2;
        d.fs.strinixI = fl->strinixI;
    }
    // whole block to zero, then medium, fault planes and profiles
    BCK(cudaMemsetAsync(b->arena_base + M.off, 0, bp.used, b->sst));
    std::vector<float> lay(LAY_N * (size_t)p.nzt);
    for (int k = 0; k < p.nzt; ++k) {
        lay[k] = (float)lam_k[k]; lay[p.nzt + k] = (float)mu_k[k]; lay[2 * p.nzt + k] = (float)d_k[k];
        lay[3 * p.nzt + k] = d.c.dth / lay[2 * p.nzt + k];  // the IEEE quotients the sweeps would form
        lay[4 * p.nzt + k] = d.c.dt / lay[2 * p.nzt + k];
    }
    BCK(cudaMemcpyAsync(layers, lay.data(), lay.size() * sizeof(float), cudaMemcpyHostToDevice, b->sst));
    k_fill_layers<<<1024, 256, 0, b->sst>>>(d.g, lam, mu, dd, layers, layers + p.nzt, layers + 2 * p.nzt);
    BCK(cudaGetLastError());
    std::vector<std::vector<float>> F;
    std::vector<double> pz, px;
    fault_planes(p, *fl, F, pz, px);
    float* dst[18] = {d.q.T0X, d.q.T0Z, d.q.Dc, d.q.peakX, d.q.dynX, d.q.DcX, d.q.peakZ, d.q.dynZ, d.q.DcZ, d.q.coh,
                      d.q.aX, d.q.bX, d.q.vwX, d.q.fwX, d.q.aZ, d.q.bZ, d.q.vwZ, d.q.fwZ};
    for (int a = 0; a < 18; ++a) BCK(cudaMemcpyAsync(dst[a], F[a].data(), n2 * sizeof(float), cudaMemcpyHostToDevice, b->sst));
    BCK(cudaMemcpyAsync(d.q.T0Xb, F[0].data(), n2 * sizeof(float), cudaMemcpyHostToDevice, b->sst));
    BCK(cudaMemcpyAsync(d.psiZ0, pz.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, b->sst));
    BCK(cudaMemcpyAsync(d.psiX0, px.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, b->sst));
    BCK(cudaMemcpyAsync(dprof, prof.data(), prof.size() * sizeof(Damp<float>), cudaMemcpyHostToDevice, b->sst));
    M.live = true;
    rc = reset_model(b, M, b->sst);
    if (rc) { b->arena.release(M.off, M.bytes); return rc; }
    ModelMaps mm;
    if (!make_interior_maps<float>(d.g, d.f, mm.v, mm.s)) { b->arena.release(M.off, M.bytes); return FD3D_ERR_CUDA; }
    BCK(cudaMemcpyAsync(b->d_maps + m, &mm, sizeof(ModelMaps), cudaMemcpyHostToDevice, b->sst));
    BCK(cudaMemcpyAsync(b->d_models + m, &M.dev, sizeof(ModelDev), cudaMemcpyHostToDevice, b->sst));
    BCK(cudaStreamSynchronize(b->sst));
    b->models[m] = M;
    b->dirty = true;
    *slot = m;
    return FD3D_OK;
}

int fd3d_batch_remove(fd3d_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->models.size()) return FD3D_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    Model& M = b->models[slot];
    if (!M.live) return FD3D_ERR_ARG;
    BCK(cudaStreamSynchronize(b->st));
    b->arena.release(M.off, M.bytes);
    M.live = false;
    b->dirty = true;
    return FD3D_OK;
}

int fd3d_batch_reset(fd3d_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->models.size() || !b->models[slot].live) return FD3D_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    int rc = reset_model(b, b->models[slot], b->st);
    if (rc) return rc;
    BCK(cudaStreamSynchronize(b->st));
    return FD3D_OK;
}

int fd3d_batch_run(fd3d_batch* b, int nsteps) {
    fd3d::TraceRange trace_("fd3d_batch_run");
    if (!b || nsteps < 0) return FD3D_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    if (b->dirty || b->built_kchunk != b->tun.kchunk) {
        int rc = build_work(b);
        if (rc) return rc;
    }
    std::vector<int> limit(b->models.size(), 0);
    int smax = 0;
    for (size_t m = 0; m < b->models.size(); ++m) {
        const Model& M = b->models[m];
        if (!M.live) continue;
        limit[m] = std::max(0, std::min(nsteps, M.p.ntfd - M.steps));
        smax = std::max(smax, limit[m]);
    }
    BCK(cudaEventRecord(b->ev0, b->st));
    if (smax > 0 && !b->work.empty()) {
        BCK(cudaMemcpyAsync(b->d_limit, limit.data(), limit.size() * sizeof(int), cudaMemcpyHostToDevice, b->st));
        int rc = launch_batch(b, smax);
        if (rc) return rc;
    }
    BCK(cudaEventRecord(b->ev1, b->st));
    for (size_t m = 0; m < b->models.size(); ++m)
        if (b->models[m].live) b->models[m].steps += limit[m];
    return FD3D_OK;
}

int fd3d_batch_sync(fd3d_batch* b) {
    if (!b) return FD3D_ERR_ARG;
    BCK(cudaStreamSynchronize(b->st));
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    if (b->dirty) {  // the status list follows the live models
        int rc = build_work(b);
        if (rc) return rc;
    }
    int st[2] = {0, 0};
    BCK(cudaMemcpy(&st[0], b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (b->n_stptr > 0) {
        k_or_status<<<1, 256, 0, b->st>>>(b->d_stptr, b->n_stptr, b->d_status_or);
        BCK(cudaGetLastError());
        BCK(cudaMemcpyAsync(&st[1], b->d_status_or, sizeof(int), cudaMemcpyDeviceToHost, b->st));
        BCK(cudaStreamSynchronize(b->st));
    }
    const int any = st[0] | st[1];
    if (any & ST_TIMEOUT) return FD3D_ERR_TIMEOUT;
    if (any & ST_NONFINITE) return FD3D_ERR_NONFINITE;
    if (any & ST_NEWTON) return FD3D_ERR_NEWTON;
    return FD3D_OK;
}

int fd3d_batch_model_status(fd3d_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->models.size() || !b->models[slot].live) return FD3D_ERR_ARG;
    int s = 0;
    BCK(cudaMemcpy(&s, b->models[slot].dev.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (s & ST_NONFINITE) return FD3D_ERR_NONFINITE;
    if (s & ST_NEWTON) return FD3D_ERR_NEWTON;
    return FD3D_OK;
}

int fd3d_batch_last_run_ms(fd3d_batch* b, float* ms) {
    if (!b || !ms) return FD3D_ERR_ARG;
    *ms = b->last_ms;
    return FD3D_OK;
}

int fd3d_batch_steps_done(fd3d_batch* b, int slot, int* it) {
    if (!b || !it || slot < 0 || slot >= (int)b->models.size() || !b->models[slot].live) return FD3D_ERR_ARG;
    *it = b->models[slot].steps;
    return FD3D_OK;
}

int fd3d_batch_live(fd3d_batch* b, int* nlive, size_t* bytes_in_use) {
    if (!b) return FD3D_ERR_ARG;
    int n = 0;
    for (const Model& M : b->models) n += M.live ? 1 : 0;
    if (nlive) *nlive = n;
    if (bytes_in_use) *bytes_in_use = b->arena.in_use();
    return FD3D_OK;
}

int fd3d_batch_fetch_plane(fd3d_batch* b, int slot, int plane, double* host) {
    if (!b || !host || slot < 0 || slot >= (int)b->models.size() || !b->models[slot].live) return FD3D_ERR_ARG;
    const Model& M = b->models[slot];
    const size_t n2 = (size_t)M.p.nxt * M.p.nzt;
    const ModelDev& d = M.dev;
    const float* ts = nullptr;
    const double* ds = nullptr;
    switch (plane) {
        case FD3D_PLANE_TX: ts = d.q.tx; break;             case FD3D_PLANE_TZ: ts = d.q.tz; break;
        case FD3D_PLANE_SLIPX: ds = d.q.slipX; break;       case FD3D_PLANE_SLIPZ: ds = d.q.slipZ; break;
        case FD3D_PLANE_RUPTIME: ds = d.q.ruptime; break;   case FD3D_PLANE_RISE: ds = d.q.rise; break;
        case FD3D_PLANE_SLIPTIME: ds = d.q.sliptime; break;
        case FD3D_PLANE_DISTX: ds = pp_wr(d.q.distX, M.steps, (int)n2); break;  // the plane of the last step
        case FD3D_PLANE_DISTZ: ds = d.q.distZ; break;       case FD3D_PLANE_PSIX: ds = d.q.psiX; break;
        case FD3D_PLANE_PSIZ: ds = d.q.psiZ; break;         case FD3D_PLANE_T0X: ts = d.q.T0X; break;
        case FD3D_PLANE_T0Z: ts = d.q.T0Z; break;           case FD3D_PLANE_SCHANGEX: ts = d.q.schangeX; break;
        case FD3D_PLANE_SCHANGEZ: ts = d.q.schangeZ; break;
        default: return FD3D_ERR_ARG;
    }
    BCK(cudaStreamSynchronize(b->st));
    if (ds) {
        BCK(cudaMemcpy(host, ds, n2 * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> v(n2);
        BCK(cudaMemcpy(v.data(), ts, n2 * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < n2; ++k) host[k] = v[k];
    }
    return FD3D_OK;
}

int fd3d_batch_fetch_final(fd3d_batch* b, int slot, double* slipX, double* slipZ, double* ruptime, double* rise,
                           double* sliptime) {
    if (!b || slot < 0 || slot >= (int)b->models.size() || !b->models[slot].live) return FD3D_ERR_ARG;
    const Model& M = b->models[slot];
    const size_t n2 = (size_t)M.p.nxt * M.p.nzt;
    int rc = 0;
    if (slipX) rc |= fd3d_batch_fetch_plane(b, slot, FD3D_PLANE_SLIPX, slipX);
    if (slipZ) rc |= fd3d_batch_fetch_plane(b, slot, FD3D_PLANE_SLIPZ, slipZ);
    std::vector<double> rt(n2);
    rc |= fd3d_batch_fetch_plane(b, slot, FD3D_PLANE_RUPTIME, rt.data());
    if (ruptime) std::memcpy(ruptime, rt.data(), n2 * sizeof(double));
    if (rise) {
        rc |= fd3d_batch_fetch_plane(b, slot, FD3D_PLANE_RISE, rise);
        for (size_t k = 0; k < n2; ++k) rise[k] -= rt[k];
    }
    if (sliptime) rc |= fd3d_batch_fetch_plane(b, slot, FD3D_PLANE_SLIPTIME, sliptime);
    return rc ? FD3D_ERR_CUDA : FD3D_OK;
}

int fd3d_batch_fetch_history(fd3d_batch* b, int slot, int field, int rec0, int nrec, double* host) {
    if (!b || !host || slot < 0 || slot >= (int)b->models.size() || !b->models[slot].live) return FD3D_ERR_ARG;
    const Model& M = b->models[slot];
    if (field < 0 || field >= M.nf || rec0 < 0 || nrec < 0) return FD3D_ERR_ARG;
    const int have = M.steps / M.p.history_stride;
    if (rec0 + nrec > have || rec0 < have - M.cap) return FD3D_ERR_ARG;
    const size_t plane = (size_t)(M.p.nxt - 2 * M.p.nabc) * (M.p.nzt - M.p.nfs - M.p.nabc);
    std::vector<float> buf(plane);
    BCK(cudaStreamSynchronize(b->st));
    for (int r = 0; r < nrec; ++r) {
        const size_t s = (size_t)((rec0 + r) % M.cap);
        BCK(cudaMemcpy(buf.data(), (const float*)M.dev.h.ring + (s * M.nf + field) * plane, plane * sizeof(float),
                       cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < plane; ++k) host[(size_t)r * plane + k] = buf[k];
    }
    return FD3D_OK;
}

int fd3d_batch_set_tuning(fd3d_batch* b, int kchunk, int ctas_per_sm) {
    if (!b || kchunk < 1 || ctas_per_sm < 0) return FD3D_ERR_ARG;
    b->tun.kchunk = kchunk;
    b->tun.per_sm = ctas_per_sm;
    return FD3D_OK;
}

int fd3d_batch_set_schedule(fd3d_batch* b, int mode) {
    if (!b || (mode != FD3D_BATCH_PERSISTENT && mode != FD3D_BATCH_GRAPH)) return FD3D_ERR_ARG;
    std::lock_guard<std::mutex> lk(b->mu);
    b->tun.mode = mode;
    return FD3D_OK;
}

int fd3d_batch_get_schedule(fd3d_batch* b, int* mode) {
    if (!b || !mode) return FD3D_ERR_ARG;
    *mode = b->tun.mode;
    return FD3D_OK;
}

int fd3d_batch_get_tuning(fd3d_batch* b, int* kchunk, int* ctas_per_sm, int* max_ctas_per_sm) {
    if (!b) return FD3D_ERR_ARG;
    if (kchunk) *kchunk = b->tun.kchunk;
    if (ctas_per_sm) *ctas_per_sm = b->tun.per_sm > 0 ? b->tun.per_sm : b->max_active;
    if (max_ctas_per_sm) *max_ctas_per_sm = b->max_active;
    return FD3D_OK;
}

// Times each (kchunk, CTAs/SM) candidate for `steps` steps on the live models (all
// of which must be at step 0), keeps the fastest, resets every model to step 0, and
// records the choice under `key` in the JSON-lines cache file (if given).  A cache
// hit skips the timing.
int fd3d_batch_autotune(fd3d_batch* b, int steps, const char* cache_path, const char* key) {
    fd3d::TraceRange trace_("fd3d_batch_autotune");
    if (!b || steps < 1) return FD3D_ERR_ARG;
    for (const Model& M : b->models)
        if (M.live && M.steps != 0) return FD3D_ERR_STATE;
    std::string k = key ? key : "";
    if (!k.empty()) {  // a tuning holds for one kind of device only
        int dev = 0;
        cudaDeviceProp prop{};
        BCK(cudaGetDevice(&dev));
        BCK(cudaGetDeviceProperties(&prop, dev));
        for (char& ch : prop.name) if (ch == '"') ch = '\'';
        k += std::string("|") + prop.name + "|sm" + std::to_string(prop.multiProcessorCount);
    }
    if (cache_path && !k.empty()) {
        std::ifstream in(cache_path);
        std::string line;
        while (std::getline(in, line)) {
            int kc = 0, ps = 0, mode = -1;
            char buf[256] = {0};
            if (std::sscanf(line.c_str(), "{\"key\": \"%255[^\"]\", \"schedule\": %d, \"kchunk\": %d, \"ctas_per_sm\": %d",
                            buf, &mode, &kc, &ps) == 4 &&
                k == buf && kc > 0 && (mode == MODE_GRAPH || mode == MODE_PERSISTENT)) {
                b->tun.mode = mode;
                b->tun.kchunk = kc;
                b->tun.per_sm = ps;
                return FD3D_OK;
            }
        }
    }
    // candidates: the graph schedule per interior tile depth, the persistent kernel per
    // tile depth and CTAs per SM
    const int kcs[] = {4, 8, 16, 32};
    std::vector<Tuning> cand;
    for (int kc : kcs) {
        Tuning t;
        t.mode = MODE_GRAPH;
        t.kchunk = kc;
        cand.push_back(t);
    }
    std::vector<int> pss;
    for (int ps = 1; ps <= b->max_active; ps *= 2) pss.push_back(ps);
    if (pss.back() != b->max_active) pss.push_back(b->max_active);
    for (int kc : kcs)
        for (int ps : pss) {
            Tuning t;
            t.mode = MODE_PERSISTENT;
            t.kchunk = kc;
            t.per_sm = ps;
            cand.push_back(t);
        }
    float best = 1e30f;
    Tuning bt = b->tun;
    for (const Tuning& t : cand) {
        b->tun = t;
        int rc = fd3d_batch_run(b, steps);
        if (rc) return rc;
        rc = fd3d_batch_sync(b);
        if (rc) return rc;
        if (b->last_ms < best) { best = b->last_ms; bt = b->tun; }
        for (size_t m = 0; m < b->models.size(); ++m)
            if (b->models[m].live) { rc = reset_model(b, b->models[m], b->st); if (rc) return rc; }
        BCK(cudaStreamSynchronize(b->st));
    }
    b->tun = bt;
    if (cache_path && !k.empty()) {
        std::ofstream out(cache_path, std::ios::app);
        out << "{\"key\": \"" << k << "\", \"schedule\": " << bt.mode << ", \"kchunk\": " << bt.kchunk
            << ", \"ctas_per_sm\": " << bt.per_sm << ", \"ms\": " << best << ", \"steps\": " << steps << "}\n";
    }
    return FD3D_OK;
}

}  // extern "C"
