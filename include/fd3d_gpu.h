/*
 * fd3d_gpu.h -- C ABI of the B200 (sm_100a) time-stepping path of FD3D_TSN.
 *
 * The reference exposes its hot path as the argument-less Fortran subroutine
 * fd3d() (src/fd3d_theo.f90:22), which reads every input from module globals
 * (src/fd3d_init.f90:15-121), runs the time loop (src/fd3d_theo.f90:187-602)
 * and writes the result files under result/.  This header replaces that seam
 * with an explicit context:
 *
 *     fd3d_ctx_create      <- fd3d_init() sizes + init_pml()      (fd3d_init.f90:126-208, fd3d_deriv.f90:1319-1493)
 *     fd3d_upload_medium   <- readcrustalmodel() output lam1,mu1,d1 (fd3d_init.f90:211-279)
 *     fd3d_upload_fault    <- forwardspecialTPV5/TPV104 or inversion_modeltofd3d output + interp_fric (fd3d_deriv.f90:3150-3190)
 *     fd3d_run / fd3d_sync <- the time loop body                   (fd3d_theo.f90:187-602)
 *     fd3d_fetch_history   <- the per-step WRITE(24..28) planes      (fd3d_theo.f90:546-553)
 *     fd3d_fetch_stations  <- the per-step station lines            (fd3d_theo.f90:456-467,555-557)
 *     fd3d_fetch_final     <- ruptime,rise,slipX/Z,sliptime after the loop (fd3d_theo.f90:604-658)
 *     fd3d_write_results   <- the files under result/ (.res)                (fd3d_theo.f90:133-145,546-558,687-749)
 *
 * Conventions
 *  - Every function returns an int status: FD3D_OK (0) or a negative FD3D_ERR_*.
 *    No function calls exit(); the reference's `stop` on CFL (fd3d_init.f90:274-278)
 *    becomes FD3D_ERR_CFL, its printed 'newton error?' (fd3d_deriv.f90:1157-1160)
 *    becomes FD3D_ERR_NEWTON from fd3d_sync().
 *  - Arrays cross the boundary in the reference's own layout: Fortran column-major,
 *    x (i) fastest, 1-based index (i,j,k) at offset (i-1) + nxt*((j-1) + nyt*(k-1));
 *    fault-plane arrays (i,k) at (i-1) + nxt*(k-1).  Host arrays are borrowed for
 *    the duration of the call only.
 *  - real_kind selects the host element type of a buffer: 4 (float) or 8 (double),
 *    as the reference's `real` is 4 bytes by default and 8 bytes with -r8.
 *  - One context is driven by one host thread at a time.  Device memory is owned by
 *    the context.  Work is enqueued on the context's own CUDA streams (a main stream,
 *    and a side stream that each step forks from it and joins back into it).
 */
#ifndef FD3D_GPU_H
#define FD3D_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define FD3D_OK              0
#define FD3D_ERR_ARG        -1   /* bad argument or size                          */
#define FD3D_ERR_CFL        -2   /* vp_max*dt/dh > 0.25 (fd3d_init.f90:274-278)    */
#define FD3D_ERR_CUDA       -3   /* a CUDA runtime call failed                    */
#define FD3D_ERR_NOMEM      -4   /* request exceeds device memory / HBM budget    */
#define FD3D_ERR_NEWTON     -5   /* FVW Newton solve hit its iteration cap        */
#define FD3D_ERR_NONFINITE  -6   /* NaN/Inf found on the fault plane              */
#define FD3D_ERR_STATE      -7   /* call out of order (e.g. run before upload)    */
#define FD3D_ERR_IO         -8   /* input or result file could not be read/written */
#define FD3D_ERR_NODEV      -9   /* no CUDA device / library built without one    */
#define FD3D_ERR_BUSY      -10   /* batch/serving object has no free slot         */
#define FD3D_ERR_TIMEOUT   -11   /* a bounded device-side wait gave up            */

/* ---- friction law (compile-time -DFVW switch of the reference) -------- */
#define FD3D_LAW_SW   0   /* linear slip weakening (reference default)   */
#define FD3D_LAW_FVW  1   /* fast-velocity-weakening rate and state      */

/* ---- arithmetic of the wave field ------------------------------------ */
#define FD3D_PREC_F32 0   /* FP32 fields and PML; FP64 slip, slip path, rupture time, psi, Newton */
#define FD3D_PREC_F64 1   /* everything FP64: the reference built with -r8 */

/* ---- history planes (unformatted stream files of the reference) ------ */
#define FD3D_HIST_SLIPRATE_X    0   /* result/sliprateX.res    */
#define FD3D_HIST_SLIPRATE_Z    1   /* result/sliprateZ.res    */
#define FD3D_HIST_SHEARSTRESS_X 2   /* result/shearstressX.res */
#define FD3D_HIST_SHEARSTRESS_Z 3   /* result/shearstressZ.res */
#define FD3D_HIST_PSI           4   /* result/psi.res (FVW)    */
#define FD3D_HIST_NFIELDS       5

/* ---- wave-field / state selectors for fd3d_fetch_field ---------------- */
#define FD3D_FIELD_U   0
#define FD3D_FIELD_V   1
#define FD3D_FIELD_W   2
#define FD3D_FIELD_XX  3
#define FD3D_FIELD_YY  4
#define FD3D_FIELD_ZZ  5
#define FD3D_FIELD_XY  6
#define FD3D_FIELD_YZ  7
#define FD3D_FIELD_XZ  8

/* fault-plane (nxt,nzt) arrays for fd3d_fetch_plane */
#define FD3D_PLANE_TX        0
#define FD3D_PLANE_TZ        1
#define FD3D_PLANE_SLIPX     2
#define FD3D_PLANE_SLIPZ     3
#define FD3D_PLANE_RUPTIME   4
#define FD3D_PLANE_RISE      5   /* last time above threshold (before rise-=ruptime) */
#define FD3D_PLANE_SLIPTIME  6
#define FD3D_PLANE_DISTX     7
#define FD3D_PLANE_DISTZ     8
#define FD3D_PLANE_PSIX      9
#define FD3D_PLANE_PSIZ     10
#define FD3D_PLANE_T0X      11
#define FD3D_PLANE_T0Z      12
#define FD3D_PLANE_SCHANGEX 13
#define FD3D_PLANE_SCHANGEZ 14
#define FD3D_PLANE_RVEL     15   /* rupture velocity (rvel.res), after fd3d_post_process */
#define FD3D_PLANE_CZONE    16   /* cohesive zone (czone.res), after fd3d_post_process   */
#define FD3D_PLANE_NPLANES  17

#define FD3D_MAX_STATIONS 10  /* units 31..40 of the reference (fd3d_theo.f90:117-128) */

/*
 * Grid and run parameters: the contents of inputfd3d.dat (fd3d_init.f90:145-173)
 * after padding.  nxt = nxtT + 2*nabc, nyt = nytT + nabc, nzt = nztT + nabc + nfs,
 * fault plane at j = nyt (nysc = nyt).
 */
typedef struct fd3d_params {
    int    nxt, nyt, nzt;      /* padded grid                                     */
    int    nabc;               /* PML thickness (cells)                           */
    int    nfs;                /* rows above the free surface: 2, or nabc with fspace */
    int    ntfd;               /* number of time steps of a full solve            */
    double dh, dt;             /* grid step [m], time step [s]                    */
    double damp_s;             /* damping near the fault                          */
    double pml_vp, pml_fact;   /* omegaM_pml = pml_fact*pml_vp/(2*dh*(nabc-1))    */
    double vp_max;             /* for the CFL check; <=0 skips it                 */
    int    law;                /* FD3D_LAW_SW | FD3D_LAW_FVW                      */
    int    precision;          /* FD3D_PREC_F32 | FD3D_PREC_F64                   */
    int    nstations;          /* 0..FD3D_MAX_STATIONS                            */
    int    staX[FD3D_MAX_STATIONS], staY[FD3D_MAX_STATIONS], staZ[FD3D_MAX_STATIONS]; /* 1-based */
    int    history_stride;     /* keep history planes every n-th step (>=1)       */
    int    history_capacity;   /* device ring capacity in records (0 = default)   */
    int    fspace;             /* 1: the FSPACE build (fd3d_init.f90:161-165): nfs = nabc and a
                                  fifth PML strip above k = nzt-nfs instead of the free surface
                                  (fd3d_deriv.f90:1413-1493, 2223-2293, 2996-3143); no fuvw/fres,
                                  the top fault row uses the full 4th-order traction
                                  (fd3d_theo.f90:213-227, 260-283); 0: free surface        */
} fd3d_params;

/*
 * Fault parameters on the (nxt,nzt) plane, Fortran order, double precision.
 * SW uses striniX/Z, peak_xz, dyn_xz, Dc, coh; interp_fric is applied inside
 * the library (X-node values are 4-point averages, fd3d_deriv.f90:3174-3189).
 * FVW uses striniX/Z, Dc, a, b, psi, vw (Z nodes) and aX, bX, psiX, vwX (X nodes
 * come straight from the setup, fd3d_init.f90:471-499), plus the scalars.
 * fwZ/fwX are optional per-node weakened friction coefficients (an extension:
 * the reference has one scalar fw, fd3d_init.f90:61); NULL means use fw.
 */
typedef struct fd3d_fault {
    const double *striniX, *striniZ, *Dc;
    const double *peak_xz, *dyn_xz, *coh;                 /* SW  */
    const double *a, *b, *psi, *vw;                       /* FVW, Z nodes */
    const double *aX, *bX, *psiX, *vwX;                   /* FVW, X nodes */
    const double *fwZ, *fwX;                              /* FVW, optional */
    double Sn, v0, f0, fw, uini, wini;                    /* FVW scalars  */
    int    nucleation;   /* 0 off; 1 TPV103/104 ramp T0X = strinixI + bump (fd3d_theo.f90:487-542);
                            2 the same bump added to each node's initial T0X (an extension that
                            equals 1 when striniX is uniform, as in the TPV104 deck) */
    double hx0, hz0, perturb, RR2, TT2, strinixI;         /* fd3d_theo.f90:487-542  */
} fd3d_fault;

typedef struct fd3d_ctx fd3d_ctx;

/* library info */
const char* fd3d_version(void);
/* sizeof(fd3d_params) and sizeof(fd3d_fault) as this library was built, for hosts that
 * declare the structs themselves (a Fortran bind(C) type, ctypes) to check their layout. */
int fd3d_struct_sizes(size_t* params_bytes, size_t* fault_bytes);
const char* fd3d_status_string(int status);
int fd3d_device_count(int* count);
/* device used by contexts created afterwards on the calling host thread */
int fd3d_set_device(int device);

/* single model */
int fd3d_ctx_create(const fd3d_params* p, fd3d_ctx** out);
int fd3d_ctx_destroy(fd3d_ctx* ctx);
int fd3d_upload_medium(fd3d_ctx* ctx, const void* lam1, const void* mu1, const void* d1, int real_kind);
/* 1-D layered medium as built by readcrustalmodel (fd3d_init.f90:241-265): one value per k */
int fd3d_upload_medium_layers(fd3d_ctx* ctx, const double* lam_k, const double* mu_k, const double* d_k);
int fd3d_upload_fault(fd3d_ctx* ctx, const fd3d_fault* f);
/* Slip-weakening fault from the control points an inversion sampler writes to
 * forwardmodel.dat (readinversionresult, fd3d_init.f90:839-857): nli x nwi arrays in
 * Fortran order of prestress T0I, static friction TsI (scaled by the normal stress
 * normstress(k), fd3d_init.f90:77-86, dip in degrees, dipslip selects the DIPSLIP
 * build) and Dc.  The bilinear interpolation onto the fault plane
 * (inversion_modeltofd3d, fd3d_init.f90:802-835) and interp_fric run on the device;
 * dynamic friction and cohesion are 0 as there. */
int fd3d_upload_fault_model(fd3d_ctx* ctx, int nli, int nwi, const double* T0I, const double* TsI,
                            const double* DcI, double dip, int dipslip);
int fd3d_reset(fd3d_ctx* ctx);                      /* zero wave field, PML and fault state (fd3d_theo.f90:59-88) */
/* Checkpoint and resume (the reference has no restart files; its state lives in module
 * arrays for one run).  fd3d_checkpoint waits for the enqueued steps and writes the
 * context's whole state -- parameters, wave field, medium, PML split components, fault
 * planes, step counter and the history/station rings -- to one file (about the context's
 * device memory in size).  fd3d_restore creates a context on the current device from such
 * a file; fd3d_run on it continues the run bit for bit.  FD3D_ERR_IO on a file that is not
 * a checkpoint of this library's layout. */
int fd3d_checkpoint(fd3d_ctx* ctx, const char* path);
int fd3d_restore(const char* path, fd3d_ctx** out);
int fd3d_run(fd3d_ctx* ctx, int nsteps);            /* enqueue nsteps time steps; asynchronous */
int fd3d_sync(fd3d_ctx* ctx);                       /* wait; returns first device error        */
/* No counterpart in the reference.  Same time steps as fd3d_run, for hosts that cannot
 * let the library allocate device memory once their run has started (device memory
 * owned by another runtime, e.g. a Fortran host's OpenACC data region, or reserved up
 * front against a fixed budget).  It calls no cudaMalloc/cudaFree and instantiates no
 * graph: it launches the step kernels one by one, the fault boundary condition as four
 * launches whose trial-traction scratch lives in a fixed device array of the library
 * (2 planes of doubles for up to 2^20 = nxt*nzt fault-plane nodes, 16 MiB held on every
 * GPU that loads the library until exit).  Larger planes are rejected with FD3D_ERR_ARG.
 * The first call on a device looks up that array's device address, so make it before
 * any stream capture; the address is kept for the life of the process, so a device
 * reset between calls is not supported.  The call runs on the context's device whatever
 * device the calling thread has current.  All calls share the array: calls whose work
 * overlaps on one GPU (contexts on different streams) race on it. */
int fd3d_run_noalloc(fd3d_ctx* ctx, int nsteps);
int fd3d_steps_done(fd3d_ctx* ctx, int* it);
/* Records rec0..rec0+nrec-1 of one history plane (x fastest per record).  Waits only for
 * the fd3d_run that made the last of them: runs enqueued after it keep the GPU busy while
 * the records are copied (they must still be in the ring, which holds history_capacity
 * records counted back from the last enqueued step).  fd3d_fetch_stations likewise. */
int fd3d_fetch_history(fd3d_ctx* ctx, int field, int rec0, int nrec, void* host, int real_kind);
int fd3d_history_records(fd3d_ctx* ctx, int* nrec);  /* records held in the device ring */
int fd3d_fetch_stations(fd3d_ctx* ctx, int rec0, int nrec, double* host /* nrec*nst*3 */);
int fd3d_fetch_field(fd3d_ctx* ctx, int field, void* host, int real_kind);     /* (nxt,nyt,nzt) */
int fd3d_fetch_plane(fd3d_ctx* ctx, int plane, double* host);                  /* (nxt,nzt)     */
int fd3d_fetch_final(fd3d_ctx* ctx, double* slipX, double* slipZ, double* ruptime,
                     double* rise, double* sliptime);
int fd3d_write_results(fd3d_ctx* ctx, const char* dir, int real_kind);
/* Moment rate of history records rec0..rec0+nrec-1 (still in the device ring): the sum
 * over the interior fault plane of |slip rate| * mu(i,nyt,k) * dh^2, reduced on the
 * device in FP64 -- MomentRate of fd3d_theo.f90:574-578 with the seismogram step equal
 * to dt (for a coarser step the reference averages consecutive records). */
int fd3d_fetch_moment_rate(fd3d_ctx* ctx, int rec0, int nrec, double* host);
/* The post-loop quantities of fd3d_theo.f90:604-749 on the device: fills the
 * FD3D_PLANE_RVEL and FD3D_PLANE_CZONE planes and out4 = {average rupture speed,
 * seismic moment M0, rupture area (0: the reference never assigns it), average
 * stress drop}. */
int fd3d_post_process(fd3d_ctx* ctx, double* out4);
/* host-visible timing of the last fd3d_run span, CUDA events on the ctx stream */
int fd3d_last_run_ms(fd3d_ctx* ctx, float* ms);
/* per-kernel timing over the last run when profiling is switched on */
int fd3d_set_profiling(fd3d_ctx* ctx, int on);
int fd3d_kernel_times(fd3d_ctx* ctx, float* ms /* FD3D_NKERNELS */, int* launches);
/* How the context runs its time step (no counterpart in the reference).  interior_variant:
 * FD3D_INTERIOR_TMA, the interior sweeps fed by 3-D tensor-memory-accelerator tiles (the
 * default), or a slower plain-load variant, taken when the tensor maps cannot be encoded for
 * this grid (a message on stderr says so at creation) or when the FD3D_INTERIOR environment
 * variable selects it.  layered_medium: 1 when the uploaded medium varies with depth only and
 * the sweeps read one value per plane.  Either pointer may be NULL. */
#define FD3D_INTERIOR_POINT 0
#define FD3D_INTERIOR_TILED 1
#define FD3D_INTERIOR_PIPE  2
#define FD3D_INTERIOR_TMA   3
int fd3d_ctx_info(fd3d_ctx* ctx, int* interior_variant, int* layered_medium);
#define FD3D_NKERNELS 8
/* kernel ids in fd3d_kernel_times: 0 vel_interior, 1 vel_fault, 2 vel_pml, 3 vel_fs,
   4 str_interior, 5 str_fault, 6 str_pml, 7 fault_bc (traction+friction+output) */

/* ---- many models in one launch schedule ---------------------------------
 * No counterpart in the reference, which runs one model per process
 * (src/dynamicsolver.f90:66).  Independent forward models of uneven size share one
 * device arena of arena_bytes; fd3d_batch_run advances every live model by up to
 * nsteps steps (each stops at its own ntfd).  Two schedules run the same work items:
 * FD3D_BATCH_PERSISTENT, one cooperative kernel per run whose CTAs walk the items
 * phase by phase between grid barriers, and FD3D_BATCH_GRAPH, CUDA graphs of 32, 16,
 * 8, 4, 2 or 1 steps with one kernel per region and step over all models, in series
 * on one stream (FD3D_BATCH_BRANCHES=1 runs the interior, fault-band and PML sweeps of
 * a half-step as parallel branches instead).
 * fd3d_batch_autotune picks the schedule and its tile shape.  Models use the FP32
 * build, a 1-D layered medium (one value per k, as readcrustalmodel builds) and keep
 * the last history_capacity records (default 16) of their history planes.  A model's
 * results are the same bits whether it runs alone or among others, in either schedule. */
#define FD3D_BATCH_PERSISTENT 0
#define FD3D_BATCH_GRAPH 1
typedef struct fd3d_batch fd3d_batch;
int fd3d_batch_create(size_t arena_bytes, int max_models, fd3d_batch** out);
int fd3d_batch_destroy(fd3d_batch* b);
int fd3d_batch_bytes_needed(const fd3d_params* p, size_t* bytes);       /* arena bytes one model takes */
int fd3d_batch_add(fd3d_batch* b, const fd3d_params* p, const double* lam_k, const double* mu_k,
                   const double* d_k, const fd3d_fault* f, int* slot);   /* FD3D_ERR_NOMEM: arena full */
int fd3d_batch_remove(fd3d_batch* b, int slot);
int fd3d_batch_reset(fd3d_batch* b, int slot);                          /* back to step 0 */
int fd3d_batch_run(fd3d_batch* b, int nsteps);
int fd3d_batch_sync(fd3d_batch* b);
int fd3d_batch_model_status(fd3d_batch* b, int slot);                   /* per-model device error */
int fd3d_batch_last_run_ms(fd3d_batch* b, float* ms);
int fd3d_batch_steps_done(fd3d_batch* b, int slot, int* it);
int fd3d_batch_live(fd3d_batch* b, int* nlive, size_t* bytes_in_use);
int fd3d_batch_fetch_plane(fd3d_batch* b, int slot, int plane, double* host);
int fd3d_batch_fetch_final(fd3d_batch* b, int slot, double* slipX, double* slipZ, double* ruptime,
                           double* rise, double* sliptime);
int fd3d_batch_fetch_history(fd3d_batch* b, int slot, int field, int rec0, int nrec, double* host);
/* tile shape: z-planes per interior tile and, for the persistent schedule, CTAs per SM (0 = max) */
int fd3d_batch_set_tuning(fd3d_batch* b, int kchunk, int ctas_per_sm);
int fd3d_batch_get_tuning(fd3d_batch* b, int* kchunk, int* ctas_per_sm, int* max_ctas_per_sm);
/* schedule: FD3D_BATCH_PERSISTENT or FD3D_BATCH_GRAPH (the default) */
int fd3d_batch_set_schedule(fd3d_batch* b, int mode);
int fd3d_batch_get_schedule(fd3d_batch* b, int* mode);
/* times the tile-shape candidates on the live models (all at step 0), keeps the fastest,
 * resets the models; cache_path/key (optional) persist the choice as JSON lines */
int fd3d_batch_autotune(fd3d_batch* b, int steps, const char* cache_path, const char* key);

/* ---- one model over several GPUs: z-slabs ------------------------------
 * No counterpart in the reference, which runs one model in one process on one GPU
 * (src/dynamicsolver.f90:66; its -DGPUMPI switch is unused).  The model's planes
 * k = 1..nzt are split into slabs of consecutive planes, one context each (on one
 * device or several); a slab stores its own planes and three halo planes on either side,
 * the full fault plane and the full PML split-component pool, and updates only its own
 * planes and fault rows.  The slabs of one model step together in a group: after the
 * velocity sweeps, the stress sweeps, the trial traction and the friction law each slab
 * pulls two halo planes (or fault-plane rows) of what its neighbours just updated.  The
 * results are the same bits as one context's.  Uploads take the whole model's arrays on
 * every slab; fd3d_fetch_field, fd3d_fetch_history, fd3d_fetch_stations and
 * fd3d_fetch_plane return the slab's own planes / rows / stations (the rest untouched in
 * the host array, or zero), so the slabs of a model fill one result between them.
 * fd3d_run, fd3d_run_noalloc, fd3d_checkpoint, fd3d_post_process,
 * fd3d_fetch_moment_rate and fd3d_write_results refuse a slab context (FD3D_ERR_STATE). */
/* a slab of at least 4 planes; the top slab (k_hi = nzt) owns nzt-nfs-2 .. nzt */
int fd3d_ctx_create_slab(const fd3d_params* p, int k_lo, int k_hi, fd3d_ctx** out);
int fd3d_slab_range(fd3d_ctx* ctx, int* k_lo, int* k_hi);
/* n slabs of about equal cost (host arithmetic only: no device is needed) */
int fd3d_slab_plan(const fd3d_params* p, int n, int* k_lo, int* k_hi);
/* the first of the two planes / fault rows a slab owning k_lo..k_hi sends to, and receives
 * from, its neighbour below (side 0) or above (side 1); host arithmetic only */
int fd3d_slab_halo_plan(int k_lo, int k_hi, int side, int* send_k0, int* recv_k0);
typedef struct fd3d_slab_group fd3d_slab_group;
/* ctxs: the slabs of one model from the bottom (k_lo = 1) up */
int fd3d_slab_group_create(fd3d_ctx* const* ctxs, int n, fd3d_slab_group** out);
int fd3d_slab_group_run(fd3d_slab_group* g, int nsteps);
/* waits for every slab; *ms = the longest slab's time of the last run */
int fd3d_slab_group_sync(fd3d_slab_group* g, float* ms);
int fd3d_slab_group_destroy(fd3d_slab_group* g);   /* the contexts stay */
/* The slabs in separate processes, one GPU each (torch.distributed ranks): the same
 * exchange as a group's, as NCCL send/receive pairs with the ranks below and above on the
 * slab's stream.  Rank r holds the r-th slab from the bottom.  NCCL (libnccl.so.2) is
 * loaded on first use; FD3D_ERR_NODEV if it cannot be.  fd3d_nccl_unique_id fills the
 * 128-byte id that rank 0 makes and every rank passes to fd3d_slab_connect. */
int fd3d_nccl_unique_id(unsigned char* id);
int fd3d_slab_connect(fd3d_ctx* ctx, const unsigned char* id, int rank, int nranks);
int fd3d_slab_run(fd3d_ctx* ctx, int nsteps);       /* then fd3d_sync(ctx) */

/* ---- self-test ----------------------------------------------------------
 * No counterpart in the reference.  The PML kernels divide by dh and by 1 + omega
 * (fd3d_deriv.f90:1498-1925) through a quotient formed from a reciprocal computed on
 * the host; this runs that routine and the IEEE division on all 2^32 float bit
 * patterns for each of the n divisors on the current device and stores the number
 * of dividends whose quotients differ (0 expected) and the first such bit pattern
 * (0xffffffff if none). */
int fd3d_check_division(const float* divisors, int n, unsigned long long* mismatches, unsigned* first_bad);
/* Self-test of the bounded device waits (no counterpart in the reference, whose GPU
 * regions never wait on each other): a kernel waits on an mbarrier phase that nothing
 * completes and a grid barrier that one CTA never reaches.  Both waits must give up after
 * their bound and record the timeout bit (4) in the status word returned here; the device
 * stays usable.  Takes about a second. */
int fd3d_check_waits(int* mbar_status, int* barrier_status);

/* ---- input decks (the reference's own files) --------------------------- */
/* Reads inputfd3d.dat and crustal.dat from dir (fd3d_init.f90:145-173, 211-279),
 * fills p and returns lam1/mu1/d1 (caller frees with fd3d_free). */
int fd3d_read_deck(const char* dir, fd3d_params* p, double** lam1, double** mu1, double** d1);
/* The same for the build selected by fspace (1: FSPACE, nfs = nabc, as the reference's
 * compile switch does in fd3d_init.f90:161-165; 0: as fd3d_read_deck). */
int fd3d_read_deck_ex(const char* dir, int fspace, fd3d_params* p, double** lam1, double** mu1, double** d1);
void fd3d_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* FD3D_GPU_H */
