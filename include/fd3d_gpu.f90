! fd3d_gpu.f90 -- Fortran interface module of the C ABI in fd3d_gpu.h, for a Fortran host
! (the reference's dynamicsolver) that replaces `call fd3d()` (src/fd3d_theo.f90:22) with
! calls into libfd3d_gpu.so.  Scalars pass by value, arrays as c_loc() of the host's own
! arrays (Fortran column-major, as the library expects); status codes are FD3D_OK (0) or a
! negative FD3D_ERR_* (fd3d_gpu.h).  The derived types mirror fd3d_params and fd3d_fault
! field for field; fd3d_struct_sizes returns the C sizes to compare with at start-up.
! (No Fortran compiler exists in the build image, so this file is not compiled by build().)
module fd3d_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: FD3D_OK = 0
  integer(c_int), parameter :: FD3D_ERR_ARG = -1, FD3D_ERR_CFL = -2, FD3D_ERR_CUDA = -3
  integer(c_int), parameter :: FD3D_ERR_NOMEM = -4, FD3D_ERR_NEWTON = -5, FD3D_ERR_NONFINITE = -6
  integer(c_int), parameter :: FD3D_ERR_STATE = -7, FD3D_ERR_IO = -8, FD3D_ERR_NODEV = -9
  integer(c_int), parameter :: FD3D_ERR_BUSY = -10, FD3D_ERR_TIMEOUT = -11
  integer(c_int), parameter :: FD3D_LAW_SW = 0, FD3D_LAW_FVW = 1
  integer(c_int), parameter :: FD3D_PREC_F32 = 0, FD3D_PREC_F64 = 1
  integer(c_int), parameter :: FD3D_INTERIOR_POINT = 0, FD3D_INTERIOR_TILED = 1
  integer(c_int), parameter :: FD3D_INTERIOR_PIPE = 2, FD3D_INTERIOR_TMA = 3

  type, bind(C) :: fd3d_params
    integer(c_int) :: nxt, nyt, nzt, nabc, nfs, ntfd
    real(c_double) :: dh, dt, damp_s, pml_vp, pml_fact, vp_max
    integer(c_int) :: law, precision, nstations
    integer(c_int) :: staX(10), staY(10), staZ(10)
    integer(c_int) :: history_stride, history_capacity, fspace
  end type

  type, bind(C) :: fd3d_fault
    type(c_ptr) :: striniX, striniZ, Dc, peak_xz, dyn_xz, coh
    type(c_ptr) :: a, b, psi, vw, aX, bX, psiX, vwX, fwZ, fwX
    real(c_double) :: Sn, v0, f0, fw, uini, wini
    integer(c_int) :: nucleation
    real(c_double) :: hx0, hz0, perturb, RR2, TT2, strinixI
  end type

  interface
    integer(c_int) function fd3d_struct_sizes(params_bytes, fault_bytes) bind(C)
      import
      integer(c_size_t) :: params_bytes, fault_bytes
    end function
    integer(c_int) function fd3d_ctx_create(p, ctx) bind(C)
      import
      type(fd3d_params), intent(in) :: p
      type(c_ptr) :: ctx
    end function
    integer(c_int) function fd3d_ctx_destroy(ctx) bind(C)
      import
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function fd3d_upload_medium(ctx, lam1, mu1, d1, real_kind) bind(C)
      import
      type(c_ptr), value :: ctx, lam1, mu1, d1
      integer(c_int), value :: real_kind
    end function
    integer(c_int) function fd3d_upload_fault(ctx, f) bind(C)
      import
      type(c_ptr), value :: ctx
      type(fd3d_fault), intent(in) :: f
    end function
    integer(c_int) function fd3d_upload_fault_model(ctx, nli, nwi, T0I, TsI, DcI, dip, dipslip) bind(C)
      import
      type(c_ptr), value :: ctx, T0I, TsI, DcI
      integer(c_int), value :: nli, nwi, dipslip
      real(c_double), value :: dip
    end function
    integer(c_int) function fd3d_reset(ctx) bind(C)
      import
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function fd3d_run(ctx, nsteps) bind(C)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function fd3d_run_noalloc(ctx, nsteps) bind(C)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function fd3d_sync(ctx) bind(C)
      import
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function fd3d_ctx_info(ctx, interior_variant, layered_medium) bind(C)
      import
      type(c_ptr), value :: ctx
      integer(c_int) :: interior_variant, layered_medium
    end function
    integer(c_int) function fd3d_fetch_history(ctx, field, rec0, nrec, host, real_kind) bind(C)
      import
      type(c_ptr), value :: ctx, host
      integer(c_int), value :: field, rec0, nrec, real_kind
    end function
    integer(c_int) function fd3d_fetch_final(ctx, slipX, slipZ, ruptime, rise, sliptime) bind(C)
      import
      type(c_ptr), value :: ctx, slipX, slipZ, ruptime, rise, sliptime
    end function
    integer(c_int) function fd3d_write_results(ctx, dir, real_kind) bind(C)
      import
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: dir(*)
      integer(c_int), value :: real_kind
    end function
    integer(c_int) function fd3d_checkpoint(ctx, path) bind(C)
      import
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function fd3d_restore(path, ctx) bind(C)
      import
      character(kind=c_char), intent(in) :: path(*)
      type(c_ptr) :: ctx
    end function
    ! one model over several GPUs: z-slabs (one MPI rank per GPU: fd3d_nccl_unique_id on
    ! rank 0, MPI_Bcast of the 128 bytes, fd3d_slab_connect and fd3d_slab_run on every rank)
    integer(c_int) function fd3d_slab_plan(p, n, k_lo, k_hi) bind(C)
      import
      type(fd3d_params), intent(in) :: p
      integer(c_int), value :: n
      integer(c_int) :: k_lo(*), k_hi(*)
    end function
    integer(c_int) function fd3d_ctx_create_slab(p, k_lo, k_hi, ctx) bind(C)
      import
      type(fd3d_params), intent(in) :: p
      integer(c_int), value :: k_lo, k_hi
      type(c_ptr) :: ctx
    end function
    integer(c_int) function fd3d_nccl_unique_id(id) bind(C)
      import
      character(kind=c_char) :: id(128)
    end function
    integer(c_int) function fd3d_slab_connect(ctx, id, rank, nranks) bind(C)
      import
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(in) :: id(128)
      integer(c_int), value :: rank, nranks
    end function
    integer(c_int) function fd3d_slab_run(ctx, nsteps) bind(C)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
    end function
  end interface
end module fd3d_gpu
