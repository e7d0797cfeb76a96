! cueva_gpu.f90 -- ISO_C_BINDING interface of include/cueva.h for the CUEVA
! Fortran driver (cueva_2D_base/main_cueva_code.f95).  Source only: no
! Fortran compiler exists in the build image, so this module is not compiled
! or tested here; the C++ stand-in driver (host/cueva_driver.cpp) exercises
! the same calls on arrays with the Fortran layout.
!
! Use from the reference driver:
!   use cueva_gpu
!   type(c_ptr) :: ctx
!   call cueva_attach(ctx)                       ! after init_var_primitive
!   do h = hini, hmax-1
!      ierr = cueva_step(ctx, 1)                 ! replaces main_cueva_code.f95:53-326
!      if (mod(h, hloc) == 0) ierr = cueva_download(ctx, CUEVA_G_PRIMS)
!      call boundary ; call lector               ! unchanged Fortran I/O path
!   end do
module cueva_gpu
  use iso_c_binding
  implicit none

  integer(c_int32_t), parameter :: CUEVA_OK = 0, CUEVA_ERR_ARG = 1, CUEVA_ERR_CUDA = 2
  integer(c_int32_t), parameter :: CUEVA_ERR_UNBOUND = 3, CUEVA_ERR_PHYSICS = 4
  integer(c_int32_t), parameter :: CUEVA_G_PRIMS = 1, CUEVA_G_CONS = 2

  ! field ids, same order as enum cueva_field
  integer(c_int32_t), parameter :: CUEVA_RHO = 0, CUEVA_P = 1, CUEVA_VX = 2, CUEVA_VY = 3, CUEVA_VZ = 4
  integer(c_int32_t), parameter :: CUEVA_PSI = 5, CUEVA_PHI = 6, CUEVA_EX = 7, CUEVA_EY = 8, CUEVA_EZ = 9
  integer(c_int32_t), parameter :: CUEVA_BX = 10, CUEVA_BY = 11, CUEVA_BZ = 12, CUEVA_Q = 13
  integer(c_int32_t), parameter :: CUEVA_D = 14, CUEVA_TAU = 15, CUEVA_SX = 16, CUEVA_SY = 17, CUEVA_SZ = 18
  integer(c_int32_t), parameter :: CUEVA_W = 19
  integer(c_int32_t), parameter :: CUEVA_PSIINT = 20, CUEVA_PHIINT = 21, CUEVA_EXINT = 22, CUEVA_EYINT = 23
  integer(c_int32_t), parameter :: CUEVA_EZINT = 24, CUEVA_BXINT = 25, CUEVA_BYINT = 26, CUEVA_BZINT = 27
  integer(c_int32_t), parameter :: CUEVA_QINT = 28, CUEVA_DDINT = 29, CUEVA_TAUINT = 30, CUEVA_SXINT = 31
  integer(c_int32_t), parameter :: CUEVA_SYINT = 32, CUEVA_SZINT = 33, CUEVA_JXINT = 34, CUEVA_JYINT = 35
  integer(c_int32_t), parameter :: CUEVA_JZINT = 36, CUEVA_EXAST = 37, CUEVA_EYAST = 38, CUEVA_EZAST = 39
  integer(c_int32_t), parameter :: CUEVA_PSIFLUX = 40, CUEVA_PHIFLUX = 41, CUEVA_EXASTFLUX = 42
  integer(c_int32_t), parameter :: CUEVA_EYASTFLUX = 43, CUEVA_EZASTFLUX = 44, CUEVA_BXFLUX = 45
  integer(c_int32_t), parameter :: CUEVA_BYFLUX = 46, CUEVA_BZFLUX = 47, CUEVA_QFLUX = 48, CUEVA_DFLUX = 49
  integer(c_int32_t), parameter :: CUEVA_TAUFLUX = 50, CUEVA_SXFLUX = 51, CUEVA_SYFLUX = 52
  integer(c_int32_t), parameter :: CUEVA_SZFLUX = 53, CUEVA_EXASTSOUR = 54, CUEVA_EYASTSOUR = 55
  integer(c_int32_t), parameter :: CUEVA_EZASTSOUR = 56
  ! stage interface fluxes (outputs of the flux routines, fourvectors.f95)
  integer(c_int32_t), parameter :: CUEVA_EXLAXPSI = 57, CUEVA_EYLAXPSI = 58, CUEVA_BXLAXPHI = 59
  integer(c_int32_t), parameter :: CUEVA_BYLAXPHI = 60, CUEVA_PHILAXBX = 61, CUEVA_EZLAXBX = 62
  integer(c_int32_t), parameter :: CUEVA_EZLAXBY = 63, CUEVA_PHILAXBY = 64, CUEVA_EYLAXBZ = 65
  integer(c_int32_t), parameter :: CUEVA_EXLAXBZ = 66, CUEVA_PSILAXEX = 67, CUEVA_BZLAXEX = 68
  integer(c_int32_t), parameter :: CUEVA_BZLAXEY = 69, CUEVA_PSILAXEY = 70, CUEVA_BYLAXEZ = 71
  integer(c_int32_t), parameter :: CUEVA_BXLAXEZ = 72, CUEVA_JXLAX = 73, CUEVA_JYLAX = 74
  integer(c_int32_t), parameter :: CUEVA_FDXLAX = 75, CUEVA_FDYLAX = 76, CUEVA_FTAUXLAX = 77
  integer(c_int32_t), parameter :: CUEVA_FTAUYLAX = 78, CUEVA_FSXXLAX = 79, CUEVA_FSXYLAX = 80
  integer(c_int32_t), parameter :: CUEVA_FSXZLAX = 81, CUEVA_FSYXLAX = 82, CUEVA_FSYYLAX = 83
  integer(c_int32_t), parameter :: CUEVA_FSYZLAX = 84
  ! final stage sums (increments of varfin / electricfield)
  integer(c_int32_t), parameter :: CUEVA_PSIFINSUM = 85, CUEVA_PHIFINSUM = 86, CUEVA_BXFINSUM = 87
  integer(c_int32_t), parameter :: CUEVA_BYFINSUM = 88, CUEVA_BZFINSUM = 89, CUEVA_EXFINSUM = 90
  integer(c_int32_t), parameter :: CUEVA_EYFINSUM = 91, CUEVA_EZFINSUM = 92, CUEVA_QFINSUM = 93
  integer(c_int32_t), parameter :: CUEVA_DFINSUM = 94, CUEVA_TAUFINSUM = 95, CUEVA_SXFINSUM = 96
  integer(c_int32_t), parameter :: CUEVA_SYFINSUM = 97, CUEVA_SZFINSUM = 98

  type, bind(c) :: cueva_params
     integer(c_int32_t) :: imax, jmax, order, flux_solver, rec_mp, c2p, bc_x, bc_y
     integer(c_int32_t) :: precision, device, intsum_reset, primitive_rec
     real(c_double)     :: lx, ly, lz, cfl, sigma, gamma, dt
  end type cueva_params

  ! run diagnostics (enum cueva_diag_slot; Fortran index = C slot + 1):
  ! v(1:35) the lector sums in unit order 80..88, 90..99, 200..215,
  ! v(36:37) max_val_bx, max_val_phi (216, 217), v(38) delta_rec_t (67),
  ! v(39) Ez(imed,jmed) (68), v(40) By(imed+1,jmed+1), v(41:45) Courant check
  integer(c_int32_t), parameter :: CUEVA_NDIAG = 45
  type, bind(c) :: cueva_diag_record
     integer(c_int64_t) :: h
     real(c_double)     :: t
     real(c_double)     :: v(CUEVA_NDIAG)
  end type cueva_diag_record
  type, bind(c) :: cueva_diag_config
     integer(c_int32_t) :: hglb, capacity
     real(c_double)     :: b0, lr, ly, delta_rec
  end type cueva_diag_config

  interface
     integer(c_int32_t) function cueva_ctx_create(p, ctx) bind(c, name="cueva_ctx_create")
       import :: c_int32_t, c_ptr, cueva_params
       type(cueva_params), intent(in) :: p
       type(c_ptr), intent(out) :: ctx
     end function cueva_ctx_create
     integer(c_int32_t) function cueva_ctx_destroy(ctx) bind(c, name="cueva_ctx_destroy")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function cueva_ctx_destroy
     type(c_ptr) function cueva_last_error() bind(c, name="cueva_last_error")
       import :: c_ptr
     end function cueva_last_error
     ! base(*): the whole module array is passed by reference, i.e. the
     ! address of element (-6,-6[,1,1]); the library keeps that address, which
     ! is valid for the life of the program for the static module arrays.
     integer(c_int32_t) function cueva_bind_field(ctx, field, base) bind(c, name="cueva_bind_field")
       import :: c_int32_t, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: field
       real(c_double), intent(inout) :: base(*)
     end function cueva_bind_field
     integer(c_int32_t) function cueva_upload(ctx, groups) bind(c, name="cueva_upload")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: groups
     end function cueva_upload
     integer(c_int32_t) function cueva_download(ctx, groups) bind(c, name="cueva_download")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: groups
     end function cueva_download
     integer(c_int32_t) function cueva_download_async(ctx, groups) bind(c, name="cueva_download_async")
       import :: c_ptr, c_int32_t
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: groups
     end function cueva_download_async
     integer(c_int32_t) function cueva_step(ctx, nsteps) bind(c, name="cueva_step")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: nsteps
     end function cueva_step
     ! one fused kernel per RK stage (1, the default for MP5 and the MC slopes)
     ! or the y-face and x-face + update kernels (0); bit-identical results
     integer(c_int32_t) function cueva_set_stage_kernel(ctx, fused) bind(c, name="cueva_set_stage_kernel")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: fused
     end function cueva_set_stage_kernel
     integer(c_int32_t) function cueva_device_bytes(ctx, nbytes) bind(c, name="cueva_device_bytes")
       import :: c_int32_t, c_int64_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(out) :: nbytes
     end function cueva_device_bytes
     integer(c_int32_t) function cueva_sync(ctx) bind(c, name="cueva_sync")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function cueva_sync
     integer(c_int32_t) function cueva_counters(ctx, out3) bind(c, name="cueva_counters")
       import :: c_int32_t, c_int64_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(out) :: out3(3)
     end function cueva_counters
     integer(c_int32_t) function cueva_startconvar(ctx) bind(c, name="cueva_startconvar")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function cueva_startconvar
     integer(c_int32_t) function cueva_electricvarint(ctx, l) bind(c, name="cueva_electricvarint")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: l
     end function cueva_electricvarint
     integer(c_int32_t) function cueva_flux_rhs(ctx, l) bind(c, name="cueva_flux_rhs")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: l
     end function cueva_flux_rhs
     integer(c_int32_t) function cueva_flux_flow(ctx, l) bind(c, name="cueva_flux_flow")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: l
     end function cueva_flux_flow
     integer(c_int32_t) function cueva_fluxandsource(ctx, l) bind(c, name="cueva_fluxandsource")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int32_t), value :: l
     end function cueva_fluxandsource
     integer(c_int32_t) function cueva_varfin(ctx) bind(c, name="cueva_varfin")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function cueva_varfin
     integer(c_int32_t) function cueva_electricfield(ctx) bind(c, name="cueva_electricfield")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function cueva_electricfield
     integer(c_int32_t) function cueva_con2prim(ctx) bind(c, name="cueva_con2prim")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: ctx
     end function cueva_con2prim
     integer(c_int32_t) function cueva_set_clock(ctx, h, t) bind(c, name="cueva_set_clock")
       import :: c_int32_t, c_int64_t, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: h
       real(c_double), value :: t
     end function cueva_set_clock
     integer(c_int32_t) function cueva_diag_enable(ctx, cfg) bind(c, name="cueva_diag_enable")
       import :: c_int32_t, c_ptr, cueva_diag_config
       type(c_ptr), value :: ctx
       type(cueva_diag_config), intent(in) :: cfg
     end function cueva_diag_enable
     integer(c_int32_t) function cueva_diag_read(ctx, out, max_records, n_out) bind(c, name="cueva_diag_read")
       import :: c_int32_t, c_ptr, cueva_diag_record
       type(c_ptr), value :: ctx
       type(cueva_diag_record), intent(out) :: out(*)
       integer(c_int32_t), value :: max_records
       integer(c_int32_t), intent(out) :: n_out
     end function cueva_diag_read
     integer(c_int32_t) function cueva_diag_now(ctx, out) bind(c, name="cueva_diag_now")
       import :: c_int32_t, c_ptr, cueva_diag_record
       type(c_ptr), value :: ctx
       type(cueva_diag_record), intent(out) :: out
     end function cueva_diag_now
  end interface

contains

  ! Creates a context for the module-global run configuration, binds the
  ! carried primitives of threevectors.f95 and uploads the initial state.
  subroutine cueva_attach(ctx)
    use parameters
    use threevectors
    type(c_ptr), intent(out) :: ctx
    type(cueva_params) :: prm
    integer(c_int32_t) :: ierr
    prm%imax = imax; prm%jmax = jmax; prm%order = order; prm%flux_solver = flux_solver
    prm%rec_mp = rec_mp; prm%c2p = conserved_to_primitive
    prm%bc_x = 0; prm%bc_y = 1                   ! BOUND 6: x copy, y periodic
    if (BOUND == 1) prm%bc_y = 0                 ! copy / copy
    if (BOUND == 2) prm%bc_x = 1                 ! periodic / periodic
    prm%precision = 0; prm%device = 0; prm%intsum_reset = 0
    prm%primitive_rec = primitive_rec           ! parameters.f95:26
    prm%lx = Longx; prm%ly = Longy; prm%lz = Longz; prm%cfl = CFL
    prm%sigma = sigma; prm%gamma = gamma; prm%dt = Delt
    ierr = cueva_ctx_create(prm, ctx)
    if (ierr /= CUEVA_OK) stop "cueva_ctx_create failed"
    ierr = ierr + cueva_bind_field(ctx, CUEVA_RHO, rho)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_P, p)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_VX, Vx)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_VY, Vy)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_VZ, Vz)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_PSI, psi)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_PHI, phi)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_EX, Ex)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_EY, Ey)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_EZ, Ez)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_BX, Bx)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_BY, By)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_BZ, Bz)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_Q, q)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_D, D)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_TAU, tau)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_SX, Sx)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_SY, Sy)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_SZ, Sz)
    ierr = ierr + cueva_bind_field(ctx, CUEVA_W, W)
    if (ierr /= CUEVA_OK) stop "cueva_bind_field failed"
    ierr = cueva_upload(ctx, CUEVA_G_PRIMS)
    if (ierr /= CUEVA_OK) stop "cueva_upload failed"
  end subroutine cueva_attach

end module cueva_gpu
