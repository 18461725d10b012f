! mhd3d_gpu.f90 -- ISO_C_BINDING interface of the B200 time-step library
! (include/mhd3d.h) for the reference's Fortran driver.
!
! The driver keeps its COMMON blocks and calls these routines in place of
! CALL STEP (3dmhd.f:912).  The derived type mirrors struct mhd3d_params
! field for field.
module mhd3d_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: MHD3D_OK = 0, MHD3D_ERR_ARG = 1, MHD3D_ERR_CUDA = 2, &
       MHD3D_ERR_NONFINITE = 3, MHD3D_ERR_DT_SMALL = 4, MHD3D_ERR_NO_DEVICE = 5, &
       MHD3D_ERR_TIMEOUT = 6, MHD3D_ERR_NOMEM = 7
  integer(c_int), parameter :: MHD3D_MODE_EXACT = 0, MHD3D_MODE_FAST = 1, MHD3D_MODE_FP32 = 2
  integer(c_int), parameter :: MHD3D_NPROF = 7, MHD3D_PROF_RHO = 0, MHD3D_PROF_T = 1, MHD3D_PROF_KE = 2, &
       MHD3D_PROF_ENTH = 3, MHD3D_PROF_FCONV = 4, MHD3D_PROF_FRAD = 5, MHD3D_PROF_ME = 6

  type, bind(C) :: mhd3d_params
     integer(c_int32_t) :: npx, npy, npz
     integer(c_int32_t) :: lmag, lrot
     integer(c_int32_t) :: izcon, itcon, ibcon
     integer(c_int32_t) :: mode, reserved0
     real(c_double) :: c13, c23, c43
     real(c_double) :: hx, h2x, hy, h2y, hz, h2z
     real(c_double) :: gam1, gam2, gam3, zeta1, zeta2
     real(c_double) :: cv, ocv, ore, re, repr, theta, grav, gamma, sf
     real(c_double) :: omx, omz
     real(c_double) :: orm, rm, obeta
     real(c_double) :: tb, tp, tc, xp, yp, hh
     real(c_double) :: timi, timc
     real(c_double) :: dtmin
  end type mhd3d_params

  interface
     integer(c_int) function mhd3d_create(p, exx, dxxdx, d2xxdx2, ddx, wyy, dyydy, d2yydy2, ddy, &
          zee, dzzdz, d2zzdz2, ddz, rkapa, dkapa, handle) bind(C, name="mhd3d_create")
       import :: c_int, c_double, c_ptr, mhd3d_params
       type(mhd3d_params), intent(in) :: p
       real(c_double), intent(in) :: exx(*), dxxdx(*), d2xxdx2(*), ddx(*)
       real(c_double), intent(in) :: wyy(*), dyydy(*), d2yydy2(*), ddy(*)
       real(c_double), intent(in) :: zee(*), dzzdz(*), d2zzdz2(*), ddz(*)
       real(c_double), intent(in) :: rkapa(*), dkapa(*)
       type(c_ptr), intent(out) :: handle
     end function mhd3d_create

     integer(c_int) function mhd3d_destroy(handle) bind(C, name="mhd3d_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
     end function mhd3d_destroy

     integer(c_int) function mhd3d_upload(handle, ru, rv, rw, tt, ro, bx, by, bz) bind(C, name="mhd3d_upload")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: handle
       real(c_double), intent(in) :: ru(*), rv(*), rw(*), tt(*), ro(*), bx(*), by(*), bz(*)
     end function mhd3d_upload

     integer(c_int) function mhd3d_download(handle, ru, rv, rw, tt, ro, bx, by, bz) bind(C, name="mhd3d_download")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: handle
       real(c_double), intent(out) :: ru(*), rv(*), rw(*), tt(*), ro(*), bx(*), by(*), bz(*)
     end function mhd3d_download

     integer(c_int) function mhd3d_step(handle, nsteps, dt, timc, timt, umach, nit) bind(C, name="mhd3d_step")
       import :: c_int, c_int32_t, c_double, c_ptr
       type(c_ptr), value :: handle
       integer(c_int32_t), value :: nsteps
       real(c_double), intent(out) :: dt, timc, timt, umach
       integer(c_int32_t), intent(out) :: nit
     end function mhd3d_step

     integer(c_int) function mhd3d_cfl(handle, dt, umach) bind(C, name="mhd3d_cfl")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: handle
       real(c_double), intent(out) :: dt, umach
     end function mhd3d_cfl

     integer(c_int) function mhd3d_bcon(handle) bind(C, name="mhd3d_bcon")
       import :: c_int, c_ptr
       type(c_ptr), value :: handle
     end function mhd3d_bcon

     ! PROF(NPZ, MHD3D_NPROF): column r+1 holds row MHD3D_PROF_* = r for K=2..NZ-1
     integer(c_int) function mhd3d_profiles(handle, prof) bind(C, name="mhd3d_profiles")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: handle
       real(c_double), intent(out) :: prof(*)
     end function mhd3d_profiles

     ! CFL/Mach reduction that allocates nothing, for hosts whose device
     ! arrays are declared statically: every array argument is a device
     ! address (c_loc of a device array), out receives DT, UMACH and the
     ! non-finite flag on the device, stream is a cudaStream_t or c_null_ptr
     integer(c_int) function mhd3d_cfl_noalloc(p, ru, rv, rw, tt, ro, bx, by, bz, ddx, ddy, ddz, rkapa, &
          out, stream) bind(C, name="mhd3d_cfl_noalloc")
       import :: c_int, c_ptr, mhd3d_params
       type(mhd3d_params), intent(in) :: p
       type(c_ptr), value :: ru, rv, rw, tt, ro, bx, by, bz
       type(c_ptr), value :: ddx, ddy, ddz, rkapa
       type(c_ptr), value :: out, stream
     end function mhd3d_cfl_noalloc

     ! Per-plane bias tendency of an FP32 coarse run's closure (no counterpart
     ! in the reference driver): BIAS(K-1, F) for plane K=2..NZ-1 and field
     ! F = RU, RV, RW, TT, BX, BY, BZ (1..7), an NPZ x 7 array; the wall
     ! planes K=2 and K=NZ-1 take none.  Without a network attached every
     ! step adds the bias alone.
     integer(c_int) function mhd3d_closure_set_bias(handle, bias) bind(C, name="mhd3d_closure_set_bias")
       import :: c_int, c_float, c_ptr
       type(c_ptr), value :: handle
       real(c_float), intent(in) :: bias(*)
     end function mhd3d_closure_set_bias

     ! steps that fell back to the plain coarse method, network evaluations,
     ! and the closure kernels' error flag
     integer(c_int) function mhd3d_closure_status(handle, trips, evals, err) bind(C, name="mhd3d_closure_status")
       import :: c_int, c_int32_t, c_ptr
       type(c_ptr), value :: handle
       integer(c_int32_t), intent(out) :: trips, evals, err
     end function mhd3d_closure_status
  end interface
end module mhd3d_gpu
