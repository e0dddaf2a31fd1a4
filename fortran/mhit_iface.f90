! iso_c_binding interface to libmhit.so (include/mhit.h).
!
! A Fortran driver that keeps the reference's module arrays
! (multi/module.f90:39-58, shape (nx, ny+2, nz+2)) passes them straight to
! mhit_set_fields / mhit_get_fields with MHIT_LAYOUT_PIX_HALO; the loop body of
! multi/main.f90:334-946 becomes one mhit_step call.
!
! This image has no Fortran compiler (gfortran, nvfortran and mpif90 are all
! absent), so this module is not compiled here; the same ABI is exercised from
! C (tests/test_host.py) and Python (mhit36_b200/capi.py).
module mhit_iface
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: MHIT_OK = 0, MHIT_ERR_INVALID = 1, MHIT_ERR_CUDA = 2, MHIT_ERR_NOMEM = 3
  integer(c_int), parameter :: MHIT_ERR_CFL = 4, MHIT_ERR_NONFINITE = 5, MHIT_ERR_IO = 6
  integer(c_int), parameter :: MHIT_ERR_UNSUPPORTED = 7, MHIT_ERR_STATE = 8
  integer(c_int), parameter :: MHIT_LAYOUT_RAW = 0, MHIT_LAYOUT_PIX_HALO = 1
  integer(c_int), parameter :: MHIT_FP64 = 0, MHIT_FP32_REFINE = 1
  integer(c_int), parameter :: MHIT_K2_SPECTRAL = 0, MHIT_K2_FD = 1
  integer(c_int), parameter :: MHIT_GRID_REFERENCE = 0, MHIT_GRID_CONSISTENT = 1

  ! struct mhit_params: input.inp lines 1-16, then the extensions
  type, bind(C) :: mhit_params
    integer(c_int32_t) :: restart, tstart, tfin, dump
    integer(c_int32_t) :: inflow, inphi
    real(c_double) :: dt, mu, rho
    real(c_double) :: f1, f2, f3, k0
    real(c_double) :: radius, sigma, epsr
    real(c_double) :: lin_force
    integer(c_int32_t) :: k2_mode, grid_mode
    real(c_double) :: cfl_limit
    integer(c_int32_t) :: tanh_identity, phi_floor
    integer(c_int32_t) :: reserved(6)
  end type mhit_params

  type, bind(C) :: mhit_diag
    real(c_double) :: umax, cfl, umean, vmean, wmean, gamma, max_div
    integer(c_int64_t) :: step
    integer(c_int32_t) :: status, reserved
  end type mhit_diag

  interface
    subroutine mhit_default_params(p) bind(C, name='mhit_default_params')
      import :: mhit_params
      type(mhit_params), intent(out) :: p
    end subroutine

    integer(c_int) function mhit_create(p, nx, ny, nz, precision, phase_field, h) bind(C, name='mhit_create')
      import :: mhit_params, c_int, c_ptr
      type(mhit_params), intent(in) :: p
      integer(c_int), value :: nx, ny, nz, precision, phase_field
      type(c_ptr), intent(out) :: h
    end function

    integer(c_int) function mhit_set_fields(h, u, v, w, phi, layout) bind(C, name='mhit_set_fields')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: u(*), v(*), w(*), phi(*)
      integer(c_int), value :: layout
    end function

    integer(c_int) function mhit_get_fields(h, u, v, w, phi, layout) bind(C, name='mhit_get_fields')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: u(*), v(*), w(*), phi(*)
      integer(c_int), value :: layout
    end function

    integer(c_int) function mhit_get_pressure(h, p, layout) bind(C, name='mhit_get_pressure')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: p(*)
      integer(c_int), value :: layout
    end function

    integer(c_int) function mhit_step(h, nsteps, diag) bind(C, name='mhit_step')
      import :: c_int, c_ptr, mhit_diag
      type(c_ptr), value :: h
      integer(c_int), value :: nsteps
      type(mhit_diag), intent(out) :: diag
    end function

    integer(c_int) function mhit_save(h, dir, t) bind(C, name='mhit_save')
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: dir(*)
      integer(c_int), value :: t
    end function

    integer(c_int) function mhit_load(h, dir, t) bind(C, name='mhit_load')
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: dir(*)
      integer(c_int), value :: t
    end function

    integer(c_int) function mhit_poisson(h, rhs, p) bind(C, name='mhit_poisson')
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: rhs(*)
      real(c_double), intent(out) :: p(*)
    end function

    integer(c_int) function mhit_destroy(h) bind(C, name='mhit_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function

    type(c_ptr) function mhit_strerror(status) bind(C, name='mhit_strerror')
      import :: c_int, c_ptr
      integer(c_int), value :: status
    end function
  end interface
end module mhit_iface
