! Thin Fortran driver: the reference's program main (multi/main.f90) with the
! loop body replaced by libmhit.  Initialisation and I/O stay in Fortran:
! input.inp is read as multi/readinput.f90 reads it, the module-shaped arrays
! (nx, ny+2, nz+2) are filled from Taylor-Green / input/*.dat, and the fields
! go to output/*_%08d.dat every `dump` steps through mhit_save.
!
! Build (on a machine with a Fortran compiler):
!   gfortran -O2 mhit_iface.f90 mhit_driver.f90 -L../mhit36_b200/_lib -lmhit -o mhit36_b200
! Not compiled in this image (no Fortran compiler); see mhit_iface.f90.
program mhit_driver
  use iso_c_binding
  use mhit_iface
  implicit none
  integer, parameter :: nx = 128
  integer :: ny = nx, nz = nx
  type(mhit_params) :: prm
  type(mhit_diag) :: diag
  type(c_ptr) :: h
  integer(c_int) :: rc
  real(c_double), allocatable :: u(:,:,:), v(:,:,:), w(:,:,:), phi(:,:,:)
  real(c_double) :: dx, twopi, pos, eps
  real(c_double), allocatable :: x(:)
  integer :: i, j, k, t

  call mhit_default_params(prm)
  open(unit=55, file='input.inp', form='formatted', status='old')
  read(55,*) prm%restart
  read(55,*) prm%tstart
  read(55,*) prm%tfin
  read(55,*) prm%dump
  read(55,*) prm%inflow
  read(55,*) prm%inphi
  read(55,*) prm%dt
  read(55,*) prm%mu
  read(55,*) prm%rho
  read(55,*) prm%f1
  read(55,*) prm%f2
  read(55,*) prm%f3
  read(55,*) prm%k0
  read(55,*) prm%radius
  read(55,*) prm%sigma
  read(55,*) prm%epsr
  read(55,*,iostat=i) prm%lin_force   ! optional 17th line
  if (i /= 0) prm%lin_force = 0.0d0
  close(55)

  allocate(u(nx,ny+2,nz+2), v(nx,ny+2,nz+2), w(nx,ny+2,nz+2), phi(nx,ny+2,nz+2), x(nx))
  twopi = 8.0d0*atan(1.0d0)
  dx = twopi/(nx-1)
  eps = prm%epsr*dx
  x(1) = 0.0d0
  do i = 2, nx
    x(i) = x(i-1) + dx
  enddo

  rc = mhit_create(prm, nx, ny, nz, MHIT_FP64, 1, h)
  if (rc /= MHIT_OK) stop 'mhit_create failed'

  if (prm%restart == 0) then
    if (prm%inflow == 0) then
      do k = 2, nz+1
        do j = 2, ny+1
          do i = 1, nx
            u(i,j,k) =  sin(x(i))*cos(x(j-1))*cos(x(k-1))
            v(i,j,k) = -cos(x(i))*sin(x(j-1))*cos(x(k-1))
            w(i,j,k) =  0.0d0
          enddo
        enddo
      enddo
    else
      call read_raw('./input/u.dat', u)
      call read_raw('./input/v.dat', v)
      call read_raw('./input/w.dat', w)
    endif
    if (prm%inphi == 0) then
      do k = 2, nz+1
        do j = 2, ny+1
          do i = 1, nx
            pos = (x(i)-twopi/2)**2 + (x(j-1)-twopi/2)**2 + (x(k-1)-twopi/2)**2
            phi(i,j,k) = 0.5d0*(1.d0-tanh((sqrt(pos)-prm%radius)/2/eps))
          enddo
        enddo
      enddo
    else
      call read_raw('./input/phi.dat', phi)
    endif
    rc = mhit_set_fields(h, u, v, w, phi, MHIT_LAYOUT_PIX_HALO)
    if (rc /= MHIT_OK) stop 'mhit_set_fields failed'
    rc = mhit_save(h, './output'//c_null_char, prm%tstart)
  else
    rc = mhit_load(h, './output'//c_null_char, prm%tstart)
    if (rc /= MHIT_OK) stop 'mhit_load failed'
  endif

  do t = prm%tstart+1, prm%tfin
    write(*,*) "Time step", t, "of", prm%tfin
    rc = mhit_step(h, 1, diag)
    write(*,*) "CFL (max among tasks)", diag%cfl
    if (rc == MHIT_ERR_CFL) exit
    if (rc /= MHIT_OK) stop 'mhit_step failed'
    if (mod(t, prm%dump) == 0) rc = mhit_save(h, './output'//c_null_char, t)
  enddo
  rc = mhit_destroy(h)

contains

  subroutine read_raw(fname, a)
    character(len=*), intent(in) :: fname
    real(c_double), intent(inout) :: a(:,:,:)
    real(c_double), allocatable :: tmp(:,:,:)
    allocate(tmp(nx,ny,nz))
    open(66, file=fname, form='unformatted', access='stream', status='old', convert='little_endian')
    read(66) tmp
    close(66)
    a(1:nx, 2:ny+1, 2:nz+1) = tmp
    deallocate(tmp)
  end subroutine read_raw
end program mhit_driver
