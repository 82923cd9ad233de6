! solar_gpu_bind.f90 -- Fortran 2003 (ISO_C_BINDING) interface to libsolar_gpu.so, the C-ABI
! of include/solar_gpu.h.  This is the binding a maintainer adds to the reference's Fortran
! driver (cube.f90) so that its RK4 call (cube.f90:74) runs on the GPU; timestep_gpu.f90 is
! the drop-in RK4 built on it.  Build (where a Fortran compiler exists):
!     gfortran -c solar_gpu_bind.f90
!     ... link with -L<repo>/solar_b200 -lsolar_gpu
!
! The derived type solar_desc mirrors struct solar_desc field for field (same order, C
! interoperable kinds); tests/test_fortran_binding.py checks that order against the C
! header's offsets.  Arrays use the header's "six-zone Fortran order": the reference's
! per-zone q(mx,my,mr,5) arrays of zones 1..6 one after another.
module solar_gpu_bind
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: SOLAR_OK = 0
  integer(c_int), parameter :: SOLAR_ERR_ARG = -1, SOLAR_ERR_CUDA = -2, SOLAR_ERR_NAN = -3
  integer(c_int), parameter :: SOLAR_ERR_TIMEOUT = -4, SOLAR_ERR_STATE = -5, SOLAR_ERR_NOMEM = -6
  integer(c_int), parameter :: SOLAR_FP64 = 0, SOLAR_FP32 = 1

  type, bind(C) :: solar_desc
    integer(c_int) :: nx
    integer(c_int) :: nr
    integer(c_int) :: precision
    integer(c_int) :: nfields
    integer(c_int) :: nruns
    integer(c_int) :: device
    real(c_double) :: dt
    type(c_ptr)    :: model
    type(c_ptr)    :: c2_3d
    real(c_double) :: sponge_amp
    real(c_double) :: sponge_exp
    integer(c_int) :: sponge_len
    integer(c_int) :: sponge_lower
    integer(c_int) :: sponge_upper
    integer(c_int) :: fix_reversed_rotation
    integer(c_int) :: tile_x
    integer(c_int) :: tile_y
    integer(c_int) :: kchunk
  end type solar_desc

  ! The one GPU context of the process (one host process drives all six zones).
  type(c_ptr), save :: solar_ctx = c_null_ptr

  interface
    subroutine solar_desc_defaults(d) bind(C, name="solar_desc_defaults")
      import :: solar_desc
      type(solar_desc), intent(inout) :: d
    end subroutine

    integer(c_int) function solar_gpu_init(d, ctx) bind(C, name="solar_gpu_init")
      import :: solar_desc, c_int, c_ptr
      type(solar_desc), intent(in) :: d
      type(c_ptr), intent(out) :: ctx
    end function

    integer(c_int) function solar_gpu_finalize(ctx) bind(C, name="solar_gpu_finalize")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    integer(c_int) function solar_gpu_set_state(ctx, run, q) bind(C, name="solar_gpu_set_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: run
      real(c_double), intent(in) :: q(*)
    end function

    integer(c_int) function solar_gpu_get_state(ctx, run, q) bind(C, name="solar_gpu_get_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: run
      real(c_double), intent(out) :: q(*)
    end function

    integer(c_int) function solar_gpu_rk4(ctx, nsteps) bind(C, name="solar_gpu_rk4")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
    end function

    integer(c_int) function solar_gpu_rk4_norms(ctx, run, field, nsteps, norms) bind(C, name="solar_gpu_rk4_norms")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: run, field, nsteps
      real(c_double), intent(out) :: norms(*)
    end function

    integer(c_int) function solar_gpu_compute_rhs(ctx, q, rhs) bind(C, name="solar_gpu_compute_rhs")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: q(*)
      real(c_double), intent(out) :: rhs(*)
    end function

    integer(c_int) function solar_gpu_bc_rhs(ctx, rhs) bind(C, name="solar_gpu_bc_rhs")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: rhs(*)
    end function

    integer(c_int) function solar_gpu_sponge(ctx, q, rhs) bind(C, name="solar_gpu_sponge")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: q(*)
      real(c_double), intent(inout) :: rhs(*)
    end function

    integer(c_int) function solar_gpu_filter_exp(ctx, q, qf) bind(C, name="solar_gpu_filter_exp")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: q(*)
      real(c_double), intent(out) :: qf(*)
    end function

    integer(c_int) function solar_gpu_norm(ctx, run, field, out) bind(C, name="solar_gpu_norm")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: run, field
      real(c_double), intent(out) :: out
    end function

    integer(c_int) function solar_gpu_diag(ctx, run, out4) bind(C, name="solar_gpu_diag")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: run
      real(c_double), intent(out) :: out4(4)
    end function

    integer(c_int) function solar_gpu_set_watchdog(ctx, every) bind(C, name="solar_gpu_set_watchdog")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: every
    end function

    integer(c_int) function solar_gpu_write_visual(ctx, run, dir, cue) bind(C, name="solar_gpu_write_visual")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      integer(c_int), value :: run, cue
      character(kind=c_char), intent(in) :: dir(*)
    end function

    integer(c_int) function solar_gpu_last_error(buf, len) bind(C, name="solar_gpu_last_error")
      import :: c_int, c_char
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int), value :: len
    end function
  end interface

contains

  ! The reference's error convention: report and stop (init_mpi.f90:31, output.f90:137).
  subroutine solar_check(ierr, what)
    integer(c_int), intent(in) :: ierr
    character(len=*), intent(in) :: what
    character(kind=c_char) :: buf(512)
    character(len=512) :: msg
    integer :: i, rc
    if (ierr == SOLAR_OK) return
    rc = solar_gpu_last_error(buf, 512_c_int)
    msg = ' '
    do i = 1, 512
      if (buf(i) == c_null_char) exit
      msg(i:i) = buf(i)
    end do
    print *, what, ' failed with status ', ierr, ': ', trim(msg)
    stop 1
  end subroutine solar_check

end module solar_gpu_bind
