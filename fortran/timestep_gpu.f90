! timestep_gpu.f90 -- drop-in replacement of timestep.o for the reference (ankitvb/solar):
! SUBROUTINE RK4 (timestep.f90:41-86) runs on the GPU through libsolar_gpu.so.  In the
! makefile (makefile:14-18) put timestep_gpu.o and solar_gpu_bind.o in OBJS in place of
! timestep.o and link -L<repo>/solar_b200 -lsolar_gpu.  COMPUTE_TIMESTEP is kept from
! timestep.f90 unchanged (it only sets deltat).
!
! One process drives all six zones: SOLAR_GPU_SETUP is called once after GENERATE_IC
! (cube.f90:47) with the six zones' q(mx,my,mr,5) arrays concatenated in zone order and the
! solar_model rows that SOLAR_DATA read (nr x 8, row-major).  Each RK4 call is then five
! 2N-storage stages of COMPUTE_RHS + BC_RHS + SPONGE + update and FILTER_EXP on the GPU,
! and the host's time advances as in timestep.f90:82.  SOLAR_GPU_FETCH copies the state back
! into the host arrays before the reference writes its output files (cube.f90:85-88).

SUBROUTINE SOLAR_GPU_SETUP(q6, model, nx_, nr_, dt_)
  USE solar_gpu_bind
  implicit none
  integer, intent(in) :: nx_, nr_
  real*8, intent(in), target :: q6(*), model(*)
  real*8, intent(in) :: dt_
  type(solar_desc) :: d
  call solar_desc_defaults(d)
  d%nx = nx_
  d%nr = nr_
  d%dt = dt_
  d%model = c_loc(model(1))
  call solar_check(solar_gpu_init(d, solar_ctx), 'solar_gpu_init')
  call solar_check(solar_gpu_set_state(solar_ctx, 0_c_int, q6), 'solar_gpu_set_state')
END SUBROUTINE SOLAR_GPU_SETUP

SUBROUTINE RK4
  USE INIT
  USE solar_gpu_bind
  implicit none
  call solar_check(solar_gpu_rk4(solar_ctx, 1_c_int), 'solar_gpu_rk4')
  time = time + deltat
  return
END SUBROUTINE RK4

SUBROUTINE SOLAR_GPU_FETCH(q6)
  USE solar_gpu_bind
  implicit none
  real*8, intent(out) :: q6(*)
  call solar_check(solar_gpu_get_state(solar_ctx, 0_c_int, q6), 'solar_gpu_get_state')
END SUBROUTINE SOLAR_GPU_FETCH

SUBROUTINE SOLAR_GPU_NORM(field, tt)
  USE solar_gpu_bind
  implicit none
  integer, intent(in) :: field
  real*8, intent(out) :: tt
  call solar_check(solar_gpu_norm(solar_ctx, 0_c_int, int(field, c_int), tt), 'solar_gpu_norm')
END SUBROUTINE SOLAR_GPU_NORM
