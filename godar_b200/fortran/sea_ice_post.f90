! Optional drop-in replacement of sea_ice_post (model/src/diagnostics_outputs.f90:1-189)
! and clear_posts (model/src/diagnostics_ini_io.f90:1-100), same names and
! signatures, for builds that also use the replacement stepper.f90: the 25
! output files are written by libgodar_gpu.so straight from the device state
! of the stepper's context (sparse bond and contact lists instead of the n x n
! scans of bond, damageb and deltan), in the layout gfortran's list-directed
! WRITE gives them.  Link it in place of the two reference routines.
subroutine sea_ice_post (tstep, expno_str)

    use, intrinsic :: iso_c_binding
    use godar_gpu_mod

    implicit none

    include "parameter.h"
    include "CB_const.h"

    integer, intent(in) :: tstep
    character(len=4), intent(in) :: expno_str
    integer(c_int) :: st

    st = godar_gpu_write_posts(godar_shim_ctx, "output" // c_null_char, &
                               trim(adjustl(expno_str)) // c_null_char, int(tstep, c_int), &
                               real(comp, c_double))
    if (st /= GODAR_OK) then
        print *, "godar_gpu_write_posts error ", st
        stop 1
    end if

end subroutine sea_ice_post


subroutine clear_posts (expno_str)

    use, intrinsic :: iso_c_binding
    use godar_gpu_mod

    implicit none

    character(len=2), intent(in) :: expno_str
    integer(c_int) :: st

    st = godar_gpu_clear_posts("output" // c_null_char, trim(adjustl(expno_str)) // c_null_char)
    if (st /= GODAR_OK) then
        print *, "godar_gpu_clear_posts error ", st
        stop 1
    end if

end subroutine clear_posts
