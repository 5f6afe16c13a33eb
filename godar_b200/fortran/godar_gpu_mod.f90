! ISO_C_BINDING interface to libgodar_gpu.so (include/godar_gpu.h).
!
! The type godar_params mirrors the C struct field by field; logicals are
! integer(c_int32_t) 0/1.  Every function returns a GODAR_* status (0 = OK).
! Floe arrays are passed as contiguous double precision arrays of length n
! (the COMMON-block arrays of CB_variables.h are contiguous already).
module godar_gpu_mod
    use, intrinsic :: iso_c_binding
    implicit none

    integer(c_int), parameter :: GODAR_OK = 0
    integer(c_int), parameter :: GODAR_PREC_FP64 = 0, GODAR_PREC_MIXED = 1
    integer(c_int), parameter :: GODAR_F_X = 0, GODAR_F_Y = 1, GODAR_F_U = 2, GODAR_F_V = 3, &
        GODAR_F_R = 4, GODAR_F_H = 5, GODAR_F_THETA = 6, GODAR_F_OMEGA = 7, GODAR_F_TFX = 8, &
        GODAR_F_TFY = 9, GODAR_F_FCX = 10, GODAR_F_FCY = 11, GODAR_F_FBX = 12, GODAR_F_FBY = 13, &
        GODAR_F_M = 14, GODAR_F_MC = 15, GODAR_F_MB = 16, GODAR_F_TSIGXX = 17, GODAR_F_TSIGYY = 18, &
        GODAR_F_TSIGXY = 19, GODAR_F_TSIGYX = 20, GODAR_F_TP = 21
    integer(c_int), parameter :: GODAR_P_CANDIDATES = 0, GODAR_P_CONTACTS = 1, GODAR_P_BONDS = 2

    ! the context of the replacement stepper, shared with the replacement
    ! sea_ice_post (godar_b200/fortran/sea_ice_post.f90)
    type(c_ptr), save :: godar_shim_ctx = c_null_ptr

    type, bind(C) :: godar_params
        integer(c_int32_t) :: dynamics, slipping, thermodyn, cohesion, ridging, shelter
        real(c_double) :: rtree, ntree, dt, nt, comp
        real(c_double) :: Cdair, Csair, Cdwater, Cswater, z0w, lat, rhoair, rhoice, rhowater
        real(c_double) :: e_modul, poiss_ratio, friction_coeff, rest_coeff, sigmanc_crit
        real(c_double) :: eb, lambda_rb, lambda_lb, sigmatb_crit, sigmacb_crit, tau_crit, &
                          bond_lim, dmax, dtd, dth
        real(c_double) :: uw, vw, ua, va
        real(c_double) :: nx, ny
        real(c_double) :: ec, gc, beta, pi, sin_lat
        integer(c_int32_t) :: boundary, bond_seed
        real(c_double) :: bond_lim_rel, bond_frac
        integer(c_int32_t) :: field_nx, field_ny
    end type godar_params

    interface
        function godar_gpu_derive_params(p) bind(C, name="godar_gpu_derive_params") result(st)
            import :: godar_params, c_int
            type(godar_params), intent(inout) :: p
            integer(c_int) :: st
        end function

        function godar_gpu_create(p, n, precision, ctx) bind(C, name="godar_gpu_create") result(st)
            import :: godar_params, c_int, c_ptr
            type(godar_params), intent(in) :: p
            integer(c_int), value :: n, precision
            type(c_ptr), intent(out) :: ctx
            integer(c_int) :: st
        end function

        function godar_gpu_upload(ctx, x, y, r, h, theta, omega, u, v, nb, bi, bj, damage) &
                bind(C, name="godar_gpu_upload") result(st)
            import :: c_ptr, c_int, c_double, c_int32_t
            type(c_ptr), value :: ctx
            real(c_double), intent(in) :: x(*), y(*), r(*), h(*), theta(*), omega(*), u(*), v(*)
            integer(c_int), value :: nb
            integer(c_int32_t), intent(in) :: bi(*), bj(*)
            real(c_double), intent(in) :: damage(*)
            integer(c_int) :: st
        end function

        function godar_gpu_step(ctx, tstep, restart, nsteps) bind(C, name="godar_gpu_step") result(st)
            import :: c_ptr, c_int
            type(c_ptr), value :: ctx
            integer(c_int), value :: tstep, restart, nsteps
            integer(c_int) :: st
        end function

        ! the same steps queued without waiting; errors come back from the
        ! next call on the context
        function godar_gpu_step_async(ctx, tstep, restart, nsteps) bind(C, name="godar_gpu_step_async") result(st)
            import :: c_ptr, c_int
            type(c_ptr), value :: ctx
            integer(c_int), value :: tstep, restart, nsteps
            integer(c_int) :: st
        end function

        function godar_gpu_get_floe_field(ctx, field, out) bind(C, name="godar_gpu_get_floe_field") result(st)
            import :: c_ptr, c_int, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: field
            real(c_double), intent(out) :: out(*)
            integer(c_int) :: st
        end function

        function godar_gpu_get_pairs(ctx, which, pi, pj, val, cap, count) bind(C, name="godar_gpu_get_pairs") result(st)
            import :: c_ptr, c_int, c_double, c_int32_t
            type(c_ptr), value :: ctx
            integer(c_int), value :: which, cap
            integer(c_int32_t), intent(out) :: pi(*), pj(*)
            real(c_double), intent(out) :: val(*)
            integer(c_int), intent(out) :: count
            integer(c_int) :: st
        end function

        ! floe_out: GODAR_F_COUNT addresses (c_loc of each output array, or
        ! c_null_ptr to skip it); which < 0: no pair list
        function godar_gpu_download(ctx, floe_out, which, pi, pj, val, cap, count) &
                bind(C, name="godar_gpu_download") result(st)
            import :: c_ptr, c_int, c_double, c_int32_t
            type(c_ptr), value :: ctx
            type(c_ptr), intent(in) :: floe_out(*)
            integer(c_int), value :: which, cap
            integer(c_int32_t), intent(out) :: pi(*), pj(*)
            real(c_double), intent(out) :: val(*)
            integer(c_int), intent(out) :: count
            integer(c_int) :: st
        end function

        function godar_gpu_set_precision(ctx, mode) bind(C, name="godar_gpu_set_precision") result(st)
            import :: c_ptr, c_int
            type(c_ptr), value :: ctx
            integer(c_int), value :: mode
            integer(c_int) :: st
        end function

        ! on = 0: step calls skip the diagnostics (forces, moments, stresses,
        ! pressure, the contact list), which keep the values of the last
        ! diagnostic step; the state advances identically.  On by default.
        function godar_gpu_set_diagnostics(ctx, on) bind(C, name="godar_gpu_set_diagnostics") result(st)
            import :: c_ptr, c_int
            type(c_ptr), value :: ctx
            integer(c_int), value :: on
            integer(c_int) :: st
        end function

        ! sea_ice_post: appends one output step to the 25 text files
        ! "<dir>/<name>.<expno>"; dir and expno are NUL-terminated, e.g.
        ! "output" // c_null_char and trim(expno_str) // c_null_char
        function godar_gpu_write_posts(ctx, dir, expno, tstep, comp) &
                bind(C, name="godar_gpu_write_posts") result(st)
            import :: c_ptr, c_int, c_double, c_char
            type(c_ptr), value :: ctx
            character(kind=c_char), intent(in) :: dir(*), expno(*)
            integer(c_int), value :: tstep
            real(c_double), value :: comp
            integer(c_int) :: st
        end function

        ! clear_posts: deletes the output files of experiment expno
        function godar_gpu_clear_posts(dir, expno) bind(C, name="godar_gpu_clear_posts") result(st)
            import :: c_int, c_char
            character(kind=c_char), intent(in) :: dir(*), expno(*)
            integer(c_int) :: st
        end function

        ! buf = c_null_ptr: only bytes is set
        function godar_gpu_checkpoint(ctx, buf, cap, bytes) bind(C, name="godar_gpu_checkpoint") result(st)
            import :: c_ptr, c_int, c_size_t
            type(c_ptr), value :: ctx, buf
            integer(c_size_t), value :: cap
            integer(c_size_t), intent(out) :: bytes
            integer(c_int) :: st
        end function

        function godar_gpu_restore(ctx, buf, bytes) bind(C, name="godar_gpu_restore") result(st)
            import :: c_ptr, c_int, c_size_t
            type(c_ptr), value :: ctx, buf
            integer(c_size_t), value :: bytes
            integer(c_int) :: st
        end function

        function godar_gpu_last_error() bind(C, name="godar_gpu_last_error") result(msg)
            import :: c_ptr
            type(c_ptr) :: msg
        end function

        subroutine godar_gpu_destroy(ctx) bind(C, name="godar_gpu_destroy")
            import :: c_ptr
            type(c_ptr), value :: ctx
        end subroutine
    end interface
end module godar_gpu_mod
