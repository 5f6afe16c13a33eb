! Drop-in replacement of model/src/stepper.f90: same name and signature
! (`subroutine stepper (tstep, restart)`, called by godar.f90:193), same
! COMMON-block inputs and outputs, with the time step computed on the GPU by
! libgodar_gpu.so.  The state stays on the device between calls; it is read
! back into the COMMON blocks on output steps (the same condition as
! godar.f90:195), when sea_ice_post and gather_bonds_to_master read it.
!
! Link: add godar_gpu_mod.f90 to the sources and -L<dir> -lgodar_gpu to the
! executable (CMakeLists.txt: target_link_libraries(godar ... godar_gpu)).
subroutine stepper (tstep, restart)

    use, intrinsic :: iso_c_binding
    use godar_gpu_mod

    implicit none

    include "parameter.h"
    include "CB_variables.h"
    include "CB_const.h"
    include "CB_bond.h"
    include "CB_forcings.h"
    include "CB_options.h"
    include "CB_diagnostics.h"

    integer, intent(in) :: tstep, restart

    type(godar_params) :: p
    integer(c_int) :: st, cnt, k, nb
    integer :: i, j
    logical :: out_step
    integer(c_int32_t), allocatable :: bi(:), bj(:)
    real(c_double), allocatable :: dmg(:)

    if (.not. c_associated(godar_shim_ctx)) then
        p%dynamics = merge(1, 0, dynamics);   p%slipping = merge(1, 0, slipping)
        p%thermodyn = merge(1, 0, thermodyn); p%cohesion = merge(1, 0, cohesion)
        p%ridging = merge(1, 0, ridging);     p%shelter = merge(1, 0, shelter)
        p%rtree = rtree; p%ntree = ntree; p%dt = dt; p%nt = nt; p%comp = comp
        p%Cdair = Cdair; p%Csair = Csair; p%Cdwater = Cdwater; p%Cswater = Cswater
        p%z0w = z0w; p%lat = lat; p%rhoair = rhoair; p%rhoice = rhoice; p%rhowater = rhowater
        p%e_modul = e_modul; p%poiss_ratio = poiss_ratio; p%friction_coeff = friction_coeff
        p%rest_coeff = rest_coeff; p%sigmanc_crit = sigmanc_crit
        p%eb = eb; p%lambda_rb = lambda_rb; p%lambda_lb = lambda_lb
        p%sigmatb_crit = sigmatb_crit; p%sigmacb_crit = sigmacb_crit; p%tau_crit = tau_crit
        p%bond_lim = bond_lim; p%dmax = dmax; p%dtd = dtd; p%dth = dth
        p%uw = uw; p%vw = vw; p%ua = ua; p%va = va
        p%nx = nx; p%ny = ny
        p%boundary = 0; p%bond_seed = 0; p%bond_lim_rel = 0d0; p%bond_frac = 0d0
        p%field_nx = 0; p%field_ny = 0
        st = godar_gpu_derive_params(p)
        st = godar_gpu_create(p, int(n, c_int), GODAR_PREC_FP64, godar_shim_ctx)
        call check(st)
        ! restart bonds and damage read by ini_get (ini_get.f90:129-130)
        nb = count(bond == 1)
        allocate(bi(max(nb, 1)), bj(max(nb, 1)), dmg(max(nb, 1)))
        k = 0
        do i = 1, n
            do j = i + 1, n
                if (bond(j, i) == 1) then
                    k = k + 1
                    bi(k) = i - 1; bj(k) = j - 1; dmg(k) = damageb(j, i)
                end if
            end do
        end do
        st = godar_gpu_upload(godar_shim_ctx, x, y, r, h, theta, omega, u, v, int(nb, c_int), bi, bj, dmg)
        call check(st)
        deallocate(bi, bj, dmg)
    end if

    ! the diagnostics (forces, moments, stresses, the contact list) are read
    ! on output steps only (godar.f90:195-203); the other steps skip them,
    ! which leaves the state and the next output step's diagnostics the same
    out_step = modulo(tstep, int(comp)) .eq. 0 .or. tstep + restart == 1
    call check(godar_gpu_set_diagnostics(godar_shim_ctx, merge(1_c_int, 0_c_int, out_step)))

    ! queued: the step runs while the time loop comes back for the next one;
    ! the downloads of an output step wait for it, and an error of a queued
    ! step is returned by the next call
    st = godar_gpu_step_async(godar_shim_ctx, int(tstep, c_int), int(restart, c_int), 1_c_int)
    call check(st)

    if (out_step) then
        call get(GODAR_F_X, x); call get(GODAR_F_Y, y); call get(GODAR_F_U, u); call get(GODAR_F_V, v)
        call get(GODAR_F_R, r); call get(GODAR_F_H, h); call get(GODAR_F_THETA, theta)
        call get(GODAR_F_OMEGA, omega); call get(GODAR_F_TFX, tfx); call get(GODAR_F_TFY, tfy)
        call get(GODAR_F_FCX, fcx); call get(GODAR_F_FCY, fcy); call get(GODAR_F_FBX, fbx)
        call get(GODAR_F_FBY, fby); call get(GODAR_F_M, m); call get(GODAR_F_MC, mc)
        call get(GODAR_F_MB, mb); call get(GODAR_F_TSIGXX, tsigxx); call get(GODAR_F_TSIGYY, tsigyy)
        call get(GODAR_F_TSIGXY, tsigxy); call get(GODAR_F_TSIGYX, tsigyx); call get(GODAR_F_TP, tp)
        ! bond/damage/contact lists scattered into the dense arrays that
        ! sea_ice_post writes (diagnostics_outputs.f90:157-167)
        bond = 0
        deltan = 0d0
        call scatter(GODAR_P_BONDS)
        call scatter(GODAR_P_CONTACTS)
    end if

contains

    subroutine check(s)
        integer(c_int), intent(in) :: s
        if (s /= GODAR_OK) then
            print *, "godar_gpu error ", s
            stop 1
        end if
    end subroutine

    subroutine get(f, arr)
        integer(c_int), intent(in) :: f
        double precision, intent(out) :: arr(n)
        call check(godar_gpu_get_floe_field(godar_shim_ctx, f, arr))
    end subroutine

    subroutine scatter(which)
        integer(c_int), intent(in) :: which
        integer(c_int32_t), allocatable :: pi(:), pj(:)
        real(c_double), allocatable :: val(:)
        integer(c_int) :: c, q
        integer(c_int32_t) :: d1(1), d2(1)
        real(c_double) :: d3(1)
        call check(godar_gpu_get_pairs(godar_shim_ctx, which, d1, d2, d3, 0_c_int, c))
        allocate(pi(max(c, 1)), pj(max(c, 1)), val(max(c, 1)))
        call check(godar_gpu_get_pairs(godar_shim_ctx, which, pi, pj, val, c, c))
        do q = 1, c
            if (which == GODAR_P_BONDS) then
                bond(pj(q) + 1, pi(q) + 1) = 1
                damageb(pj(q) + 1, pi(q) + 1) = val(q)
            else
                deltan(pj(q) + 1, pi(q) + 1) = val(q)
            end if
        end do
        deallocate(pi, pj, val)
    end subroutine

end subroutine stepper
