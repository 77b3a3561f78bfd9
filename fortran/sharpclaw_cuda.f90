! sharpclaw_cuda.f90 -- the Fortran side of the B200 SharpClaw step.
!
! Drop-in replacements for the reference's hot-path routines, with the
! reference's names and argument lists, forwarding through iso_c_binding to
! the C ABI of include/sharpclaw_cuda.h (library libsharpclaw_b200.so):
!
!   flux1      src/flux1.f90:2                          -> scl_flux1
!   flux2      src/2d/flux2.f90:2                       -> scl_step_dq (2-D)
!   step       src/1d/step1d.f90:2, src/2d/step2d.f90:2 -> scl_step_dq
!   sharpclaw  src/sharpclaw.f90:2 (called at main.f90:192) -> scl_sharpclaw
!
! An app links this file in place of flux1.o, flux2.o, step1d.o / step2d.o,
! sharpclaw.o and reconstruct.o, and keeps its own main.f90, qinit, setaux
! and setprob.  The externals rp, tfluct, src, bc and b4step stay in the
! argument lists and are not called: device code cannot call a Fortran
! procedure, so the device plugins (Riemann solver, tfluct, eigenvectors,
! source and b4step hooks) are chosen by id once, by a call of
! sharpclaw_cuda_setup from the app's setprob, where its COMMON-block
! constants (/comrp/ u or grav, /param/ gamma, ...) are known.
!
! Errors: every entry point of the library returns a status; a non-zero one
! is reported with the library's message and ends the run with `stop`, as the
! reference's own error paths do.
module sharpclaw_cuda
    use iso_c_binding
    implicit none

    ! ---- status codes and ids (include/sharpclaw_cuda.h) ----------------
    integer(c_int), parameter :: SCL_OK = 0, SCL_E_INVALID = -1, SCL_E_CUDA = -2, SCL_E_UNSUPPORTED = -3, &
                                 SCL_E_NONFINITE = -4, SCL_E_TIMEOUT = -5, SCL_E_IO = -6
    integer(c_int), parameter :: SCL_FP64 = 0, SCL_FP64_STRICT = 1, SCL_MIXED = 2, SCL_FP32 = 3
    integer(c_int), parameter :: SCL_RP_ADVECTION = 1, SCL_RP_EULER = 2, SCL_RP_SW2D = 3, &
                                 SCL_RP_ACOUSTICS1D = 4, SCL_RP_ACOUSTICS2D = 5, SCL_RP_ADVECTION2D = 6, &
                                 SCL_RP_SW1D = 7, SCL_RP_SWF_BATHY = 8, SCL_RP_SWF_RADIAL = 9, &
                                 SCL_RP_SWF_KAPPA = 10, SCL_RP_ACOUSTICS_CONST = 11, SCL_RP_ACOUSTICS_FWAVE = 12, &
                                 SCL_RP_TRAFFIC = 13, SCL_RP_ADVECTION_CONS = 14, SCL_RP_STEGOTON = 15
    integer(c_int), parameter :: SCL_SRC_NONE = 0, SCL_SRC_RADIAL_SW = 1, SCL_SRC_BATHYMETRY_SW = 2
    integer(c_int), parameter :: SCL_B4STEP_NONE = 0, SCL_B4STEP_SWIRL = 1, SCL_B4STEP_TIME_REVERSAL = 2
    integer(c_int), parameter :: SCL_BC_USER_NONE = 0, SCL_BC_USER_OSCILLATING_WALL = 1
    integer(c_int), parameter :: SCL_INFO_NONFINITE = 20

    ! ---- the C structs, field for field ---------------------------------
    type, bind(C) :: scl_params
        integer(c_int) :: ndim, mx, my, meqn, mwaves, mbc, maux, mcapa
        integer(c_int) :: lim_type, char_decomp, tfluct_solver
        integer(c_int) :: mthbc(4)
        real(c_double) :: dx, dy, xlower, ylower
        integer(c_int) :: rp, efix
        real(c_double) :: u, gamma, grav
        integer(c_int) :: time_integrator, precision
        integer(c_int) :: mthlim(4)
        integer(c_int) :: src_term
        real(c_double) :: rho, bulk
        integer(c_int) :: bc_user
        real(c_double) :: wall(6)
    end type scl_params

    type, bind(C) :: scl_run
        real(c_double) :: tstart, tend, dt_initial, dt_max, cfl_max, cfl_desired
        integer(c_int) :: max_steps, dt_variable
    end type scl_run

    type, bind(C) :: scl_result
        real(c_double) :: tend, cfl_maxused, cfl_last, dt_minused, dt_maxused, dt_last
        integer(c_int) :: steps_taken, info, rejected, status
    end type scl_result

    ! ---- entry points ---------------------------------------------------
    interface
        type(c_ptr) function scl_last_error() bind(C, name="scl_last_error")
            import :: c_ptr
        end function scl_last_error
        integer(c_int) function scl_create(p, h) bind(C, name="scl_create")
            import :: c_int, c_ptr, scl_params
            type(scl_params), intent(in) :: p
            type(c_ptr), intent(out) :: h
        end function scl_create
        integer(c_int) function scl_destroy(h) bind(C, name="scl_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function scl_destroy
        integer(c_int) function scl_set_q(h, q) bind(C, name="scl_set_q")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: q(*)
        end function scl_set_q
        integer(c_int) function scl_get_q(h, q) bind(C, name="scl_get_q")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: q(*)
        end function scl_get_q
        integer(c_int) function scl_set_aux(h, aux) bind(C, name="scl_set_aux")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: aux(*)
        end function scl_set_aux
        integer(c_int) function scl_step_dq(h, q, dq, dt, t, cfl) bind(C, name="scl_step_dq")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(inout) :: q(*)
            real(c_double), intent(out) :: dq(*)
            real(c_double), value :: dt, t
            real(c_double), intent(out) :: cfl
        end function scl_step_dq
        integer(c_int) function scl_flux1(h, q1d, aux1d, dq1d, dt, ixy, mx, cfl) bind(C, name="scl_flux1")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: q1d(*), aux1d(*)
            real(c_double), intent(out) :: dq1d(*)
            real(c_double), value :: dt
            integer(c_int), value :: ixy, mx
            real(c_double), intent(out) :: cfl
        end function scl_flux1
        integer(c_int) function scl_rk_step(h, dt, told, cfl) bind(C, name="scl_rk_step")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), value :: dt, told
            real(c_double), intent(out) :: cfl
        end function scl_rk_step
        integer(c_int) function scl_sharpclaw(h, run, res) bind(C, name="scl_sharpclaw")
            import :: c_int, c_ptr, scl_run, scl_result
            type(c_ptr), value :: h
            type(scl_run), intent(in) :: run
            type(scl_result), intent(out) :: res
        end function scl_sharpclaw
        integer(c_int) function scl_set_b4step(h, kind, param) bind(C, name="scl_set_b4step")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: kind
            real(c_double), value :: param
        end function scl_set_b4step
        integer(c_int) function scl_rk_step_noalloc(p, q_dev, aux_dev, dt, cfl, stream) &
                bind(C, name="scl_rk_step_noalloc")
            import :: c_int, c_ptr, c_double, scl_params
            type(scl_params), intent(in) :: p
            type(c_ptr), value :: q_dev, aux_dev
            real(c_double), value :: dt
            real(c_double), intent(out) :: cfl
            type(c_ptr), value :: stream
        end function scl_rk_step_noalloc
    end interface

    ! ---- the run's device handle and its plugin choice -------------------
    type(c_ptr), save :: scl_h = c_null_ptr
    type(scl_params), save :: scl_p
    logical, save :: scl_configured = .false.
    integer(c_int), save :: cfg_rp = 0, cfg_precision = SCL_FP64, cfg_efix = -1, cfg_src = SCL_SRC_NONE
    integer(c_int), save :: cfg_b4step = SCL_B4STEP_NONE, cfg_bc_user = SCL_BC_USER_NONE
    real(c_double), save :: cfg_u = 1.d0, cfg_gamma = 1.4d0, cfg_grav = 1.d0, cfg_rho = 1.d0, cfg_bulk = 1.d0
    real(c_double), save :: cfg_b4param = 0.d0, cfg_wall(6) = 0.d0

contains

    ! Choose the device plugin and its constants; call once, e.g. from the
    ! app's setprob after it has read setprob.data.  efix < 0 keeps the
    ! plugin's default (rp1eu.f:40 and rp1sw.f: on; rpn2sw.f:48: off).
    subroutine sharpclaw_cuda_setup(rp, precision, u, gamma, grav, efix, src_term, rho, bulk, &
                                    b4step_kind, b4step_param, bc_user, wall)
        integer, intent(in) :: rp, precision
        double precision, intent(in), optional :: u, gamma, grav, rho, bulk, b4step_param
        integer, intent(in), optional :: efix, src_term, b4step_kind, bc_user
        double precision, intent(in), optional :: wall(6)
        cfg_rp = int(rp, c_int)
        cfg_precision = int(precision, c_int)
        if (present(u)) cfg_u = u
        if (present(gamma)) cfg_gamma = gamma
        if (present(grav)) cfg_grav = grav
        if (present(efix)) cfg_efix = int(efix, c_int)
        if (present(src_term)) cfg_src = int(src_term, c_int)
        if (present(rho)) cfg_rho = rho
        if (present(bulk)) cfg_bulk = bulk
        if (present(b4step_kind)) cfg_b4step = int(b4step_kind, c_int)
        if (present(b4step_param)) cfg_b4param = b4step_param
        if (present(bc_user)) cfg_bc_user = int(bc_user, c_int)
        if (present(wall)) cfg_wall = wall
        scl_configured = .true.
        call sharpclaw_cuda_release()
    end subroutine sharpclaw_cuda_setup

    ! Destroy the device handle (a later call creates a new one).
    subroutine sharpclaw_cuda_release()
        integer(c_int) :: ierr
        if (c_associated(scl_h)) then
            ierr = scl_destroy(scl_h)
            scl_h = c_null_ptr
        end if
    end subroutine sharpclaw_cuda_release

    ! The library's message for the last failed call of this thread.
    function scl_error_message() result(msg)
        character(len=512) :: msg
        character(kind=c_char), pointer :: cs(:)
        type(c_ptr) :: p
        integer :: k
        msg = ' '
        p = scl_last_error()
        if (.not. c_associated(p)) return
        call c_f_pointer(p, cs, [len(msg)])
        do k = 1, len(msg)
            if (cs(k) == c_null_char) exit
            msg(k:k) = cs(k)
        end do
    end function scl_error_message

    ! Report a failed call as the reference reports its errors, then stop.
    subroutine scl_stop(where, ierr)
        character(len=*), intent(in) :: where
        integer(c_int), intent(in) :: ierr
        write(6,*) '*** ERROR in ', where, ' (sharpclaw_cuda status ', ierr, '): ', trim(scl_error_message())
        stop
    end subroutine scl_stop

    ! The device handle of the run described by module ClawParams
    ! (src/ClawParams.f90) with the integrator ti (0: keep the handle's, or
    ! SSPRK(3,3) for a new one).  Made on first use, and again when the grid
    ! or the integrator changes; aux (module Global) is uploaded with it.
    function scl_handle_for(ti) result(h)
        use ClawParams
        use Global, only: aux
        integer, intent(in) :: ti
        type(c_ptr) :: h
        type(scl_params) :: p
        integer(c_int) :: ierr
        integer :: k
        if (.not. scl_configured) then
            write(6,*) '*** ERROR: sharpclaw_cuda_setup must be called (from setprob) before the first step'
            stop
        end if
        p%ndim = int(ndim, c_int)
        p%mx = int(nx(1), c_int)
        p%my = 1
        if (ndim > 1) p%my = int(nx(2), c_int)
        p%meqn = int(meqn, c_int)
        p%mwaves = int(mwaves, c_int)
        p%mbc = int(mbc, c_int)
        p%maux = int(maux, c_int)
        p%mcapa = int(mcapa, c_int)
        p%lim_type = int(lim_type, c_int)
        p%char_decomp = int(char_decomp, c_int)
        p%tfluct_solver = int(tfluct_solver, c_int)
        p%mthbc = 2
        do k = 1, 2 * ndim
            p%mthbc(k) = int(mthbc(k), c_int)
        end do
        p%dx = dx(1)
        p%dy = dx(1)
        p%xlower = xlower(1)
        p%ylower = 0.d0
        if (ndim > 1) then
            p%dy = dx(2)
            p%ylower = xlower(2)
        end if
        p%rp = cfg_rp
        p%efix = cfg_efix
        if (cfg_efix < 0) then
            p%efix = 0
            if (cfg_rp == SCL_RP_EULER .or. cfg_rp == SCL_RP_SW1D) p%efix = 1
        end if
        p%u = cfg_u
        p%gamma = cfg_gamma
        p%grav = cfg_grav
        p%time_integrator = 3
        if (c_associated(scl_h)) p%time_integrator = scl_p%time_integrator
        if (ti > 0) p%time_integrator = int(ti, c_int)
        p%precision = cfg_precision
        p%mthlim = 1
        do k = 1, min(4, size(mthlim))
            p%mthlim(k) = int(mthlim(k), c_int)
        end do
        p%src_term = cfg_src
        p%rho = cfg_rho
        p%bulk = cfg_bulk
        p%bc_user = cfg_bc_user
        p%wall = cfg_wall
        if (c_associated(scl_h)) then
            if (same_run(p, scl_p)) then
                h = scl_h
                return
            end if
            call sharpclaw_cuda_release()
        end if
        ierr = scl_create(p, scl_h)
        if (ierr /= SCL_OK) call scl_stop('scl_create', ierr)
        scl_p = p
        if (maux > 0) then
            ierr = scl_set_aux(scl_h, aux)
            if (ierr /= SCL_OK) call scl_stop('scl_set_aux', ierr)
        end if
        if (cfg_b4step /= SCL_B4STEP_NONE) then
            ierr = scl_set_b4step(scl_h, cfg_b4step, cfg_b4param)
            if (ierr /= SCL_OK) call scl_stop('scl_set_b4step', ierr)
        end if
        h = scl_h
    end function scl_handle_for

    logical function same_run(a, b)
        type(scl_params), intent(in) :: a, b
        same_run = a%ndim == b%ndim .and. a%mx == b%mx .and. a%my == b%my .and. a%meqn == b%meqn .and. &
                   a%maux == b%maux .and. a%mcapa == b%mcapa .and. a%lim_type == b%lim_type .and. &
                   a%char_decomp == b%char_decomp .and. a%tfluct_solver == b%tfluct_solver .and. &
                   all(a%mthbc == b%mthbc) .and. a%dx == b%dx .and. a%dy == b%dy .and. &
                   a%xlower == b%xlower .and. a%ylower == b%ylower .and. &
                   a%time_integrator == b%time_integrator .and. all(a%mthlim == b%mthlim)
    end function same_run

end module sharpclaw_cuda


! ======================================================================
! flux1(q1d,g,dq1d,aux,dt,cfl,t,rp,tfluct,ixy) -- src/flux1.f90:2
! dq1d(1:mx,:) gets dq1d - dtdx*(fluctuations) of one line; in 2-D dq1d is
! zeroed first (flux1.f90:62).  The library returns 0 - dtdx*(...), and
! adding it to dq1d is exactly the reference's dq1d - dtdx*(...).
! ======================================================================
subroutine flux1(q1d,g,dq1d,aux,dt,cfl,t,rp,tfluct,ixy)
    use ClawData
    use ClawParams
    use sharpclaw_cuda
    implicit none
    type(griddat) g
    integer, intent(in) :: ixy
    double precision :: q1d(1-mbc:nx(ixy)+mbc, meqn)
    double precision :: dq1d(1-mbc:maxnx+mbc, meqn)
    double precision :: aux(1-mbc:nx(ixy)+mbc, maux)
    double precision, intent(in) :: dt
    double precision, intent(out) :: cfl
    integer :: t                          ! declared integer and unused by the reference (flux1.f90:52)
    external rp, tfluct
    double precision, allocatable :: dqt(:,:)
    double precision :: auxd(1)
    integer(c_int) :: ierr
    integer :: mx, m
    type(c_ptr) :: h
    mx = nx(ixy)
    allocate(dqt(1-mbc:mx+mbc, meqn))
    if (ndim > 1) dq1d = 0.d0
    h = scl_handle_for(0)
    if (maux > 0) then
        ierr = scl_flux1(h, q1d, aux, dqt, dt, int(ixy, c_int), int(mx, c_int), cfl)
    else
        ierr = scl_flux1(h, q1d, auxd, dqt, dt, int(ixy, c_int), int(mx, c_int), cfl)
    end if
    if (ierr /= SCL_OK) call scl_stop('flux1', ierr)
    do m = 1, meqn
        dq1d(1:mx, m) = dq1d(1:mx, m) + dqt(1:mx, m)
    end do
    deallocate(dqt)
end subroutine flux1


! ======================================================================
! flux2(q,g,dq,aux,dt,cfl,t,rp,tfluct) -- src/2d/flux2.f90:2
! dq(1:nx,1:ny,:) += the x- and y-sweeps, cfl = the largest line CFL
! including the ghost lines (flux2.f90:36,47,68,80).  q is intent(in) here,
! and the library refills the ghost cells of the copy it is given (from the
! same bc as step applied).  With dq entering as zero (src/2d/src2.f90) the
! sum is the reference's ((0 + dq_x) + dq_y) bit for bit.
! ======================================================================
subroutine flux2(q,g,dq,aux,dt,cfl,t,rp,tfluct)
    use ClawData
    use ClawParams
    use sharpclaw_cuda
    implicit none
    type(griddat) g
    external rp, tfluct
    double precision, intent(in) :: q(1-mbc:nx(1)+mbc, 1-mbc:nx(2)+mbc, meqn)
    double precision, intent(inout) :: dq(1-mbc:nx(1)+mbc, 1-mbc:nx(2)+mbc, meqn)
    double precision, intent(in) :: aux(1-mbc:nx(1)+mbc, 1-mbc:nx(2)+mbc, maux)
    double precision, intent(in) :: dt, t
    double precision, intent(out) :: cfl
    double precision, allocatable :: qt(:,:,:), dqt(:,:,:)
    integer(c_int) :: ierr
    allocate(qt(1-mbc:nx(1)+mbc, 1-mbc:nx(2)+mbc, meqn), dqt(1-mbc:nx(1)+mbc, 1-mbc:nx(2)+mbc, meqn))
    qt = q
    ierr = scl_step_dq(scl_handle_for(0), qt, dqt, dt, t, cfl)
    if (ierr /= SCL_OK) call scl_stop('flux2', ierr)
    dq(1:nx(1), 1:nx(2), :) = dq(1:nx(1), 1:nx(2), :) + dqt(1:nx(1), 1:nx(2), :)
    deallocate(qt, dqt)
end subroutine flux2


! ======================================================================
! step(q,g,dq,aux,dt,cfl,t,rp,src,tfluct) -- src/1d/step1d.f90:2 and
! src/2d/step2d.f90:2 (one routine for both: the library reads ndim)
! bc (q's ghost cells, in place), src (the device hook chosen in
! sharpclaw_cuda_setup; zero without one) and flux1 / flux2: dq = dt*L(q).
! ======================================================================
subroutine step(q,g,dq,aux,dt,cfl,t,rp,src,tfluct)
    use ClawData
    use ClawParams
    use sharpclaw_cuda
    implicit none
    type(griddat) g
    double precision :: q(*), dq(*), aux(*)
    double precision, intent(in) :: dt, t
    double precision, intent(out) :: cfl
    external rp, src, tfluct
    integer(c_int) :: ierr
    ierr = scl_step_dq(scl_handle_for(0), q, dq, dt, t, cfl)
    if (ierr /= SCL_OK) call scl_stop('step', ierr)
end subroutine step


! ======================================================================
! sharpclaw(...) -- src/sharpclaw.f90:2, called at src/main.f90:192
! The whole time loop (b4step, the integrator's stages, dt control,
! rejection and retake, info codes) runs on the device; q (module Global)
! goes in and comes back.  r1, r2 and the externals are not used.
! ======================================================================
subroutine sharpclaw(tstart,tend,cfl_maxused,cfl_last,dt_minused, &
                dt_maxused,dt_last,steps_taken,info,dt_initial,dt_max, &
                dt_variable,time_integrator,verbosity, &
                cfl_max,cfl_desired,max_steps,r1,r2,bc,rp,tfluct,src,b4step)
    use ClawData
    use ClawParams
    use Global
    use sharpclaw_cuda
    implicit none
    external bc, rp, tfluct, src, b4step
    type(rkreg) r1, r2
    double precision :: tstart, tend
    double precision :: cfl_maxused, cfl_last, dt_minused, dt_maxused, dt_last
    double precision :: dt_initial, dt_max, cfl_max, cfl_desired
    integer :: steps_taken, info, max_steps, dt_variable, time_integrator, verbosity
    type(scl_run) :: run
    type(scl_result) :: res
    type(c_ptr) :: h
    integer(c_int) :: ierr
    h = scl_handle_for(time_integrator)
    run%tstart = tstart
    run%tend = tend
    run%dt_initial = dt_initial
    run%dt_max = dt_max
    run%cfl_max = cfl_max
    run%cfl_desired = cfl_desired
    run%max_steps = int(max_steps, c_int)
    run%dt_variable = int(dt_variable, c_int)
    ierr = scl_set_q(h, q)
    if (ierr == SCL_OK) ierr = scl_sharpclaw(h, run, res)
    if (ierr == SCL_OK) ierr = scl_get_q(h, q)
    if (ierr /= SCL_OK) call scl_stop('sharpclaw', ierr)
    tend = res%tend
    cfl_maxused = res%cfl_maxused
    cfl_last = res%cfl_last
    dt_minused = res%dt_minused
    dt_maxused = res%dt_maxused
    dt_last = res%dt_last
    steps_taken = res%steps_taken
    info = res%info
    if (verbosity > 0) write(6,601) steps_taken, res%rejected, tend, cfl_maxused
601 format('SHARPCLAW (device): ', i8, ' steps, ', i6, ' rejected, t = ', d12.4, ', max CFL ', f8.4)
end subroutine sharpclaw
