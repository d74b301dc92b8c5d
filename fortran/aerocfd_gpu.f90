!! ISO_C_BINDING interface to libaerocfd_gpu.so (include/aerocfd_gpu.h).
!!
!! Every hot-path routine of aerocfd keeps its argument list; the interfaces
!! below bind the same arguments (all by reference, explicit-shape arrays) to
!! the C entry points.  A call site such as main.f90:359
!!
!!   call inviscid_flux_1(blk(m0)%rhsi, blk(m0)%q, blk(m0)%dxidx, blk(m0)%inv_j, &
!!                        is,ie,js,je,ks,ke, is0,ie0,js0,je0,ks0,ke0, is1,ie1,js1,je1,ks1,ke1, gamma)
!!
!! becomes
!!
!!   ierr = aero_inviscid_flux_1(blk(m0)%rhsi, blk(m0)%q, blk(m0)%dxidx, blk(m0)%inv_j, &
!!                        is,ie,js,je,ks,ke, is0,ie0,js0,je0,ks0,ke0, is1,ie1,js1,je1,ks1,ke1, gamma)
!!   call aero_check(ierr)
!!
!! This file is source only: the image it was written in has no Fortran
!! compiler.
module aerocfd_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: AERO_OK = 0
  integer(c_int), parameter :: AERO_F_Q = 0, AERO_F_PRI_V = 1, AERO_F_RHSI = 2, AERO_F_RHSV = 3, &
                               AERO_F_RHS = 4, AERO_F_DT = 5, AERO_F_DXIDX = 6, AERO_F_INV_J = 7, &
                               AERO_F_AMU = 8, AERO_F_NUT = 9, AERO_F_SA_RHS = 10, AERO_F_X = 11, &
                               AERO_F_Y = 12, AERO_F_Z = 13, AERO_F_DIST = 14, AERO_F_ALPHA = 15, &
                               AERO_F_BETA = 16, AERO_F_GGAMMA = 17, AERO_F_DUDX = 18, AERO_F_TAO = 19, &
                               AERO_F_VOR = 20, AERO_F_LENGTH = 21, AERO_F_SPACING = 22, AERO_F_Q0 = 23

  interface
    integer(c_int) function aero_init(device) bind(C, name="aero_init")
      import :: c_int
      integer(c_int), value :: device
    end function

    integer(c_int) function aero_finalize() bind(C, name="aero_finalize")
      import :: c_int
    end function

    integer(c_int) function aero_configure(iflags, params) bind(C, name="aero_configure")
      import :: c_int, c_double
      integer(c_int) :: iflags(8)
      real(c_double) :: params(7)
    end function

    integer(c_int) function aero_register_block(m, box18, num_subface, subfaces) &
        bind(C, name="aero_register_block")
      import :: c_int
      integer(c_int), value :: m, num_subface
      integer(c_int) :: box18(18), subfaces(11, *)
    end function

    integer(c_int) function aero_bind_field(m, field, host) bind(C, name="aero_bind_field")
      import :: c_int, c_ptr
      integer(c_int), value :: m, field
      type(c_ptr), value :: host
    end function

    ! sub_timeadvancement_2ndcrank.f90:1 (crank2nd)
    integer(c_int) function aero_crank2nd(q, q0, dt, pri_v, rhs, rhsi, rhsv, dxidx, inv_j, &
        is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1, &
        gamma, mm, ssub) bind(C, name="aero_crank2nd")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0
      integer(c_int) :: is1, ie1, js1, je1, ks1, ke1, mm, ssub
      real(c_double) :: q(5, is:ie, js:je, ks:ke), q0(-1:0, 5, is:ie, js:je, ks:ke), dt(is:ie, js:je, ks:ke)
      real(c_double) :: pri_v(7, is:ie, js:je, ks:ke), rhs(5, is:ie, js:je, ks:ke)
      real(c_double) :: rhsi(5, is:ie, js:je, ks:ke), rhsv(5, is:ie, js:je, ks:ke)
      real(c_double) :: dxidx(9, is:ie, js:je, ks:ke), inv_j(is:ie, js:je, ks:ke), gamma
    end function

    ! main.f90:692 (update_q0)
    integer(c_int) function aero_update_q0(q0, q, is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0) &
        bind(C, name="aero_update_q0")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0
      real(c_double) :: q0(-1:0, 5, is:ie, js:je, ks:ke), q(5, is:ie, js:je, ks:ke)
    end function

    ! sub_output_forceintegration.f90:8 (clcd_output): out8 = fp(3), fv(3), cl, cd
    integer(c_int) function aero_clcd_output(sref, out8) bind(C, name="aero_clcd_output")
      import :: c_int, c_double
      real(c_double), value :: sref
      real(c_double) :: out8(8)
    end function

    ! sub_output_surface.f90:8 (surface_output): node and zone counts, then
    ! xyzcp(4, n_nodes) and zones(5, n_zones) = block, face, idim, jdim, kdim
    integer(c_int) function aero_surface_count(n_nodes, n_zones) bind(C, name="aero_surface_count")
      import :: c_int, c_long_long
      integer(c_long_long) :: n_nodes
      integer(c_int) :: n_zones
    end function

    integer(c_int) function aero_surface_output(xyzcp, zones) bind(C, name="aero_surface_output")
      import :: c_int, c_double
      real(c_double) :: xyzcp(*)
      integer(c_int) :: zones(*)
    end function

    ! CTAs per block of the LU-SGS sweep: 1, 2, 4 or 8 (no counterpart in the reference)
    integer(c_int) function aero_set_sweep_cluster(ctas) bind(C, name="aero_set_sweep_cluster")
      import :: c_int
      integer(c_int), value :: ctas
    end function

    ! plane-value exchange of a cluster sweep: 0 through L2, 1 bulk copies
    ! between shared memories, 2 pipelined k-slabs, 3 as 1 with two CTAs per
    ! SM (no counterpart in the reference)
    integer(c_int) function aero_set_sweep_exchange(mode) bind(C, name="aero_set_sweep_exchange")
      import :: c_int
      integer(c_int), value :: mode
    end function

    ! L2 prefetch distance of the bulk-exchange sweep in planes (2..4)
    integer(c_int) function aero_set_sweep_prefetch(planes) bind(C, name="aero_set_sweep_prefetch")
      import :: c_int
      integer(c_int), value :: planes
    end function

    ! register-bounded FP64 viscous part a kernel (0 / 1)
    integer(c_int) function aero_set_register_bound(on) bind(C, name="aero_set_register_bound")
      import :: c_int
      integer(c_int), value :: on
    end function

    ! CTAs per block of the SA sweep, pipelined by k-slabs (1, 2, 4, 8, 16)
    integer(c_int) function aero_set_sa_sweep_cluster(ctas) bind(C, name="aero_set_sa_sweep_cluster")
      import :: c_int
      integer(c_int), value :: ctas
    end function

    ! polls of each bounded wait of the staged LU-SGS sweep (fault-injection
    ! hook; default and largest 1048576)
    integer(c_int) function aero_set_poll_budget(polls) bind(C, name="aero_set_poll_budget")
      import :: c_int, c_long_long
      integer(c_long_long), value :: polls
    end function

    ! fault injection: copies of forward hyperplane `plane` withheld (-1: off)
    integer(c_int) function aero_inject_sweep_stall(plane) bind(C, name="aero_inject_sweep_stall")
      import :: c_int
      integer(c_int), value :: plane
    end function

    integer(c_int) function aero_finish_setup() bind(C, name="aero_finish_setup")
      import :: c_int
    end function

    integer(c_int) function aero_sync_to_device(mask) bind(C, name="aero_sync_to_device")
      import :: c_long_long
      integer(c_long_long), value :: mask
    end function

    integer(c_int) function aero_sync_to_host(mask) bind(C, name="aero_sync_to_host")
      import :: c_long_long
      integer(c_long_long), value :: mask
    end function

    ! sub_getpri_v.f90:19
    integer(c_int) function aero_get_primitivevariables(mm, pri_v, q, gamma, cv, is, ie, js, je, ks, ke) &
        bind(C, name="aero_get_primitivevariables")
      import :: c_int, c_double
      integer(c_int) :: mm, is, ie, js, je, ks, ke
      real(c_double) :: pri_v(7, is:ie, js:je, ks:ke), q(5, is:ie, js:je, ks:ke), gamma, cv
    end function

    ! sub_inviscid1.f90:8
    integer(c_int) function aero_inviscid_flux_1(rhsi, q, dxidx, inv_j, is, ie, js, je, ks, ke, &
        is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1, gamma) bind(C, name="aero_inviscid_flux_1")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1
      real(c_double) :: rhsi(5, is:ie, js:je, ks:ke), q(5, is:ie, js:je, ks:ke)
      real(c_double) :: dxidx(9, is:ie, js:je, ks:ke), inv_j(is:ie, js:je, ks:ke), gamma
    end function

    ! thirdorder_weno and roe_3d as routines of their own (unit tests)
    integer(c_int) function aero_thirdorder_weno(df, f, is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, &
        coord, direction) bind(C, name="aero_thirdorder_weno")
      import :: c_int, c_double
      real(c_double) :: df(*), f(*)
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, coord, direction
    end function

    integer(c_int) function aero_roe_3d(ql, qr, flux, dxidx, inv_j, gamma, is, ie, js, je, ks, ke, &
        is0, ie0, js0, je0, ks0, ke0, coord) bind(C, name="aero_roe_3d")
      import :: c_int, c_double
      real(c_double) :: ql(*), qr(*), flux(*), dxidx(*), inv_j(*), gamma
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, coord
    end function

    ! Steger-Warming splitting + WENO5 (no counterpart in the reference: iflag_inviscid = 5, bufferLength = 3)
    integer(c_int) function aero_inviscid_flux_weno5(rhsi, q, dxidx, inv_j, is, ie, js, je, ks, ke, &
        is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1, gamma) bind(C, name="aero_inviscid_flux_weno5")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1
      real(c_double) :: rhsi(5, is:ie, js:je, ks:ke), q(5, is:ie, js:je, ks:ke)
      real(c_double) :: dxidx(9, is:ie, js:je, ks:ke), inv_j(is:ie, js:je, ks:ke), gamma
    end function

    ! WCNS5 + Roe flux (no counterpart in the reference: iflag_inviscid = 8, bufferLength = 3)
    integer(c_int) function aero_inviscid_flux_wcns5(rhsi, q, dxidx, inv_j, is, ie, js, je, ks, ke, &
        is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1, gamma) bind(C, name="aero_inviscid_flux_wcns5")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1
      real(c_double) :: rhsi(5, is:ie, js:je, ks:ke), q(5, is:ie, js:je, ks:ke)
      real(c_double) :: dxidx(9, is:ie, js:je, ks:ke), inv_j(is:ie, js:je, ks:ke), gamma
    end function

    ! sub_viscous.f90:9
    integer(c_int) function aero_viscous_flux(rhsv, pri_v, amu, vor, dudx, tao, dxidx, inv_j, tinf, prl, prt, &
        gamma, cv, re, is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1, mm) &
        bind(C, name="aero_viscous_flux")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1, mm
      real(c_double) :: rhsv(5, is:ie, js:je, ks:ke), pri_v(7, is:ie, js:je, ks:ke), amu(3, is:ie, js:je, ks:ke)
      real(c_double) :: vor(is:ie, js:je, ks:ke), dudx(9, is:ie, js:je, ks:ke), tao(6, is:ie, js:je, ks:ke)
      real(c_double) :: dxidx(9, is:ie, js:je, ks:ke), inv_j(is:ie, js:je, ks:ke)
      real(c_double) :: tinf, prl, prt, gamma, cv, re
    end function

    ! sub_timeadvancement_finddt.f90:24
    integer(c_int) function aero_find_dt(dt, dtmax, dtmin, cflmax, cflmin, pri_v, amu, dxidx, re, cfl, &
        is, ie, js, je, ks, ke, iflag_time, iflag_steady, iflag_unsteady) bind(C, name="aero_find_dt")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, iflag_time, iflag_steady, iflag_unsteady
      real(c_double) :: dt(is:ie, js:je, ks:ke), dtmax, dtmin, cflmax, cflmin, re, cfl
      real(c_double) :: pri_v(7, is:ie, js:je, ks:ke), amu(3, is:ie, js:je, ks:ke), dxidx(9, is:ie, js:je, ks:ke)
    end function

    ! sub_timeadvancement_1stimplicit.f90:7
    integer(c_int) function aero_implicit1st(q, dt, pri_v, rhs, rhsi, rhsv, dxidx, inv_j, &
        is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1, &
        gamma, cfl, xx, yy, zz) bind(C, name="aero_implicit1st")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1
      real(c_double) :: q(5, is:ie, js:je, ks:ke), dt(is:ie, js:je, ks:ke), pri_v(7, is:ie, js:je, ks:ke)
      real(c_double) :: rhs(5, is:ie, js:je, ks:ke), rhsi(5, is:ie, js:je, ks:ke), rhsv(5, is:ie, js:je, ks:ke)
      real(c_double) :: dxidx(9, is:ie, js:je, ks:ke), inv_j(is:ie, js:je, ks:ke), gamma, cfl
      real(c_double) :: xx(is:ie, js:je, ks:ke), yy(is:ie, js:je, ks:ke), zz(is:ie, js:je, ks:ke)
    end function

    ! sub_init_gridtransformation.f90:27
    integer(c_int) function aero_gridtransformation(dxidx, inv_j, alpha, beta, gamma, x, y, z, &
        is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, m0) bind(C, name="aero_gridtransformation")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, m0
      real(c_double) :: dxidx(9, is:ie, js:je, ks:ke), inv_j(is:ie, js:je, ks:ke)
      real(c_double) :: alpha(3, is:ie, js:je, ks:ke), beta(3, is:ie, js:je, ks:ke), gamma(3, is:ie, js:je, ks:ke)
      real(c_double) :: x(is:ie, js:je, ks:ke), y(is:ie, js:je, ks:ke), z(is:ie, js:je, ks:ke)
    end function

    ! module-state routines: no arguments, as in the reference
    integer(c_int) function aero_physical_bc() bind(C, name="aero_physical_bc")
      import :: c_int
    end function
    integer(c_int) function aero_updatebuffer() bind(C, name="aero_updatebuffer")
      import :: c_int
    end function
    integer(c_int) function aero_average1() bind(C, name="aero_average1")
      import :: c_int
    end function
    integer(c_int) function aero_average2() bind(C, name="aero_average2")
      import :: c_int
    end function
    integer(c_int) function aero_updatebuffercoordinate() bind(C, name="aero_updatebuffercoordinate")
      import :: c_int
    end function
    ! the reference's 2-D names (2-D cases only)
    integer(c_int) function aero_updatebuffer2d() bind(C, name="aero_updatebuffer2d")
      import :: c_int
    end function
    integer(c_int) function aero_average2d1() bind(C, name="aero_average2d1")
      import :: c_int
    end function
    integer(c_int) function aero_average2d2() bind(C, name="aero_average2d2")
      import :: c_int
    end function
    integer(c_int) function aero_updatebuffercoordinate2d() bind(C, name="aero_updatebuffercoordinate2d")
      import :: c_int
    end function
    integer(c_int) function aero_init_walldist() bind(C, name="aero_init_walldist")
      import :: c_int
    end function
    integer(c_int) function aero_residual(out7) bind(C, name="aero_residual")
      import :: c_int, c_double
      real(c_double) :: out7(7)
    end function
    integer(c_int) function aero_step(nsteps, resid_hist, dt_minmax) bind(C, name="aero_step")
      import :: c_int, c_ptr
      integer(c_int), value :: nsteps
      type(c_ptr), value :: resid_hist, dt_minmax
    end function

    function aero_last_error() bind(C, name="aero_last_error")
      import :: c_ptr
      type(c_ptr) :: aero_last_error
    end function

    ! device status word (AERO_ST_* bits raised since the last call; clears them)
    integer(c_int) function aero_get_status(status) bind(C, name="aero_get_status")
      import :: c_int
      integer(c_int) :: status
    end function

    ! the first cluster-sweep wait that gave up: sweep, block, rank, step, wait
    ! (all -1 when none did); clears the record
    integer(c_int) function aero_timeout_site(out5) bind(C, name="aero_timeout_site")
      import :: c_int
      integer(c_int) :: out5(5)
    end function

    ! per-block status words and retirement of failed blocks (batches)
    integer(c_int) function aero_get_block_status(out) bind(C, name="aero_get_block_status")
      import :: c_int
      integer(c_int) :: out(*)
    end function

    integer(c_int) function aero_clear_block_status() bind(C, name="aero_clear_block_status")
      import :: c_int
    end function

    integer(c_int) function aero_set_retirement(on) bind(C, name="aero_set_retirement")
      import :: c_int
      integer(c_int), value :: on
    end function

    ! sub_tur_sa.f90:7 (sa_model; main.f90:415, :538).  The arrays are passed
    ! by address as the reference passes them: dxidx and dudx are the blocks'
    ! (9, ...) arrays that sa_model views as (3, ..., 3).
    integer(c_int) function aero_sa_model(nut, sa_rhs, dt, pri_v, amu, dudx, vor, dxidx, inv_j, alpha, beta, &
        gamma, length, dist, spac, re, cfl, is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, &
        is1, ie1, js1, je1, ks1, ke1) bind(C, name="aero_sa_model")
      import :: c_int, c_double
      integer(c_int) :: is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0, ke0, is1, ie1, js1, je1, ks1, ke1
      real(c_double) :: nut(*), sa_rhs(*), dt(*), pri_v(*), amu(*), dudx(*), vor(*), dxidx(*), inv_j(*)
      real(c_double) :: alpha(*), beta(*), gamma(*), length(*), dist(*), spac(*), re, cfl
    end function

    ! module-state routines of the registered set (main.f90:142-318, :446)
    integer(c_int) function aero_compute_geometry(with_walldist) bind(C, name="aero_compute_geometry")
      import :: c_int
      integer(c_int), value :: with_walldist
    end function

    integer(c_int) function aero_init_flowfield() bind(C, name="aero_init_flowfield")
      import :: c_int
    end function

    integer(c_int) function aero_getpri_all() bind(C, name="aero_getpri_all")
      import :: c_int
    end function

    ! per-block residual norms of the last aero_step (7 per block)
    integer(c_int) function aero_residual_blocks(out7_per_block) bind(C, name="aero_residual_blocks")
      import :: c_int, c_double
      real(c_double) :: out7_per_block(7, *)
    end function

    ! a block's own Control.in values (batches of independent cases)
    integer(c_int) function aero_set_block_params(m, params) bind(C, name="aero_set_block_params")
      import :: c_int, c_double
      integer(c_int), value :: m
      real(c_double) :: params(7)
    end function

    ! execution options (no counterpart in the reference)
    integer(c_int) function aero_set_precision(mode) bind(C, name="aero_set_precision")
      import :: c_int
      integer(c_int), value :: mode
    end function

    integer(c_int) function aero_use_graphs(on) bind(C, name="aero_use_graphs")
      import :: c_int
      integer(c_int), value :: on
    end function

    integer(c_int) function aero_autotune(iters) bind(C, name="aero_autotune")
      import :: c_int
      integer(c_int), value :: iters
    end function

    integer(c_int) function aero_set_tuning(inv_tile, ew, visc, mats, nst_max) bind(C, name="aero_set_tuning")
      import :: c_int
      integer(c_int), value :: inv_tile, ew, visc, mats, nst_max
    end function

    function aero_tuning() bind(C, name="aero_tuning")
      import :: c_ptr
      type(c_ptr) :: aero_tuning
    end function

    ! benchmarking and profiling
    integer(c_int) function aero_step_timed(nsteps, flush_l2, device_ms) bind(C, name="aero_step_timed")
      import :: c_int, c_double
      integer(c_int), value :: nsteps, flush_l2
      real(c_double) :: device_ms
    end function

    integer(c_int) function aero_launch_count(count) bind(C, name="aero_launch_count")
      import :: c_int, c_long_long
      integer(c_long_long) :: count
    end function

    integer(c_int) function aero_profile(enable) bind(C, name="aero_profile")
      import :: c_int
      integer(c_int), value :: enable
    end function

    integer(c_int) function aero_profile_read(ms, counts, n) bind(C, name="aero_profile_read")
      import :: c_int, c_double, c_long_long
      real(c_double) :: ms(*)
      integer(c_long_long) :: counts(*)
      integer(c_int), value :: n
    end function

    function aero_profile_name(id) bind(C, name="aero_profile_name")
      import :: c_int, c_ptr
      integer(c_int), value :: id
      type(c_ptr) :: aero_profile_name
    end function

    integer(c_int) function aero_profile_timeline(ids, start_ms, end_ms, n) bind(C, name="aero_profile_timeline")
      import :: c_int, c_double
      integer(c_int) :: ids(*)
      real(c_double) :: start_ms(*), end_ms(*)
      integer(c_int), value :: n
    end function

    ! test hook: the device's correctly rounded pow (fn 0) and exp (fn 1)
    integer(c_int) function aero_math_eval(fn, x, y, out, n) bind(C, name="aero_math_eval")
      import :: c_int, c_double, c_long_long
      integer(c_int), value :: fn
      real(c_double) :: x(*), y(*), out(*)
      integer(c_long_long), value :: n
    end function

    ! residual norms from caller-owned device arrays (arrays of device
    ! addresses, one per block), allocating nothing; sa_rhs is c_loc of an
    ! array of device addresses or c_null_ptr (laminar), out7 the DEVICE
    ! address of 7 doubles (c_devloc of a CUDA Fortran device array, or
    ! acc_deviceptr under OpenACC), stream a cudaStream_t or c_null_ptr
    integer(c_int) function aero_residual_device_noalloc(nblocks, rhs, dt, inv_j, sa_rhs, boxes, totalnodes, &
        out7, stream) bind(C, name="aero_residual_device_noalloc")
      import :: c_int, c_double, c_ptr
      integer(c_int), value :: nblocks
      type(c_ptr) :: rhs(*), dt(*), inv_j(*)
      type(c_ptr), value :: sa_rhs
      integer(c_int) :: boxes(*)
      real(c_double), value :: totalnodes
      type(c_ptr), value :: out7, stream
    end function

    ! warm-start network on the tcgen05 tensor cores (no counterpart in the
    ! reference); BF16 operands as 16-bit integers
    integer(c_int) function aero_mlp_create(n_in, n_out, width, depth, batch, seed) bind(C, name="aero_mlp_create")
      import :: c_int, c_long_long
      integer(c_int), value :: n_in, n_out, width, depth, batch
      integer(c_long_long), value :: seed
    end function

    integer(c_int) function aero_mlp_destroy() bind(C, name="aero_mlp_destroy")
      import :: c_int
    end function

    integer(c_int) function aero_mlp_gemm(a, b, c, m, n, k, splits) bind(C, name="aero_mlp_gemm")
      import :: c_int, c_short, c_float
      integer(c_short) :: a(*), b(*)
      real(c_float) :: c(*)
      integer(c_int), value :: m, n, k, splits
    end function

    integer(c_int) function aero_mlp_gemm_timed(m, n, k, reps, ms_per_gemm) bind(C, name="aero_mlp_gemm_timed")
      import :: c_int, c_double
      integer(c_int), value :: m, n, k, reps
      real(c_double) :: ms_per_gemm
    end function

    integer(c_int) function aero_mlp_param_count(count) bind(C, name="aero_mlp_param_count")
      import :: c_int, c_long_long
      integer(c_long_long) :: count
    end function

    integer(c_int) function aero_mlp_get_params(out) bind(C, name="aero_mlp_get_params")
      import :: c_int, c_float
      real(c_float) :: out(*)
    end function

    integer(c_int) function aero_mlp_gradients(x, t, n, loss, grad) bind(C, name="aero_mlp_gradients")
      import :: c_int, c_float
      real(c_float) :: x(*), t(*), loss, grad(*)
      integer(c_int), value :: n
    end function

    integer(c_int) function aero_mlp_train(x, t, n, steps, lr, seed, loss_hist) bind(C, name="aero_mlp_train")
      import :: c_int, c_float, c_long_long, c_ptr
      real(c_float) :: x(*), t(*)
      type(c_ptr), value :: loss_hist
      integer(c_long_long), value :: n, seed
      integer(c_int), value :: steps
      real(c_float), value :: lr
    end function

    integer(c_int) function aero_mlp_predict(x, n, y) bind(C, name="aero_mlp_predict")
      import :: c_int, c_float, c_long_long
      real(c_float) :: x(*), y(*)
      integer(c_long_long), value :: n
    end function
  end interface

contains

  !! The reference prints and stops on errors (main.f90:87-90, :647-650);
  !! a non-zero status from the library does the same.
  subroutine aero_check(ierr)
    integer(c_int), intent(in) :: ierr
    character(kind=c_char), pointer :: msg(:)
    integer :: n
    if (ierr == AERO_OK) return
    call c_f_pointer(aero_last_error(), msg, [512])
    n = 0
    do while (n < 512)
      if (msg(n + 1) == c_null_char) exit
      n = n + 1
    end do
    print *, "aerocfd_gpu error", ierr, ": ", msg(1:n)
    stop
  end subroutine
end module aerocfd_gpu
