! stx_interface.F90 -- Fortran 2003 iso_c_binding interface to libstx.so (include/stx.h).
!
! A Fortran host (the reference's equation_multideal_gpu_object,
! src/multideal/multideal_gpu.F90:164-211) uses this module to call the B200
! kernels in place of its CUDA-Fortran ones.  Derived types mirror the C structs
! field by field (kinds and order must match stx.h); every entry point returns
! STX_OK (0) or a negative STX_E_* code.  Device arrays are passed as type(c_ptr)
! values, e.g. c_devloc(w_gpu) with nvfortran's cudafor; the stream as
! transfer(stream1, c_null_ptr) (or c_null_ptr for stream 0).  Tables passed to
! stx_ctx_create are HOST pointers (the context copies them); the tables of
! stx_rosenbrock_krylov_noalloc are DEVICE pointers.
module stx_interface
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: STX_ABI_VERSION = 1
  integer(c_int), parameter :: STX_OK = 0, STX_E_INVALID = -1, STX_E_CUDA = -2, STX_E_NOMEM = -3
  integer(c_int), parameter :: STX_E_UNSUPPORTED = -4, STX_E_TOO_LARGE = -5, STX_E_LOCAL_MEM = -6
  integer(c_int32_t), parameter :: STX_ST_NEWTON_CAP = 1, STX_ST_ROS_STEPS_CAP = 2, STX_ST_ROS_TRY_CAP = 4
  integer(c_int32_t), parameter :: STX_ST_NONFINITE = 8, STX_ST_WAIT_TIMEOUT = 16
  integer(c_int32_t), parameter :: STX_BC_EXCHANGE = -1
  integer(c_int), parameter :: STX_PREC_FP64 = 0, STX_PREC_MIXED = 1
  integer(c_int), parameter :: STX_NK = 8

  type, bind(c) :: stx_tables
    integer(c_int32_t) :: ns, nr
    integer(c_int32_t) :: indx_cp_l, indx_cp_r, nsetcv, num_t_tab
    real(c_double)     :: t_min_tab, dt_tab, R_univ
    type(c_ptr) :: mw, mwinv, rgas
    type(c_ptr) :: trange
    type(c_ptr) :: cp_coeff, cv_coeff
    type(c_ptr) :: visc, lambda
    type(c_ptr) :: diffbin
    type(c_ptr) :: reac_ty, is_rev
    type(c_ptr) :: arr_a, arr_b, arr_ea
    type(c_ptr) :: falloff
    type(c_ptr) :: tb_eff, r_coeffs, p_coeffs
    type(c_ptr) :: kc_tab
    integer(c_int32_t) :: n_eoi
    type(c_ptr) :: aw_eoi, coeff_eoi
    type(c_ptr) :: nainsp
    type(c_ptr) :: beta0
  end type stx_tables

  type, bind(c) :: stx_grid
    integer(c_int32_t) :: nx, ny, nz, ng
    type(c_ptr) :: x, y, z
    type(c_ptr) :: dcsidx, detady, dzitdz
    type(c_ptr) :: dcsidxs, detadys, dzitdzs
  end type stx_grid

  type, bind(c) :: stx_params
    integer(c_int32_t) :: nv_aux
    real(c_double)     :: p0, rho0, u0, eps_sensor, tol_iter_nr
    integer(c_int32_t) :: ep_order, nkeep, weno_scheme, weno_version, flux_splitting
    integer(c_int32_t) :: sensor_type, visc_order, conservative_viscous
    real(c_double)     :: sensor_threshold
    integer(c_int32_t) :: bctags(6)
    integer(c_int32_t) :: bctags_nr(6)
    integer(c_int32_t) :: force_zero_flux(6)
    integer(c_int32_t) :: eul_imin, eul_imax, eul_jmin, eul_jmax, eul_kmin, eul_kmax
    integer(c_int32_t) :: enable_chemistry
    integer(c_int32_t) :: rosenbrock_version
    integer(c_int32_t) :: operator_splitting
    integer(c_int32_t) :: ros_maxsteps, ros_maxtry
    real(c_double)     :: ros_eps
    integer(c_int32_t) :: nrk
    real(c_double)     :: rhork(4), gamrk(4)
    type(c_ptr)        :: winf
    real(c_double)     :: T_wall
  end type stx_params

  type, bind(c) :: stx_fields
    type(c_ptr) :: w, w_aux, fl, fln, fl_sav
    type(c_ptr) :: fluid_mask
  end type stx_fields

  type, bind(c) :: stx_tuning
    integer(c_int32_t) :: sweep_kind(3)
    integer(c_int32_t) :: weno_list(3)
    integer(c_int32_t) :: chem_ctas_per_sm
    integer(c_int32_t) :: chem_ctas_max
    integer(c_int32_t) :: batch_ctas_max
    real(c_float)      :: sweep_ms(3)
    real(c_float)      :: chem_ms
  end type stx_tuning

  type, bind(c) :: stx_kprof
    integer(c_int64_t) :: launches
    integer(c_int64_t) :: timed
    real(c_double)     :: ms
    real(c_double)     :: bytes
  end type stx_kprof

  interface
    ! ------------------------------------------------------------ library
    integer(c_int) function stx_abi_version() bind(c, name="stx_abi_version")
      import :: c_int
    end function
    type(c_ptr) function stx_strerror(code) bind(c, name="stx_strerror")
      import :: c_ptr, c_int
      integer(c_int), value :: code
    end function

    ! ------------------------------------------------------------ contexts (multideal_gpu.F90:1361-1468)
    integer(c_int) function stx_ctx_create(par, tab, grid, ctx) bind(c, name="stx_ctx_create")
      import :: c_int, c_ptr, stx_params, stx_tables, stx_grid
      type(stx_params), intent(in) :: par
      type(stx_tables), intent(in) :: tab
      type(stx_grid),   intent(in) :: grid
      type(c_ptr), intent(out)     :: ctx
    end function
    integer(c_int) function stx_ctx_create_like(base, par, grid, ctx) bind(c, name="stx_ctx_create_like")
      import :: c_int, c_ptr, stx_params, stx_grid
      type(c_ptr), value           :: base
      type(stx_params), intent(in) :: par
      type(stx_grid),   intent(in) :: grid
      type(c_ptr), intent(out)     :: ctx
    end function
    integer(c_int) function stx_ctx_create_like_on(base, par, grid, stream, ctx) bind(c, name="stx_ctx_create_like_on")
      import :: c_int, c_ptr, stx_params, stx_grid
      type(c_ptr), value           :: base, stream
      type(stx_params), intent(in) :: par
      type(stx_grid),   intent(in) :: grid
      type(c_ptr), intent(out)     :: ctx
    end function
    integer(c_int) function stx_ctx_destroy(ctx) bind(c, name="stx_ctx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    ! fn: integer(c_int) function fn(user, stream, field, nvar) bind(c), values c_ptr/c_ptr/c_ptr/c_int
    integer(c_int) function stx_set_exchange(ctx, fn, user) bind(c, name="stx_set_exchange")
      import :: c_int, c_ptr, c_funptr
      type(c_ptr), value    :: ctx
      type(c_funptr), value :: fn
      type(c_ptr), value    :: user
    end function

    ! ------------------------------------------------------------ auxiliary fields and ghosts
    integer(c_int) function stx_eval_aux(ctx, stream, w, w_aux, istart, iend, jstart, jend, kstart, kend) &
        bind(c, name="stx_eval_aux")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w, w_aux
      integer(c_int), value :: istart, iend, jstart, jend, kstart, kend
    end function
    integer(c_int) function stx_compute_aux(ctx, stream, w, w_aux, central, ghost) bind(c, name="stx_compute_aux")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w, w_aux
      integer(c_int), value :: central, ghost
    end function
    integer(c_int) function stx_eval_aux2(ctx, stream, w_aux) bind(c, name="stx_eval_aux2")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w_aux
    end function
    integer(c_int) function stx_bcextr_var(ctx, stream, var) bind(c, name="stx_bcextr_var")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, var
    end function
    integer(c_int) function stx_bcswap(ctx, stream, field, nvar) bind(c, name="stx_bcswap")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, field
      integer(c_int), value :: nvar
    end function
    integer(c_int) function stx_update_ghost(ctx, stream, w, do_swap) bind(c, name="stx_update_ghost")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w
      integer(c_int), value :: do_swap
    end function
    integer(c_int) function stx_update_ghost_aux(ctx, stream, w, w_aux, do_swap) bind(c, name="stx_update_ghost_aux")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w, w_aux
      integer(c_int), value :: do_swap
    end function
    integer(c_int) function stx_bc_nr(ctx, stream, w_aux, w, fl) bind(c, name="stx_bc_nr")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w_aux, w, fl
    end function

    ! ------------------------------------------------------------ fluxes
    integer(c_int) function stx_euler_x(ctx, stream, w_aux, fl, imin, imax, overwrite) bind(c, name="stx_euler_x")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w_aux, fl
      integer(c_int), value :: imin, imax, overwrite
    end function
    integer(c_int) function stx_euler_y(ctx, stream, w_aux, fl, jmin, jmax, overwrite) bind(c, name="stx_euler_y")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w_aux, fl
      integer(c_int), value :: jmin, jmax, overwrite
    end function
    integer(c_int) function stx_euler_z(ctx, stream, w_aux, fl, kmin, kmax, overwrite) bind(c, name="stx_euler_z")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w_aux, fl
      integer(c_int), value :: kmin, kmax, overwrite
    end function
    integer(c_int) function stx_visflx(ctx, stream, w_aux, fl, mode) bind(c, name="stx_visflx")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w_aux, fl
      integer(c_int), value :: mode
    end function

    ! ------------------------------------------------------------ RK bookkeeping
    integer(c_int) function stx_init_flux(ctx, stream, fl, fln, rhodt) bind(c, name="stx_init_flux")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, fl, fln
      real(c_double), value :: rhodt
    end function
    integer(c_int) function stx_init_flux_simpler(ctx, stream, fl, fln, fl_sav, rhodt) &
        bind(c, name="stx_init_flux_simpler")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, fl, fln, fl_sav
      real(c_double), value :: rhodt
    end function
    integer(c_int) function stx_sav_flx(ctx, stream, fl, fl_sav) bind(c, name="stx_sav_flx")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, fl, fl_sav
    end function
    integer(c_int) function stx_update_flux(ctx, stream, fl, fln, gamdt) bind(c, name="stx_update_flux")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, fl, fln
      real(c_double), value :: gamdt
    end function
    integer(c_int) function stx_update_simpler_flux(ctx, stream, fl, fln, fl_sav, gamdt) &
        bind(c, name="stx_update_simpler_flux")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, fl, fln, fl_sav
      real(c_double), value :: gamdt
    end function
    integer(c_int) function stx_update_field(ctx, stream, w, fln, fluid_mask) bind(c, name="stx_update_field")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w, fln, fluid_mask
    end function
    integer(c_int) function stx_rk_finish(ctx, stream, w, fl, fln, fl_sav, fluid_mask, gamdt, simpler) &
        bind(c, name="stx_rk_finish")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, w, fl, fln, fl_sav, fluid_mask
      real(c_double), value :: gamdt
      integer(c_int), value :: simpler
    end function
    integer(c_int) function stx_compute_dt(ctx, stream, w_aux, fluid_mask, out9) bind(c, name="stx_compute_dt")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, w_aux, fluid_mask
      real(c_double), intent(out) :: out9(9)
    end function

    integer(c_int) function stx_compute_residual(ctx, stream, fln, w_aux, fluid_mask, dt, out7) &
        bind(c, name="stx_compute_residual")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, fln, w_aux, fluid_mask
      real(c_double), value :: dt
      real(c_double), intent(out) :: out7(7)
    end function

    ! ------------------------------------------------------------ chemistry
    integer(c_int) function stx_rosenbrock(ctx, stream, w, w_aux, dttry, time_start, time_end) &
        bind(c, name="stx_rosenbrock")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, w, w_aux
      real(c_double), value :: dttry, time_start, time_end
    end function
    integer(c_int) function stx_rosenbrock_krylov(ctx, stream, w, w_aux, fl_sav, dttry, time_start, time_end, &
        simpler) bind(c, name="stx_rosenbrock_krylov")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream, w, w_aux, fl_sav
      real(c_double), value :: dttry, time_start, time_end
      integer(c_int), value :: simpler
    end function
    integer(c_int) function stx_compute_chemistry(ctx, stream, w, w_aux, fl) bind(c, name="stx_compute_chemistry")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, w, w_aux, fl
    end function
    ! no context, no allocation; tab_dev holds DEVICE pointers; raise cudaLimitStackSize once first
    integer(c_int) function stx_rosenbrock_krylov_noalloc(par, tab_dev, grid, stream, w, w_aux, fl_sav, dttry, &
        time_start, time_end, simpler, status) bind(c, name="stx_rosenbrock_krylov_noalloc")
      import :: c_int, c_ptr, c_double, stx_params, stx_tables, stx_grid
      type(stx_params), intent(in) :: par
      type(stx_tables), intent(in) :: tab_dev
      type(stx_grid),   intent(in) :: grid
      type(c_ptr), value :: stream, w, w_aux, fl_sav
      real(c_double), value :: dttry, time_start, time_end
      integer(c_int), value :: simpler
      type(c_ptr), value :: status
    end function
    integer(c_int) function stx_batch0d_integrate(ctx, stream, n, T0, p0, Y0, t_max, dttry, ign_factor, &
        end_factor, max_steps, Y, T, t_ign, t_end, nsteps) bind(c, name="stx_batch0d_integrate")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx, stream
      integer(c_int), value :: n
      type(c_ptr), value :: T0, p0, Y0
      real(c_double), value :: t_max, dttry, ign_factor, end_factor
      integer(c_int), value :: max_steps
      type(c_ptr), value :: Y, T, t_ign, t_end, nsteps
    end function

    ! ------------------------------------------------------------ whole steps (multideal_gpu.F90:536-621, 1853-1931)
    integer(c_int) function stx_rk_sync(ctx, stream, f, dt, simpler) bind(c, name="stx_rk_sync")
      import :: c_int, c_ptr, c_double, stx_fields
      type(c_ptr), value :: ctx, stream
      type(stx_fields), intent(in) :: f
      real(c_double), value :: dt
      integer(c_int), value :: simpler
    end function
    integer(c_int) function stx_advance_solution(ctx, stream, f, dt, time) bind(c, name="stx_advance_solution")
      import :: c_int, c_ptr, c_double, stx_fields
      type(c_ptr), value :: ctx, stream
      type(stx_fields), intent(in) :: f
      real(c_double), value :: dt, time
    end function
    integer(c_int) function stx_set_precision(ctx, mode) bind(c, name="stx_set_precision")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: mode
    end function
    integer(c_int) function stx_graph_create(ctx, f, dt, nsteps, g) bind(c, name="stx_graph_create")
      import :: c_int, c_ptr, c_double, stx_fields
      type(c_ptr), value :: ctx
      type(stx_fields), intent(in) :: f
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
      type(c_ptr), intent(out) :: g
    end function
    integer(c_int) function stx_graph_create_cfl(ctx, f, cfl, nsteps, g) bind(c, name="stx_graph_create_cfl")
      import :: c_int, c_ptr, c_double, stx_fields
      type(c_ptr), value :: ctx
      type(stx_fields), intent(in) :: f
      real(c_double), value :: cfl
      integer(c_int), value :: nsteps
      type(c_ptr), intent(out) :: g
    end function
    integer(c_int) function stx_graph_state(g, stream, time, dt) bind(c, name="stx_graph_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: g, stream
      real(c_double), intent(out) :: time, dt
    end function
    integer(c_int) function stx_graph_launch(g, stream, time) bind(c, name="stx_graph_launch")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: g, stream
      real(c_double), value :: time
    end function
    integer(c_int) function stx_graph_destroy(g) bind(c, name="stx_graph_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: g
    end function

    ! ------------------------------------------------------------ tuning, status, instrumentation
    integer(c_int) function stx_get_tuning(ctx, t) bind(c, name="stx_get_tuning")
      import :: c_int, c_ptr, stx_tuning
      type(c_ptr), value :: ctx
      type(stx_tuning), intent(out) :: t
    end function
    integer(c_int) function stx_set_tuning(ctx, t) bind(c, name="stx_set_tuning")
      import :: c_int, c_ptr, stx_tuning
      type(c_ptr), value :: ctx
      type(stx_tuning), intent(in) :: t
    end function
    integer(c_int) function stx_autotune(ctx, stream, f, dt_chem, t) bind(c, name="stx_autotune")
      import :: c_int, c_ptr, c_double, stx_fields, stx_tuning
      type(c_ptr), value :: ctx, stream
      type(stx_fields), intent(in) :: f
      real(c_double), value :: dt_chem
      type(stx_tuning), intent(out) :: t
    end function
    integer(c_int) function stx_status(ctx, stream, bits, reset) bind(c, name="stx_status")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx, stream
      integer(c_int32_t), intent(out) :: bits
      integer(c_int), value :: reset
    end function
    integer(c_int) function stx_status_enqueue(ctx, stream, bits, reset) bind(c, name="stx_status_enqueue")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream, bits
      integer(c_int), value :: reset
    end function
    integer(c_int) function stx_profile_enable(ctx, on) bind(c, name="stx_profile_enable")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: on
    end function
    integer(c_int) function stx_profile_read(ctx, out) bind(c, name="stx_profile_read")
      import :: c_int, c_ptr, stx_kprof, STX_NK
      type(c_ptr), value :: ctx
      type(stx_kprof), intent(out) :: out(STX_NK)
    end function
  end interface
end module stx_interface
