!
! hipft_gpu.f90 -- Fortran interface (iso_c_binding) to the C ABI declared in
! hipft_gpu.h, for HipFT's own driver (src/hipft.f90).
!
! HipFT keeps its solver state in module arrays and runs its hot path as
! do-concurrent loops; with this module the bodies of those routines become
! calls into the B200 library: setup's device part -> hipft_gpu_create,
! update_flow (src/hipft.f90:3371) -> hipft_gpu_update_flow, get_flow_dtmax
! (7287) -> hipft_gpu_flow_dtmax, flux_transport_step (4463) ->
! hipft_gpu_flux_transport_step, apply_data_assimilation (4148) ->
! hipft_gpu_assimilate, analysis_step (3098) -> hipft_gpu_analysis, and so on
! (the call-site table is in INTEGRATION.md).  Every function returns 0 on
! success; on a nonzero status the driver calls hipft_gpu_last_error and
! endrun(.true.), as the reference does on its own errors (970-1004).
!
! Arrays cross the ABI in the reference's layout: f(ntm,npm,nr) theta
! fastest with the two-point phi overlap, assimilation maps (npm1,ntm,3).
! The derived types below mirror the C structs field for field; the CPU
! test tests/test_fortran_layout.py checks their layouts against the header.
!
module hipft_gpu_c
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: HIPFT_OK = 0, HIPFT_EINVAL = 1, HIPFT_ECUDA = 2, &
                               HIPFT_ETIMEOUT = 3, HIPFT_ENAN = 4, HIPFT_ESTATE = 5, &
                               HIPFT_EIO = 6, HIPFT_ENOMEM = 7, HIPFT_ECOMM = 8
  integer(c_int), parameter :: HIPFT_RED_MIN = 0, HIPFT_RED_MAX = 1

  type, bind(c) :: hipft_grid
    integer(c_int) :: ntm, npm1, nr, device
    type(c_ptr) :: t, p
  end type

  type, bind(c) :: hipft_params
    integer(c_int) :: advance_flow, flow_num_method
    real(c_double) :: upwind, weno_eps
    integer(c_int) :: strang_splitting, advance_diffusion, diffusion_num_method
    integer(c_int) :: diffusion_subcycles, diffusion_coef_grid
    real(c_double) :: diffusion_coef_factor
    type(c_ptr) :: diffusion_coef_constants
    real(c_double) :: pole_flux_lat_limit
    integer(c_int) :: verbose, advance_source
  end type

  type, bind(c) :: hipft_flow_def
    integer(c_int) :: flow_dr_model, flow_mf_model
    type(c_ptr) :: dr_p0, dr_p2, dr_p4, mf_p1, mf_p3, mf_p5
    real(c_double) :: flow_vp_rigid_omega, flow_vt_const, flow_rigid_omega
    integer(c_int) :: flow_attenuate
    type(c_ptr) :: flow_attenuate_values
  end type

  type, bind(c) :: hipft_da_opts
    integer(c_int) :: add, custom_from_mu, balance_flux
    real(c_double) :: mult_fac
    type(c_ptr) :: mu_power, mu_limit, lat_limit
  end type

  type, bind(c) :: hipft_diffusion_info
    real(c_double) :: dtime_diffusion_euler
    integer(c_int64_t) :: sts_s, subcycles, total_stages
  end type

  type, bind(c) :: hipft_info
    integer(c_int) :: ntm, npm, nr, ldt
    real(c_double) :: dtime_diffusion_euler
    integer(c_int64_t) :: sts_s, kernel_launches, cell_stage_updates
    integer(c_size_t) :: device_bytes
    integer(c_int64_t) :: rkg2_stages, rkg2_cell_stages
  end type

  type, bind(c) :: hipft_shard
    integer(c_int) :: rank, nranks
    type(c_funptr) :: allreduce, gather
    type(c_ptr) :: user
  end type

  interface

    ! ---- lifecycle (setup: set_mesh 6495, load_flows 2535, load_weno 6846,
    !      load_diffusion 6655, get_dtime_diffusion_euler 4985)
    integer(c_int) function hipft_gpu_create(grid, params, h) bind(c, name="hipft_gpu_create")
      import :: c_int, c_ptr, hipft_grid, hipft_params
      type(hipft_grid), intent(in) :: grid
      type(hipft_params), intent(in) :: params
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function hipft_gpu_destroy(h) bind(c, name="hipft_gpu_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function hipft_gpu_last_error(h, buf, len) bind(c, name="hipft_gpu_last_error")
      import :: c_int, c_ptr, c_char, c_size_t
      type(c_ptr), value :: h
      character(kind=c_char) :: buf(*)
      integer(c_size_t), value :: len
    end function

    ! ---- field I/O (2159, 2844; load_initial_condition 2116-2172)
    integer(c_int) function hipft_gpu_set_field(h, f) bind(c, name="hipft_gpu_set_field")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: f(*)
    end function
    integer(c_int) function hipft_gpu_get_field(h, f) bind(c, name="hipft_gpu_get_field")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: f(*)
    end function
    integer(c_int) function hipft_gpu_load_initial_map(h, map_pt, flux_balance, mult_fac) &
        bind(c, name="hipft_gpu_load_initial_map")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: map_pt(*)
      integer(c_int), value :: flux_balance
      real(c_double), value :: mult_fac
    end function

    ! ---- ranks (MPI reductions 5036, 5103, 5141, 7345)
    integer(c_int) function hipft_gpu_set_allreduce(h, cb, user) bind(c, name="hipft_gpu_set_allreduce")
      import :: c_int, c_ptr, c_funptr
      type(c_ptr), value :: h
      type(c_funptr), value :: cb
      type(c_ptr), value :: user
    end function

    ! ---- flows (update_flow 3371, add_flow_from_files 3525, get_flow_dtmax 7287)
    integer(c_int) function hipft_gpu_set_flow(h, def) bind(c, name="hipft_gpu_set_flow")
      import :: c_int, c_ptr, hipft_flow_def
      type(c_ptr), value :: h
      type(hipft_flow_def), intent(in) :: def
    end function
    integer(c_int) function hipft_gpu_update_flow(h, updated) bind(c, name="hipft_gpu_update_flow")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), intent(out) :: updated
    end function
    integer(c_int) function hipft_gpu_set_flow_from_files(h, vt_pt, vp_pt, at_load) &
        bind(c, name="hipft_gpu_set_flow_from_files")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: vt_pt(*), vp_pt(*)
      integer(c_int), value :: at_load
    end function
    integer(c_int) function hipft_gpu_flow_dtmax(h, dtmax) bind(c, name="hipft_gpu_flow_dtmax")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: dtmax
    end function

    ! ---- sources (load_source 7050, generate_rfe 8809, update_source 3875,
    !      source_step 4697)
    integer(c_int) function hipft_gpu_set_source_file(h, data_tp) bind(c, name="hipft_gpu_set_source_file")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: data_tp(*)
    end function
    integer(c_int) function hipft_gpu_set_rfe_frame(h, slot, model, rnd_tp, uf) &
        bind(c, name="hipft_gpu_set_rfe_frame")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: slot, model
      real(c_double), intent(in) :: rnd_tp(*), uf(*)
    end function
    integer(c_int) function hipft_gpu_update_source(h, use_file, use_rfe, slot1, slot2, alpha) &
        bind(c, name="hipft_gpu_update_source")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: use_file, use_rfe, slot1, slot2
      real(c_double), value :: alpha
    end function
    integer(c_int) function hipft_gpu_source_step(h, dt) bind(c, name="hipft_gpu_source_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
    end function

    ! ---- the time step (advection_step 4509, diffusion_step 4551,
    !      flux_transport_step 4463)
    integer(c_int) function hipft_gpu_advection_step(h, dt) bind(c, name="hipft_gpu_advection_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: dt
    end function
    integer(c_int) function hipft_gpu_diffusion_step(h, dt, cb, user, info) bind(c, name="hipft_gpu_diffusion_step")
      import :: c_int, c_ptr, c_double, c_funptr, hipft_diffusion_info
      type(c_ptr), value :: h
      real(c_double), value :: dt
      type(c_funptr), value :: cb
      type(c_ptr), value :: user
      type(hipft_diffusion_info), intent(out) :: info
    end function
    integer(c_int) function hipft_gpu_flux_transport_step(h, dt, cb, user, info) &
        bind(c, name="hipft_gpu_flux_transport_step")
      import :: c_int, c_ptr, c_double, c_funptr, hipft_diffusion_info
      type(c_ptr), value :: h
      real(c_double), value :: dt
      type(c_funptr), value :: cb
      type(c_ptr), value :: user
      type(hipft_diffusion_info), intent(out) :: info
    end function

    ! ---- data assimilation (assimilate_new_data 4083, apply_data_assimilation 4148)
    integer(c_int) function hipft_gpu_assimilate(h, data3_pt, opts) bind(c, name="hipft_gpu_assimilate")
      import :: c_int, c_ptr, c_double, hipft_da_opts
      type(c_ptr), value :: h
      real(c_double), intent(in) :: data3_pt(*)
      type(hipft_da_opts), intent(in) :: opts
    end function

    ! ---- diagnostics (analysis_step 3098, get_flux 8672, balance_flux 8752)
    integer(c_int) function hipft_gpu_set_validation(h, mode, fval_u0_pt, width, vt_const, vp_omega, time_start) &
        bind(c, name="hipft_gpu_set_validation")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: mode
      real(c_double), intent(in) :: fval_u0_pt(*)
      real(c_double), value :: width, vt_const, vp_omega, time_start
    end function
    integer(c_int) function hipft_gpu_analysis(h, time, hist) bind(c, name="hipft_gpu_analysis")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: time
      real(c_double), intent(out) :: hist(*)
    end function
    integer(c_int) function hipft_gpu_get_flux(h, flux_p, flux_m) bind(c, name="hipft_gpu_get_flux")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: flux_p(*), flux_m(*)
    end function
    integer(c_int) function hipft_gpu_balance_flux(h) bind(c, name="hipft_gpu_balance_flux")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function hipft_gpu_info(h, info) bind(c, name="hipft_gpu_info")
      import :: c_int, c_ptr, hipft_info
      type(c_ptr), value :: h
      type(hipft_info), intent(out) :: info
    end function

    ! ---- ragged batches (no reference counterpart)
    integer(c_int) function hipft_gpu_set_ragged(h, on) bind(c, name="hipft_gpu_set_ragged")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: on
    end function
    ! ---- each step as one CUDA-graph launch (no reference counterpart)
    integer(c_int) function hipft_gpu_set_graph(h, on) bind(c, name="hipft_gpu_set_graph")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: on
    end function
    integer(c_int) function hipft_gpu_flow_dtmax_each(h, dtmax) bind(c, name="hipft_gpu_flow_dtmax_each")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: dtmax(*)
    end function
    integer(c_int) function hipft_gpu_ragged_schedule(h, sts_s, subcycles, adv_substeps, dt_euler) &
        bind(c, name="hipft_gpu_ragged_schedule")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: h
      integer(c_int64_t), intent(out) :: sts_s(*), subcycles(*), adv_substeps(*)
      real(c_double), intent(out) :: dt_euler(*)
    end function

    ! ---- allocation-free flux integral of a caller-owned device field
    integer(c_int) function hipft_get_flux_noalloc(f_dev, ntm, npm1, nr, ldt, t, p, flux_p, flux_m, &
                                                   cuda_stream, err, err_len) bind(c, name="hipft_get_flux_noalloc")
      import :: c_int, c_ptr, c_double, c_char, c_size_t
      type(c_ptr), value :: f_dev
      integer(c_int), value :: ntm, npm1, nr, ldt
      real(c_double), intent(in) :: t(*), p(*)
      real(c_double), intent(out) :: flux_p(*), flux_m(*)
      type(c_ptr), value :: cuda_stream
      character(kind=c_char) :: err(*)
      integer(c_size_t), value :: err_len
    end function

    ! ---- map files (rdh5 5678, wrh5 6155)
    integer(c_int) function hipft_h5_read(path, ndim, dims, data, s1, s2, s3) bind(c, name="hipft_h5_read")
      import :: c_int, c_char, c_int64_t, c_ptr
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), intent(out) :: ndim
      integer(c_int64_t), intent(out) :: dims(3)
      type(c_ptr), value :: data, s1, s2, s3
    end function
    integer(c_int) function hipft_h5_write(path, ndim, dims, data, s1, s2, s3, single_precision) &
        bind(c, name="hipft_h5_write")
      import :: c_int, c_char, c_int64_t, c_double, c_ptr
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), value :: ndim
      integer(c_int64_t), intent(in) :: dims(3)
      real(c_double), intent(in) :: data(*)
      type(c_ptr), value :: s1, s2, s3
      integer(c_int), value :: single_precision
    end function

  end interface

end module hipft_gpu_c
