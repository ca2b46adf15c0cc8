! mrlbm_gpu.f90 -- ISO_C_BINDING interface of include/mrlbm.h for a Fortran host.
!
! The reference's time loop (2d_mrlbm.f90:229-535) keeps its own input, output and control
! flow and calls the B200 step through these interfaces: create a handle after get_coord and
! initialize (2d_mrlbm.f90:83-214), mrlbm_load_state when restarting (read_restart_file,
! 2d_mrlbm.f90:2204-2220), one mrlbm_step per iteration in place of the body
! 2d_mrlbm.f90:231-535, and the getters before the files are written (write_function_plot3d
! 2d_mrlbm.f90:371-386, write_restart_file 2d_mrlbm.f90:2186-2202, forces_time.dat
! 2d_mrlbm.f90:492-494).  Compile with the host program, link with -L<dir> -lmrlbm.
!
! Type layouts are part of the C ABI: the components of mrlbm_config and mrlbm_geometry_info
! below are in the order, kinds and alignment of the C structs (tests/test_cpu_fortran_module.py
! checks the offsets against the C compiler's).  Unsigned C fields map to the signed Fortran
! integer of the same size.
module mrlbm_gpu
  use iso_c_binding
  implicit none

  ! status codes
  integer(c_int), parameter :: MRLBM_OK = 0, MRLBM_EINVAL = 1, MRLBM_ENAMELIST = 2
  integer(c_int), parameter :: MRLBM_EGEOMETRY = 3, MRLBM_EUNSUPPORTED = 4, MRLBM_ESTATE = 5
  integer(c_int), parameter :: MRLBM_ECUDA = -1, MRLBM_EDEVICE_NAN = -2, MRLBM_ENODEVICE = -3
  integer(c_int), parameter :: MRLBM_EDEVICE_TIMEOUT = -4
  ! precision of a handle, step flags
  integer(c_int), parameter :: MRLBM_FP64 = 64, MRLBM_FP32 = 32
  integer(c_int32_t), parameter :: MRLBM_STEP_MACRO = 1
  ! extension switches (0 is always the reference behaviour)
  integer(c_int32_t), parameter :: MRLBM_GEOM_REFERENCE = 0, MRLBM_GEOM_EXPLICIT = 1
  integer(c_int32_t), parameter :: MRLBM_WALL_REFERENCE = 0, MRLBM_WALL_FREESLIP = 1
  integer(c_int32_t), parameter :: MRLBM_LABEL15_REJECT = 0, MRLBM_LABEL15_ALLNINE = 1
  integer(c_int32_t), parameter :: MRLBM_NU_REFERENCE = 0, MRLBM_NU_DIAMETER = 1
  integer(c_int32_t), parameter :: MRLBM_INIT_REFERENCE = 0, MRLBM_INIT_NOISE = 1
  ! batch schedules (mrlbm_batch_set_schedule)
  integer(c_int32_t), parameter :: MRLBM_BATCH_PERSISTENT = 0, MRLBM_BATCH_GRAPH = 1, MRLBM_BATCH_STREAMS = 2

  ! struct mrlbm_config: the namelists DomainSize, Cylinder, Numbers, Parallel, Controls and
  ! LogicalControls (2d_mrlbm.f90:2227-2233) plus the extension switches
  type, bind(c) :: mrlbm_config
     real(c_double) :: x_c
     real(c_double) :: y_c
     real(c_double) :: r_c
     real(c_double) :: Re
     real(c_double) :: uo
     real(c_double) :: rho_infty
     real(c_double) :: noise_amp
     integer(c_int64_t) :: seed
     integer(c_int32_t) :: nx
     integer(c_int32_t) :: ny
     integer(c_int32_t) :: channel_with_cylinder
     integer(c_int32_t) :: ncy
     integer(c_int32_t) :: L_front
     integer(c_int32_t) :: L_back
     integer(c_int32_t) :: L_top
     integer(c_int32_t) :: L_bot
     integer(c_int32_t) :: iplot
     integer(c_int32_t) :: max_iter
     integer(c_int32_t) :: isave
     integer(c_int32_t) :: irestart
     integer(c_int32_t) :: statsbegin
     integer(c_int32_t) :: statsend
     integer(c_int32_t) :: iplotstats
     integer(c_int32_t) :: num_threads
     integer(c_int32_t) :: lattice_type
     integer(c_int32_t) :: post_process
     integer(c_int32_t) :: x_periodic
     integer(c_int32_t) :: y_periodic
     integer(c_int32_t) :: channel_with_square
     integer(c_int32_t) :: incomp_bc
     integer(c_int32_t) :: incomp_bulk
     integer(c_int32_t) :: vel_interp
     integer(c_int32_t) :: mom_interp
     integer(c_int32_t) :: rotated_coordinate
     integer(c_int32_t) :: strong_mass_bc
     integer(c_int32_t) :: eq_mass_bc
     integer(c_int32_t) :: weak_mass_bc
     integer(c_int32_t) :: geometry_mode
     integer(c_int32_t) :: wall_mode
     integer(c_int32_t) :: label15_rule
     integer(c_int32_t) :: nu_length
     integer(c_int32_t) :: init_mode
     integer(c_int32_t) :: reserved
  end type mrlbm_config

  ! struct mrlbm_geometry_info (get_coord's results, 2d_mrlbm.f90:931-1156, and the layout)
  type, bind(c) :: mrlbm_geometry_info
     integer(c_int32_t) :: nx
     integer(c_int32_t) :: ny
     integer(c_int32_t) :: nbct
     integer(c_int32_t) :: n_label15
     real(c_double) :: x_c
     real(c_double) :: y_c
     real(c_double) :: r_c
     real(c_double) :: r_cyl
     real(c_double) :: nu
     real(c_double) :: omega
     integer(c_int32_t) :: pitch
     integer(c_int32_t) :: off
     integer(c_int64_t) :: plane
     integer(c_int64_t) :: state_bytes
  end type mrlbm_geometry_info

  interface
     integer(c_size_t) function mrlbm_config_sizeof() bind(c)
       import
     end function
     integer(c_int) function mrlbm_config_defaults(cfg) bind(c)
       import
       type(mrlbm_config) :: cfg
     end function
     ! path: a NUL-terminated string, e.g. 'input.dat'//c_null_char
     integer(c_int) function mrlbm_config_from_namelist(path, cfg) bind(c)
       import
       character(kind=c_char), dimension(*) :: path
       type(mrlbm_config) :: cfg
     end function
     integer(c_int) function mrlbm_config_resolve_geometry(cfg) bind(c)
       import
       type(mrlbm_config) :: cfg
     end function
     integer(c_int) function mrlbm_create(cfg, precision, device, h) bind(c)
       import
       type(mrlbm_config), intent(in) :: cfg
       integer(c_int), value :: precision, device
       type(c_ptr) :: h
     end function
     integer(c_int) function mrlbm_destroy(h) bind(c)
       import
       type(c_ptr), value :: h
     end function
     integer(c_int) function mrlbm_last_error(h, buf, len) bind(c)
       import
       type(c_ptr), value :: h
       character(kind=c_char), dimension(*) :: buf
       integer(c_size_t), value :: len
     end function
     integer(c_int) function mrlbm_status(h) bind(c)
       import
       type(c_ptr), value :: h
     end function
     integer(c_int) function mrlbm_set_stream(h, stream) bind(c)
       import
       type(c_ptr), value :: h, stream
     end function
     integer(c_int) function mrlbm_get_geometry_info(h, info) bind(c)
       import
       type(c_ptr), value :: h
       type(mrlbm_geometry_info) :: info
     end function
     integer(c_int) function mrlbm_get_boundary_nodes(h, bou_i, bou_j, label_bc, delta_uk, ref_xy, stencil) bind(c)
       import
       type(c_ptr), value :: h, bou_i, bou_j, label_bc, delta_uk, ref_xy, stencil
     end function
     integer(c_int) function mrlbm_get_node_classes(h, isfluid, issolid, isbound) bind(c)
       import
       type(c_ptr), value :: h, isfluid, issolid, isbound
     end function
     ! f(nx,ny,0:8) exactly as the reference's f(1:nx,1:ny,0:q-1) (2d_mrlbm.f90:2285)
     integer(c_int) function mrlbm_load_state(h, f, iter) bind(c)
       import
       type(c_ptr), value :: h
       real(c_double), intent(in) :: f(*)
       integer(c_int32_t), value :: iter
     end function
     integer(c_int) function mrlbm_get_state(h, f) bind(c)
       import
       type(c_ptr), value :: h
       real(c_double) :: f(*)
     end function
     integer(c_int) function mrlbm_set_inlet_profile(h, u_in) bind(c)
       import
       type(c_ptr), value :: h, u_in
     end function
     integer(c_int) function mrlbm_step(h, nsteps, flags) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t), value :: nsteps, flags
     end function
     integer(c_int) function mrlbm_get_iter(h, iter) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t) :: iter
     end function
     ! pass c_null_ptr for the fields not wanted; c_loc(array) for the others
     integer(c_int) function mrlbm_get_macro(h, rho, ux, uy, mxx, myy, mxy) bind(c)
       import
       type(c_ptr), value :: h, rho, ux, uy, mxx, myy, mxy
     end function
     integer(c_int) function mrlbm_get_forces(h, iter, f_drag, f_lift, rho_inlet_sum, cap, n) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t) :: iter(*)
       real(c_double) :: f_drag(*), f_lift(*), rho_inlet_sum(*)
       integer(c_int32_t), value :: cap
       integer(c_int32_t) :: n
     end function
     integer(c_int) function mrlbm_force_statistics(f_drag, f_lift, nstep, r_cy, uo, rho_infty, St, Cd_mean, Cl_rms, &
                                                    cycle_start, period, n_cycle) bind(c)
       import
       real(c_double), intent(in) :: f_drag(*), f_lift(*)
       integer(c_int32_t), value :: nstep
       real(c_double), value :: r_cy, uo, rho_infty
       real(c_double) :: St, Cd_mean, Cl_rms
       integer(c_int32_t) :: cycle_start, period, n_cycle
     end function
     integer(c_int) function mrlbm_cp_statistics(p_surface, nstep, nbct, cycle_start, period, n_cycle, rho_infty, uo, &
                                                 cp) bind(c)
       import
       real(c_double), intent(in) :: p_surface(*)
       integer(c_int32_t), value :: nstep, nbct, cycle_start, period, n_cycle
       real(c_double), value :: rho_infty, uo
       real(c_double) :: cp(*)
     end function
     integer(c_int) function mrlbm_step_noalloc(h, d_state, d_f0, nsteps, records, n_records, stream) bind(c)
       import
       type(c_ptr), value :: h, d_state, d_f0
       integer(c_int32_t), value :: nsteps
       real(c_double) :: records(*)
       integer(c_int32_t) :: n_records
       type(c_ptr), value :: stream
     end function
     integer(c_int) function mrlbm_set_tile_config(h, cfg) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t), value :: cfg
     end function
     integer(c_int) function mrlbm_autotune(h, trial_steps, best_cfg, best_ms) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t), value :: trial_steps
       integer(c_int32_t) :: best_cfg
       real(c_double) :: best_ms
     end function
     integer(c_int) function mrlbm_field_stats_window(h, begin_iter, end_iter) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t), value :: begin_iter, end_iter
     end function
     integer(c_int) function mrlbm_field_stats_get(h, mean_u, mean_v, mean_p, rms_u, rms_v, rms_p, n_samples) bind(c)
       import
       type(c_ptr), value :: h, mean_u, mean_v, mean_p, rms_u, rms_v, rms_p
       integer(c_int64_t) :: n_samples
     end function
     integer(c_int) function mrlbm_surface_enable(h, enable) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t), value :: enable
     end function
     integer(c_int) function mrlbm_get_surface(h, iter, p_surface, p_smooth, probes, cap, n) bind(c)
       import
       type(c_ptr), value :: h, iter, p_surface, p_smooth, probes
       integer(c_int32_t), value :: cap
       integer(c_int32_t) :: n
     end function
     integer(c_int) function mrlbm_set_body_force(h, g) bind(c)
       import
       type(c_ptr), value :: h, g
     end function
     integer(c_int) function mrlbm_adjoint_drag(h, nsteps, window, checkpoint_every, J, grad_body, grad_uin) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t), value :: nsteps, window, checkpoint_every
       real(c_double) :: J
       type(c_ptr), value :: grad_body, grad_uin
     end function
     integer(c_int) function mrlbm_get_tile_config(h, cfg) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t) :: cfg
     end function
     integer(c_int) function mrlbm_get_probe_nodes(h, pi, pj) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int32_t), dimension(*) :: pi, pj
     end function
     integer(c_int) function mrlbm_get_launch_count(h, n) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int64_t) :: n
     end function
     ! x-slabs of one domain: global columns gx0..gx1 of the case, faces exchanged by the host
     integer(c_int) function mrlbm_create_slab(cfg, precision, device, gx0, gx1, h) bind(c)
       import
       type(mrlbm_config), intent(in) :: cfg
       integer(c_int), value :: precision, device
       integer(c_int32_t), value :: gx0, gx1
       type(c_ptr) :: h
     end function
     integer(c_int) function mrlbm_halo_size(h, n_values, elem_bytes) bind(c)
       import
       type(c_ptr), value :: h
       integer(c_int64_t) :: n_values
       integer(c_int32_t) :: elem_bytes
     end function
     integer(c_int) function mrlbm_halo_pack(h, side, dst) bind(c)
       import
       type(c_ptr), value :: h, dst
       integer(c_int32_t), value :: side
     end function
     integer(c_int) function mrlbm_halo_unpack(h, side, src) bind(c)
       import
       type(c_ptr), value :: h, src
       integer(c_int32_t), value :: side
     end function
     integer(c_int) function mrlbm_step_faces(h) bind(c)
       import
       type(c_ptr), value :: h
     end function
     integer(c_int) function mrlbm_halo_pack_next(h, side, dst) bind(c)
       import
       type(c_ptr), value :: h, dst
       integer(c_int32_t), value :: side
     end function
     integer(c_int) function mrlbm_halo_unpack_next(h, side, src) bind(c)
       import
       type(c_ptr), value :: h, src
       integer(c_int32_t), value :: side
     end function
     ! hs: an array of n slab handles, left to right
     integer(c_int) function mrlbm_slabs_step(hs, n, nsteps) bind(c)
       import
       type(c_ptr), dimension(*) :: hs
       integer(c_int32_t), value :: n, nsteps
     end function
     ! batched cases: cfgs is an array of ncases configurations
     integer(c_int) function mrlbm_batch_create(cfgs, ncases, precision, device, b) bind(c)
       import
       type(mrlbm_config), dimension(*), intent(in) :: cfgs
       integer(c_int32_t), value :: ncases
       integer(c_int), value :: precision, device
       type(c_ptr) :: b
     end function
     integer(c_int) function mrlbm_batch_destroy(b) bind(c)
       import
       type(c_ptr), value :: b
     end function
     integer(c_int) function mrlbm_batch_case(b, c, h) bind(c)
       import
       type(c_ptr), value :: b
       integer(c_int32_t), value :: c
       type(c_ptr) :: h
     end function
     integer(c_int) function mrlbm_batch_step(b, nsteps, flags) bind(c)
       import
       type(c_ptr), value :: b
       integer(c_int32_t), value :: nsteps, flags
     end function
     integer(c_int) function mrlbm_batch_set_schedule(b, tile_cfg, schedule, steps_per_launch) bind(c)
       import
       type(c_ptr), value :: b
       integer(c_int32_t), value :: tile_cfg, schedule, steps_per_launch
     end function
     integer(c_int) function mrlbm_batch_get_schedule(b, tile_cfg, schedule, steps_per_launch) bind(c)
       import
       type(c_ptr), value :: b
       integer(c_int32_t) :: tile_cfg, schedule, steps_per_launch
     end function
     integer(c_int) function mrlbm_batch_autotune(b, trial_steps, best_ms_per_step) bind(c)
       import
       type(c_ptr), value :: b
       integer(c_int32_t), value :: trial_steps
       real(c_double) :: best_ms_per_step
     end function
     integer(c_int) function mrlbm_batch_set_wait_limit(b, polls) bind(c)
       import
       type(c_ptr), value :: b
       integer(c_int64_t), value :: polls
     end function
     integer(c_int) function mrlbm_batch_status(b) bind(c)
       import
       type(c_ptr), value :: b
     end function
     integer(c_int) function mrlbm_batch_last_error(b, buf, len) bind(c)
       import
       type(c_ptr), value :: b
       character(kind=c_char), dimension(*) :: buf
       integer(c_size_t), value :: len
     end function
     integer(c_int) function mrlbm_batch_launch_count(b, n) bind(c)
       import
       type(c_ptr), value :: b
       integer(c_int64_t) :: n
     end function
     integer(c_int) function mrlbm_batch_get_stream(b, stream) bind(c)
       import
       type(c_ptr), value :: b
       type(c_ptr) :: stream
     end function
  end interface
end module mrlbm_gpu
