! =====================================================================
!     eup_mod -- iso_c_binding interface to the B200 D3Q19 BGK step
!
!     Declares the C ABI of include/eup.h for the Fortran driver of
!     Euplectella_HPC (CODE/SRC/bgk3d.F90).  With this module the driver
!     keeps its namelist, its arrays a01..a19(0:l+1,0:m+1,0:n+1) and all of
!     its output routines; only the calls of the time loop change (in
!     bgk3d.F90, initialize.F90 and diagnostic.F90).  Same pattern as the
!     reference's own C interop in CODE/SRC/get_mem_mod.F90:1-10.
! =====================================================================
      module eup_mod
      use iso_c_binding
      implicit none

      integer(c_int), parameter :: EUP_OK = 0
      integer(c_int), parameter :: EUP_FP32 = 0, EUP_FP64 = 1
      integer(c_int), parameter :: EUP_FP16_DEV = 2, EUP_BF16_DEV = 3

      type, bind(c) :: eup_config
         integer(c_int32_t) :: lx, ly, lz
         integer(c_int32_t) :: bc(6)        ! front, rear, right, left, up, down
         real(c_double)     :: svisc, u0, u_inflow, u00
         integer(c_int32_t) :: precision, device
         real(c_double)     :: dev_scale
         real(c_double)     :: cd_rho0, cd_uref, cd_length, cd_span
         integer(c_int64_t) :: series_capacity
      end type eup_config

      ! voxel shapes of eup_geometry%kind and the variant bits of eup_geometry_reference
      integer(c_int), parameter :: EUP_GEOM_NONE = 0, EUP_GEOM_REF_SPHERE = 1, EUP_GEOM_REF_COLUMN = 2
      integer(c_int), parameter :: EUP_GEOM_CYLINDER_Z = 3, EUP_GEOM_RETICULAR_SHELL = 4
      integer(c_int), parameter :: EUP_GEOM_RIDGED_SHELL = 5
      integer(c_int), parameter :: EUP_GEOM_VARIANT_CYLINDER_INF = 1, EUP_GEOM_VARIANT_TEST1 = 2

      type, bind(c) :: eup_geometry
         integer(c_int32_t) :: kind
         integer(c_int32_t) :: offset(3)      ! mpicoords(d) * (l, m, n), as build_obs
         integer(c_int32_t) :: center(3), kstop
         integer(c_int64_t) :: r2_lo, r2_hi
         real(c_double)     :: xc, yc, zc, radius
         real(c_double)     :: x0, length, outer_d, strut_d, pitch
         real(c_double)     :: ridge_h, ridge_t, cap_t, pore_d
         integer(c_int64_t) :: seed
      end type eup_geometry

      type, bind(c) :: eup_adjoint_config
         integer(c_int32_t) :: nsteps, avg_steps, checkpoints, reserved
      end type eup_adjoint_config

      interface
         integer(c_int) function eup_create(cfg, h) bind(c, name="eup_create")
            import :: c_int, c_ptr, eup_config
            type(eup_config), intent(in) :: cfg
            type(c_ptr), intent(out)     :: h
         end function

         integer(c_int) function eup_destroy(h) bind(c, name="eup_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
         end function

         integer(c_int) function eup_set_obstacles(h, obs) bind(c, name="eup_set_obstacles")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            type(c_ptr), value :: obs             ! c_loc(obs(1,1,1))
         end function

         integer(c_int) function eup_upload(h, pops, elem_bytes, itime) bind(c, name="eup_upload")
            import :: c_int, c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value          :: h
            type(c_ptr), intent(in)     :: pops(19)    ! c_loc(a01(0,0,0)) ... c_loc(a19(0,0,0))
            integer(c_int32_t), value   :: elem_bytes  ! 4 (sp) or 8 (-DDOUBLE_P)
            integer(c_int64_t), value   :: itime
         end function

         integer(c_int) function eup_download(h, pops, elem_bytes) bind(c, name="eup_download")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value          :: h
            type(c_ptr), intent(in)     :: pops(19)
            integer(c_int32_t), value   :: elem_bytes
         end function

         integer(c_int) function eup_step(h, nsteps) bind(c, name="eup_step")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: nsteps
         end function

         integer(c_int) function eup_get_forces(h, fxyz) bind(c, name="eup_get_forces")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value    :: h
            real(c_double)        :: fxyz(3)
         end function

         integer(c_int) function eup_get_cd_series(h, first, cnt, cd) bind(c, name="eup_get_cd_series")
            import :: c_int, c_ptr, c_int64_t, c_int32_t, c_double
            type(c_ptr), value        :: h
            integer(c_int64_t), value :: first
            integer(c_int32_t), value :: cnt
            real(c_double)            :: cd(*)
         end function

         integer(c_int) function eup_get_monitor(h, sums) bind(c, name="eup_get_monitor")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double)     :: sums(5)
         end function

         type(c_ptr) function eup_last_error(h) bind(c, name="eup_last_error")
            import :: c_ptr
            type(c_ptr), value :: h
         end function

         integer(c_int) function eup_step_profiled(h, nsteps, ms) bind(c, name="eup_step_profiled")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: nsteps
            real(c_double)            :: ms(4)
         end function

         integer(c_int) function eup_get_probes(h, npts, ijk, rho_u) bind(c, name="eup_get_probes")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: npts
            integer(c_int32_t)        :: ijk(3, *)
            real(c_double)            :: rho_u(4, *)
         end function

         integer(c_int) function eup_get_region_sums(h, region, sums) bind(c, name="eup_get_region_sums")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            type(c_ptr), value :: region            ! c_loc of an integer(c_int8_t) mask(l,m,n)
            real(c_double)     :: sums(6)
         end function

         integer(c_int) function eup_init_state(h, u_in, amp, seed, itime) bind(c, name="eup_init_state")
            import :: c_int, c_ptr, c_double, c_int64_t
            type(c_ptr), value         :: h
            real(c_double), value      :: u_in, amp
            integer(c_int64_t), value  :: seed, itime
         end function

         integer(c_int) function eup_set_solid_fraction(h, ns) bind(c, name="eup_set_solid_fraction")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            type(c_ptr), value :: ns                ! c_loc of real(c_double) ns(l,m,n), or c_null_ptr
         end function

         integer(c_int) function eup_adjoint_run(h, cfg, objective, grad_ns, stats) bind(c, name="eup_adjoint_run")
            import :: c_int, c_ptr, c_double, eup_adjoint_config
            type(c_ptr), value            :: h
            type(eup_adjoint_config)      :: cfg
            real(c_double)                :: objective
            real(c_double)                :: grad_ns(*)
            real(c_double)                :: stats(8)
         end function

         ! checkpoint schedule of eup_adjoint_run for nsteps steps and checkpoints states (host only)
         integer(c_int) function eup_adjoint_plan(nsteps, checkpoints, forward_steps, recomputed, repetitions) &
               bind(c, name="eup_adjoint_plan")
            import :: c_int, c_int32_t, c_int64_t
            integer(c_int32_t), value :: nsteps, checkpoints
            integer(c_int64_t)        :: forward_steps, recomputed
            integer(c_int32_t)        :: repetitions
         end function

         ! x-slab step (one GPU per slab): boundaries, planes out, interior | exchange, planes in, faces
         integer(c_int) function eup_step_boundaries(h) bind(c, name="eup_step_boundaries")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
         end function

         integer(c_int) function eup_step_stream(h) bind(c, name="eup_step_stream")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
         end function

         integer(c_int) function eup_step_stream_interior(h) bind(c, name="eup_step_stream_interior")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
         end function

         integer(c_int) function eup_step_stream_faces(h) bind(c, name="eup_step_stream_faces")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
         end function

         integer(c_int) function eup_get_x_planes(h, side, dst) bind(c, name="eup_get_x_planes")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: side          ! 0: x = 1 (to the left), 1: x = l (to the right)
            type(c_ptr), value        :: dst           ! device buffer, 5 (m+2)(n+2) reals
         end function

         integer(c_int) function eup_set_x_planes(h, side, src) bind(c, name="eup_set_x_planes")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: side
            type(c_ptr), value        :: src
         end function

         integer(c_int) function eup_get_x_planes_view(h, side, dev) bind(c, name="eup_get_x_planes_view")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: side
            type(c_ptr)               :: dev           ! out: device address, 5 (m+2)(n+2) reals
         end function

         integer(c_int) function eup_set_x_planes_view(h, side, src) bind(c, name="eup_set_x_planes_view")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: side
            type(c_ptr), value        :: src
         end function

         integer(c_int) function eup_init_reference(opt, l, m, n, glob, start, periodic, u0, elem_bytes, &
                                                     pops) bind(c, name="eup_init_reference")
            import :: c_int, c_int32_t, c_double, c_ptr
            integer(c_int32_t), value   :: opt, l, m, n   ! opt = init_v
            integer(c_int32_t)          :: glob(3), start(3)  ! (lx,ly,lz), mpicoords*(l,m,n)
            integer(c_int32_t), value   :: periodic       ! 1 for the -DPERIODIC coordinates
            real(c_double), value       :: u0
            integer(c_int32_t), value   :: elem_bytes
            type(c_ptr), intent(in)     :: pops(19)       ! c_loc(a01(0,0,0)) ... c_loc(a19(0,0,0))
         end function

         integer(c_int) function eup_geometry_reference(flag2, lx, ly, lz, variant, g) &
                                 bind(c, name="eup_geometry_reference")
            import :: c_int, c_int32_t, eup_geometry
            integer(c_int32_t), value :: flag2, lx, ly, lz, variant
            type(eup_geometry)        :: g
         end function

         integer(c_int) function eup_build_obstacles(h, g) bind(c, name="eup_build_obstacles")
            import :: c_int, c_ptr, eup_geometry
            type(c_ptr), value             :: h
            type(eup_geometry), intent(in) :: g
         end function

         integer(c_int) function eup_get_obstacles(h, obs, nobs) bind(c, name="eup_get_obstacles")
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: h
            type(c_ptr), value :: obs               ! c_loc(obs(1,1,1)) or c_null_ptr
            integer(c_int64_t) :: nobs
         end function

         integer(c_int) function eup_write_obstacles(h, path) bind(c, name="eup_write_obstacles")
            import :: c_int, c_ptr, c_char
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: path(*)   ! 'obs.0000.00000000.bin'//c_null_char
         end function

         integer(c_int) function eup_voxelise(g, l, m, n, obs) bind(c, name="eup_voxelise")
            import :: c_int, c_int32_t, c_ptr, eup_geometry
            type(eup_geometry), intent(in) :: g
            integer(c_int32_t), value      :: l, m, n
            type(c_ptr), value             :: obs
         end function

         integer(c_int) function eup_read_obs_file(path, l, m, n, obs, nobs) bind(c, name="eup_read_obs_file")
            import :: c_int, c_char, c_int32_t, c_ptr, c_int64_t
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int32_t), value :: l, m, n
            type(c_ptr), value        :: obs
            integer(c_int64_t)        :: nobs
         end function

         ! ---- the remaining entry points of include/eup.h ----
         integer(c_int32_t) function eup_abi_version() bind(c, name="eup_abi_version")
            import :: c_int32_t
         end function

         integer(c_int32_t) function eup_device_count() bind(c, name="eup_device_count")
            import :: c_int32_t
         end function

         integer(c_int) function eup_synchronize(h) bind(c, name="eup_synchronize")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
         end function

         integer(c_int) function eup_get_stream(h, stream) bind(c, name="eup_get_stream")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            type(c_ptr)        :: stream            ! the handle's cudaStream_t
         end function

         integer(c_int) function eup_get_itime(h, itime) bind(c, name="eup_get_itime")
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: h
            integer(c_int64_t) :: itime
         end function

         integer(c_int) function eup_get_launch_count(h, launches) bind(c, name="eup_get_launch_count")
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: h
            integer(c_int64_t) :: launches
         end function

         integer(c_int) function eup_get_force_series(h, first, cnt, fxyz) bind(c, name="eup_get_force_series")
            import :: c_int, c_ptr, c_int64_t, c_int32_t, c_double
            type(c_ptr), value        :: h
            integer(c_int64_t), value :: first
            integer(c_int32_t), value :: cnt
            real(c_double)            :: fxyz(3, *)
         end function

         integer(c_int) function eup_get_links(h, links) bind(c, name="eup_get_links")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            type(c_ptr), value :: links             ! c_loc of integer(c_int32_t) links(l,m,n)
         end function

         integer(c_int) function eup_get_boundary_solid(h, list, cap, count) bind(c, name="eup_get_boundary_solid")
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value        :: h
            type(c_ptr), value        :: list       ! integer(c_int64_t) list(cap), or c_null_ptr
            integer(c_int64_t), value :: cap
            integer(c_int64_t)        :: count
         end function

         integer(c_int) function eup_get_line(h, axis, c1, c2, out) bind(c, name="eup_get_line")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: axis, c1, c2   ! prof_i/j/k: 0, 1, 2
            real(c_double)            :: out(4, *)      ! u, w, v, den per node
         end function

         integer(c_int) function eup_get_plane_means(h, axis, out) bind(c, name="eup_get_plane_means")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value        :: h
            integer(c_int32_t), value :: axis
            real(c_double)            :: out(4, *)
         end function

         integer(c_int) function eup_get_cv_drag(h, box, out) bind(c, name="eup_get_cv_drag")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t) :: box(6)            ! i1, i2, j1, j2, k1, k2
            real(c_double)     :: out(2)            ! fluxX, fluxY
         end function

         integer(c_int) function eup_save_state(h, path, elem_bytes) bind(c, name="eup_save_state")
            import :: c_int, c_ptr, c_char, c_int32_t
            type(c_ptr), value                 :: h
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int32_t), value          :: elem_bytes
         end function

         integer(c_int) function eup_restore_state(h, path, elem_bytes) bind(c, name="eup_restore_state")
            import :: c_int, c_ptr, c_char, c_int32_t
            type(c_ptr), value                 :: h
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int32_t), value          :: elem_bytes
         end function

         integer(c_int) function eup_write_obs_file(path, l, m, n, obs) bind(c, name="eup_write_obs_file")
            import :: c_int, c_char, c_int32_t, c_ptr
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int32_t), value :: l, m, n
            type(c_ptr), value        :: obs
         end function

         integer(c_int) function eup_read_raw_state(path, l, m, n, elem_bytes, pops, itime) &
                                 bind(c, name="eup_read_raw_state")
            import :: c_int, c_char, c_int32_t, c_int64_t, c_ptr
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int32_t), value :: l, m, n, elem_bytes
            type(c_ptr), intent(in)   :: pops(19)
            integer(c_int64_t)        :: itime
         end function

         integer(c_int) function eup_write_raw_state(path, l, m, n, elem_bytes, pops, itime) &
                                 bind(c, name="eup_write_raw_state")
            import :: c_int, c_char, c_int32_t, c_int64_t, c_ptr
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int32_t), value  :: l, m, n, elem_bytes
            type(c_ptr), intent(in)    :: pops(19)
            integer(c_int64_t), value  :: itime
         end function

         integer(c_int) function eup_init_equilibrium(l, m, n, u_in, amp, seed, elem_bytes, pops) &
                                 bind(c, name="eup_init_equilibrium")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            integer(c_int32_t), value :: l, m, n
            real(c_double), value     :: u_in, amp
            integer(c_int64_t), value :: seed
            integer(c_int32_t), value :: elem_bytes
            type(c_ptr), intent(in)   :: pops(19)
         end function

         integer(c_int) function eup_mem_force_noalloc(l, m, n, bc, pops, elem_bytes, obs, force, stream) &
                                 bind(c, name="eup_mem_force_noalloc")
            import :: c_int, c_int32_t, c_ptr
            integer(c_int32_t), value :: l, m, n
            integer(c_int32_t)        :: bc(6)
            type(c_ptr), intent(in)   :: pops(19)   ! device pointers (host_data use_device)
            integer(c_int32_t), value :: elem_bytes
            type(c_ptr), value        :: obs, force, stream
         end function

         integer(c_int) function eup_geometry_cylinder_z(l, m, n, xc, yc, r, obs) bind(c, name="eup_geometry_cylinder_z")
            import :: c_int, c_int32_t, c_double, c_ptr
            integer(c_int32_t), value :: l, m, n
            real(c_double), value     :: xc, yc, r
            type(c_ptr), value        :: obs
         end function

         integer(c_int) function eup_geometry_reticular_shell(l, m, n, x0, length, yc, zc, outer_d, strut_d, pitch, &
                                                               seed, obs) bind(c, name="eup_geometry_reticular_shell")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            integer(c_int32_t), value :: l, m, n
            real(c_double), value     :: x0, length, yc, zc, outer_d, strut_d, pitch
            integer(c_int64_t), value :: seed
            type(c_ptr), value        :: obs
         end function

         integer(c_int) function eup_geometry_ridged_shell(l, m, n, x0, length, yc, zc, outer_d, strut_d, pitch, &
                                                            ridge_h, ridge_t, cap_t, pore_d, smooth_w, seed, ns, &
                                                            dns_dh) bind(c, name="eup_geometry_ridged_shell")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            integer(c_int32_t), value :: l, m, n
            real(c_double), value     :: x0, length, yc, zc, outer_d, strut_d, pitch
            real(c_double), value     :: ridge_h, ridge_t, cap_t, pore_d, smooth_w
            integer(c_int64_t), value :: seed
            type(c_ptr), value        :: ns, dns_dh
         end function
      end interface

      end module eup_mod
