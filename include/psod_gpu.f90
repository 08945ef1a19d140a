! psod_gpu.f90 -- iso_c_binding interface of libpsod.so for the Fortran
! driver of sod/sod_profile_rdfof_parallel_hdf5.f90.
!
! Mirrors include/psod.h.  The driver keeps its zone loop, reader and
! writers; the four hot-path calls (cic main:673, cicm1 main:679,
! tri_cic main:713, spherover main:740) become psod_* calls on a context.
! Compile with any Fortran 2003 compiler and link -lpsod.
module psod_gpu
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: PSOD_OK = 0, PSOD_ERR_NSEL = 1, &
       PSOD_ERR_SELRADIUS = 2, PSOD_ERR_TIMEOUT = 3, PSOD_ERR_CUDA = 4, &
       PSOD_ERR_ARG = 5, PSOD_ERR_STATE = 6, PSOD_ERR_NOMEM = 7, PSOD_ERR_IO = 8
  integer(c_int), parameter :: PSOD_MODE_PLAIN = 0, PSOD_MODE_BATCHED = 1, &
       PSOD_MODE_LEARNED = 2

  type, bind(C) :: psod_params
     integer(c_int32_t) :: nx
     integer(c_int32_t) :: nmin
     real(c_double)     :: delta
     real(c_double)     :: delta2
     integer(c_int32_t) :: ncut
     integer(c_int64_t) :: nsel
     integer(c_int32_t) :: nxbuffer
     integer(c_int64_t) :: npu
     integer(c_int32_t) :: nbins
     real(c_double)     :: rbin_lo
     real(c_double)     :: rbin_hi
     integer(c_int32_t) :: ndelta_extra
     real(c_double)     :: delta_extra(4)
     integer(c_int32_t) :: mode
     integer(c_int32_t) :: device
     integer(c_int32_t) :: nxcpu
     integer(c_int32_t) :: nzone
  end type psod_params

  type, bind(C) :: psod_halo_table
     type(c_ptr) :: halo_id, halo_mass, halo_rank, halo_center, halo_rdelta
     type(c_ptr) :: halo_mass2, halo_mextra, halo_profile
     type(c_ptr) :: member_offset, member_index, member_id
  end type psod_halo_table

  type, bind(C) :: psod_run_stats
     integer(c_int64_t) :: npart_new, nprocessed, nhalo, nmember, rounds
     integer(c_int64_t) :: fail_rank, touched
     real(c_double)     :: ms_total, ms_sod_kernel
     integer(c_int64_t) :: sod_launches, kernel_launches
     real(c_double)     :: ms_sched, ms_prep, ms_refine, ms_select, ms_cross
     integer(c_int64_t) :: ncandidates, refine_pairs, cross_touch, refine_slots
     real(c_double) :: ms_setup, ms_output, ms_learn
     integer(c_int64_t) :: bracket_hits, bracket_seeds, cross_balls, cross_records
     real(c_double) :: ms_refine_bound
     integer(c_int64_t) :: refine_items, refine_pruned
     real(c_double) :: ms_tail
     integer(c_int64_t) :: tail_rounds, tail_touch, cross_members, tail_members
  end type psod_run_stats

  type, bind(C) :: psod_train_params
     integer(c_int32_t) :: epochs, batch
     real(c_float)      :: lr, beta1, beta2, eps
     integer(c_int64_t) :: seed
  end type psod_train_params

  ! scheduling thresholds of psod_spherover (no effect on any result)
  type, bind(C) :: psod_tuning
     integer(c_int32_t) :: warp_cross_min_ready, bound_min_cand, tail_max_ready, tail_max_cand
  end type psod_tuning

  ! friends-of-friends (pFoF fofpara on one rank): param%percolation_length,
  ! nres (0: cube root of the particle count), param%Mmin
  type, bind(C) :: psod_fof_params
     real(c_float)      :: percolation
     integer(c_int32_t) :: reserved
     integer(c_int64_t) :: nres, mmin
  end type psod_fof_params

  type, bind(C) :: psod_fof_stats
     integer(c_int64_t) :: nhalo, nmember, ngroups, fine_cells, pair_tests, cell_pairs
     real(c_double)     :: ms_total, ms_sort, ms_link, ms_label, ms_props
  end type psod_fof_stats

  ! haloID, haloMass, halocomPos, halocomVel, haloRadius of modhalo, and the
  ! member lists (0-based input indices and IDs)
  type, bind(C) :: psod_fof_table
     type(c_ptr) :: halo_id, halo_mass, halo_com, halo_vel, halo_radius
     type(c_ptr) :: member_offset, member_index, member_id
  end type psod_fof_table

  ! haloanalyzer's halo_properties on the SOD table or the FoF catalogue
  integer(c_int32_t), parameter :: PSOD_PROPS_FROM_SOD = 0, PSOD_PROPS_FROM_FOF = 1
  integer(c_int32_t), parameter :: PSOD_PROPS_NBIN1 = 100, PSOD_PROPS_NBIN2 = 30
  type, bind(C) :: psod_props_params
     real(c_double)     :: unit_l, unit_d, unit_t, aexp, h0, hz, delta_vir
     integer(c_int32_t) :: levelmin, center_on_mass, periodic, source, epot_threshold, reserved
  end type psod_props_params

  type, bind(C) :: psod_props_stats
     integer(c_int64_t) :: nhalo, nmember, potential_items
     real(c_double)     :: ms_total
  end type psod_props_stats

  ! haloNpart, haloMvir, haloRvir, haloRvircom, haloVvir, haloCOMX, haloCOMV,
  ! ..., the five profiles (psod.h lists the sizes per halo)
  type, bind(C) :: psod_props_table
     type(c_ptr) :: npart, mvir, rvir, rvircom, vvir, com, comv
     type(c_ptr) :: rmax, vmax, dispx, dispv, ekin, epot, lambda, lambda_prime
     type(c_ptr) :: eig_val, eig_vec, cos_alpha, center_pot, circ, delta_vals
     type(c_ptr) :: dens, dens_int, vcirc, dens178, dens_int178
  end type psod_props_table

  interface
     subroutine psod_params_default(p) bind(C, name="psod_params_default")
       import :: psod_params
       type(psod_params), intent(out) :: p
     end subroutine
     integer(c_int) function psod_ctx_create(p, ctx) bind(C, name="psod_ctx_create")
       import :: c_int, c_ptr, psod_params
       type(psod_params), intent(in) :: p
       type(c_ptr), intent(out) :: ctx
     end function
     integer(c_int) function psod_ctx_destroy(ctx) bind(C, name="psod_ctx_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function
     integer(c_int) function psod_load_particles(ctx, n, pos, vel, id, npart_total) &
          bind(C, name="psod_load_particles")
       import :: c_int, c_ptr, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: n, npart_total
       type(c_ptr), value :: pos, vel, id
     end function
     integer(c_int) function psod_cic(ctx, grid) bind(C, name="psod_cic")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx, grid
     end function
     integer(c_int) function psod_cicm1(ctx, rho) bind(C, name="psod_cicm1")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx, rho
     end function
     integer(c_int) function psod_tri_cic(ctx, isort, npart_new) bind(C, name="psod_tri_cic")
       import :: c_int, c_ptr, c_int64_t
       type(c_ptr), value :: ctx, isort
       integer(c_int64_t), intent(out) :: npart_new
     end function
     integer(c_int) function psod_spherover(ctx, stats) bind(C, name="psod_spherover")
       import :: c_int, c_ptr, psod_run_stats
       type(c_ptr), value :: ctx
       type(psod_run_stats), intent(out) :: stats
     end function
     integer(c_int) function psod_halo_count(ctx, nhalo, nmember) bind(C, name="psod_halo_count")
       import :: c_int, c_ptr, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(out) :: nhalo, nmember
     end function
     integer(c_int) function psod_get_halos(ctx, t) bind(C, name="psod_get_halos")
       import :: c_int, c_ptr, psod_halo_table
       type(c_ptr), value :: ctx
       type(psod_halo_table), intent(in) :: t
     end function
     integer(c_int) function psod_learn_collect(ctx, capacity) bind(C, name="psod_learn_collect")
       import :: c_int, c_ptr, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), value :: capacity
     end function
     integer(c_int) function psod_learn_train(ctx, tp, loss) bind(C, name="psod_learn_train")
       import :: c_int, c_ptr, psod_train_params
       type(c_ptr), value :: ctx
       type(psod_train_params), intent(in) :: tp
       type(c_ptr), value :: loss
     end function
     integer(c_int) function psod_learn_get_model(ctx, model, nfloats) bind(C, name="psod_learn_get_model")
       import :: c_int, c_ptr, c_int64_t
       type(c_ptr), value :: ctx, model
       integer(c_int64_t), value :: nfloats
     end function
     integer(c_int) function psod_learn_set_model(ctx, model, nfloats) bind(C, name="psod_learn_set_model")
       import :: c_int, c_ptr, c_int64_t
       type(c_ptr), value :: ctx, model
       integer(c_int64_t), value :: nfloats
     end function
     type(c_ptr) function psod_last_error(ctx) bind(C, name="psod_last_error")
       import :: c_ptr
       type(c_ptr), value :: ctx
     end function
     ! binary halo files of a build without HDF5 (main:2230-2259); path is a
     ! NUL-terminated character array (trim(name)//c_null_char), t a table
     ! filled into host arrays
     integer(c_int) function psod_write_masst(path, t, nhalo) bind(C, name="psod_write_masst")
       import :: c_int, c_char, c_int64_t, psod_halo_table
       character(kind=c_char), dimension(*), intent(in) :: path
       type(psod_halo_table), intent(in) :: t
       integer(c_int64_t), value :: nhalo
     end function
     integer(c_int) function psod_write_strct(path, t, nhalo, n, pos, vel, id, pot, force) &
          bind(C, name="psod_write_strct")
       import :: c_int, c_char, c_int64_t, c_ptr, psod_halo_table
       character(kind=c_char), dimension(*), intent(in) :: path
       type(psod_halo_table), intent(in) :: t
       integer(c_int64_t), value :: nhalo, n
       type(c_ptr), value :: pos, vel, id, pot, force
     end function
     ! the zone's particles from the binary cube files (main:455-534):
     ! first with pos = c_null_ptr for the count, then with posf/velf/idf
     integer(c_int) function psod_read_cube_zone(root, ncpu, nzone, nx, nxbuffer, id_bytes, capacity, &
          npart, pos, vel, id) bind(C, name="psod_read_cube_zone")
       import :: c_int, c_char, c_int32_t, c_int64_t, c_ptr
       character(kind=c_char), dimension(*), intent(in) :: root
       integer(c_int32_t), value :: ncpu, nzone, nx, nxbuffer, id_bytes
       integer(c_int64_t), value :: capacity
       integer(c_int64_t), intent(out) :: npart
       type(c_ptr), value :: pos, vel, id
     end function
     ! the driver's zone selection (main:573-600): keep(i) = 1 for the
     ! zone's particles with their buffer
     integer(c_int) function psod_select_zone(nx, nxcpu, nzone, nxbuffer, pos, n, keep, nkeep) &
          bind(C, name="psod_select_zone")
       import :: c_int, c_int32_t, c_int64_t, c_ptr
       integer(c_int32_t), value :: nx, nxcpu, nzone, nxbuffer
       type(c_ptr), value :: pos
       integer(c_int64_t), value :: n
       type(c_ptr), value :: keep
       integer(c_int64_t), intent(out) :: nkeep
     end function
     ! friends-of-friends on the loaded particles (replaces fofpara's local
     ! scan, mergehaloes, gatherhaloes, selecthaloes, computecom and
     ! computeradius for one rank)
     integer(c_int) function psod_fof(ctx, p, stats) bind(C, name="psod_fof")
       import :: c_int, c_ptr, psod_fof_params, psod_fof_stats
       type(c_ptr), value :: ctx
       type(psod_fof_params), intent(in) :: p
       type(psod_fof_stats), intent(out) :: stats
     end function
     integer(c_int) function psod_fof_halo_count(ctx, nhalo, nmember) bind(C, name="psod_fof_halo_count")
       import :: c_int, c_ptr, c_int64_t
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(out) :: nhalo, nmember
     end function
     integer(c_int) function psod_fof_get_halos(ctx, t) bind(C, name="psod_fof_get_halos")
       import :: c_int, c_ptr, psod_fof_table
       type(c_ptr), value :: ctx
       type(psod_fof_table), intent(in) :: t
     end function
     integer(c_int) function psod_autotune(ctx, chosen, ms_best, runs) bind(C, name="psod_autotune")
       import :: c_int, c_ptr, c_double, c_int32_t, psod_tuning
       type(c_ptr), value :: ctx
       type(psod_tuning), intent(out) :: chosen
       real(c_double), intent(out) :: ms_best
       integer(c_int32_t), intent(out) :: runs
     end function
     integer(c_int) function psod_set_tuning(ctx, t) bind(C, name="psod_set_tuning")
       import :: c_int, c_ptr, psod_tuning
       type(c_ptr), value :: ctx
       type(psod_tuning), intent(in) :: t
     end function
     integer(c_int) function psod_halo_properties(ctx, p, stats) bind(C, name="psod_halo_properties")
       import :: c_int, c_ptr, psod_props_params, psod_props_stats
       type(c_ptr), value :: ctx
       type(psod_props_params), intent(in) :: p
       type(psod_props_stats), intent(out) :: stats
     end function
     integer(c_int) function psod_props_get(ctx, t) bind(C, name="psod_props_get")
       import :: c_int, c_ptr, psod_props_table
       type(c_ptr), value :: ctx
       type(psod_props_table), intent(in) :: t
     end function
  end interface
end module psod_gpu
