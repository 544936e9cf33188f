! lbm_b200_iface.F90 -- Fortran 2003 ISO_C_BINDING interface to liblbmb200.so.
!
! Mirrors include/lbm_b200.h.  Every array argument is a device address passed
! by value as type(c_ptr); with nvfortran obtain it with c_devloc() from the
! cudafor module, e.g.  ierr = lbm_drift(ctx, c_devloc(f2), c_devloc(f1)).
! Return values are 0 on success or a negative LBM_ERR_* code.
!
! Each per-call function replaces the reference subroutine named beside it,
! with the arrays in the same order; dimensions and options come from the
! lbm_params given to lbm_create (the reference reads them from the modules
! mod_dimensions and m_readinfile).
module lbm_b200_iface
   use iso_c_binding
   implicit none

   integer(c_int), parameter :: LBM_OK = 0
   integer(c_int), parameter :: LBM_ERR_ARG = -1, LBM_ERR_UNSUPPORTED = -2, LBM_ERR_CUDA = -3
   integer(c_int), parameter :: LBM_ERR_STATE = -4, LBM_ERR_NUMERIC = -5, LBM_ERR_OOM = -6
   integer(c_int32_t), parameter :: LBM_STORE_F32 = 0, LBM_STORE_F16 = 1

   type, bind(C) :: lbm_params
      integer(c_int32_t) :: nx, ny, nz, nl, ibgk, ihrr, ivreman, ibnd, jbnd, kbnd, iturb_pos, storage
      real(c_float)      :: kinevisc, smagorinsky, rho0, udir
   end type

   interface
      ! ---- context ------------------------------------------------------------------
      integer(c_int) function lbm_create(ctx, p) bind(C, name="lbm_create")
         import :: c_ptr, c_int, lbm_params
         type(c_ptr), intent(out)     :: ctx
         type(lbm_params), intent(in) :: p
      end function
      integer(c_int) function lbm_destroy(ctx) bind(C, name="lbm_destroy")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx
      end function
      type(c_ptr) function lbm_last_error(ctx) bind(C, name="lbm_last_error")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function lbm_set_stream(ctx, stream) bind(C, name="lbm_set_stream")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, stream
      end function
      integer(c_int) function lbm_synchronize(ctx) bind(C, name="lbm_synchronize")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx
      end function

      ! ---- per-call entry points (reference subroutines) ---------------------------------
      ! call fequil3(feq,rho,u,v,w)                       m_fequil3.F90:4
      integer(c_int) function lbm_fequil3(ctx, feq, rho, u, v, w) bind(C, name="lbm_fequil3")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, feq, rho, u, v, w
      end function
      ! call postcoll(f,tau,rho,u,v,w)                    m_postcoll.F90:4 (ablvisc may be c_null_ptr)
      integer(c_int) function lbm_postcoll(ctx, f, tau, rho, u, v, w, ablvisc) bind(C, name="lbm_postcoll")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, tau, rho, u, v, w, ablvisc
      end function
      ! call drift(f,feq)                                 m_drift.F90:3
      integer(c_int) function lbm_drift(ctx, f, feq) bind(C, name="lbm_drift")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq
      end function
      ! call macrovars(rho,u,v,w,f)                       m_macrovars.F90:4
      integer(c_int) function lbm_macrovars(ctx, rho, u, v, w, f) bind(C, name="lbm_macrovars")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, rho, u, v, w, f
      end function
      ! call regularization(f,feq,u,v,w)                  m_regularization.F90:4
      integer(c_int) function lbm_regularization(ctx, f, feq, u, v, w) bind(C, name="lbm_regularization")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq, u, v, w
      end function
      ! call vreman(f,tau)                                m_vreman.F90:5
      integer(c_int) function lbm_vreman(ctx, f, tau) bind(C, name="lbm_vreman")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, tau
      end function
      ! call compute_fneq(f,feq)                          m_compute_fneq.F90:4
      integer(c_int) function lbm_compute_fneq(ctx, f, feq) bind(C, name="lbm_compute_fneq")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq
      end function
      ! call compute_f(f,feq)                             m_compute_f.F90:4
      integer(c_int) function lbm_compute_f(ctx, f, feq) bind(C, name="lbm_compute_f")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq
      end function
      ! call boundarycond(f1,f2,uvel,tracer,pottemp)      m_boundarycond.F90:14
      integer(c_int) function lbm_boundarycond(ctx, f1, f2, uvel) bind(C, name="lbm_boundarycond")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f1, f2, uvel
      end function
      ! call solids(f,lblanking)                          m_solids.F90:3
      integer(c_int) function lbm_solids(ctx, f, blanking) bind(C, name="lbm_solids")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, blanking
      end function
      ! call inflow_turbulence_forcing(rho,u,v,w,ampl,it,nrturb)   m_inflow_turbulence_forcing.F90:5
      integer(c_int) function lbm_inflow_turbulence_forcing(ctx, df, rho, u, v, w, uu, vv, ww, ampl, it, nrturb) &
            bind(C, name="lbm_inflow_turbulence_forcing")
         import :: c_ptr, c_int, c_float, c_int32_t
         type(c_ptr), value        :: ctx, df, rho, u, v, w, uu, vv, ww
         real(c_float), value      :: ampl
         integer(c_int32_t), value :: it, nrturb
      end function
      ! call inflow_turbulence_apply(f,turbulence_df)     m_inflow_turbulence_apply.F90:4
      integer(c_int) function lbm_inflow_turbulence_apply(ctx, f, df) bind(C, name="lbm_inflow_turbulence_apply")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, df
      end function
      ! call fillghosts(f)                                m_fillghosts.F90:4
      integer(c_int) function lbm_fillghosts(ctx, f) bind(C, name="lbm_fillghosts")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f
      end function

      ! ---- the DP build (DP=1, every real in double precision): the same calls on
      ! real(c_double) device arrays, passed as c_devloc / c_loc pointers -------------
      integer(c_int) function lbm_set_params_f64(ctx, kinevisc, smagorinsky, rho0, udir) &
            bind(C, name="lbm_set_params_f64")
         import :: c_ptr, c_int, c_double
         type(c_ptr), value    :: ctx
         real(c_double), value :: kinevisc, smagorinsky, rho0, udir
      end function
      integer(c_int) function lbm_fequil3_f64(ctx, feq, rho, u, v, w) bind(C, name="lbm_fequil3_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, feq, rho, u, v, w
      end function
      integer(c_int) function lbm_postcoll_f64(ctx, f, tau, rho, u, v, w, ablvisc) bind(C, name="lbm_postcoll_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, tau, rho, u, v, w, ablvisc
      end function
      integer(c_int) function lbm_drift_f64(ctx, f, feq) bind(C, name="lbm_drift_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq
      end function
      integer(c_int) function lbm_macrovars_f64(ctx, rho, u, v, w, f) bind(C, name="lbm_macrovars_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, rho, u, v, w, f
      end function
      integer(c_int) function lbm_regularization_f64(ctx, f, feq, u, v, w) bind(C, name="lbm_regularization_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq, u, v, w
      end function
      integer(c_int) function lbm_vreman_f64(ctx, f, tau) bind(C, name="lbm_vreman_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, tau
      end function
      integer(c_int) function lbm_compute_fneq_f64(ctx, f, feq) bind(C, name="lbm_compute_fneq_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq
      end function
      integer(c_int) function lbm_compute_f_f64(ctx, f, feq) bind(C, name="lbm_compute_f_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, feq
      end function
      integer(c_int) function lbm_boundarycond_f64(ctx, f1, f2, uvel) bind(C, name="lbm_boundarycond_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f1, f2, uvel
      end function
      integer(c_int) function lbm_forcings_apply_f64(ctx, f, external_forcing, rho, u, v, w) bind(C, name="lbm_forcings_apply_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, external_forcing, rho, u, v, w
      end function
      integer(c_int) function lbm_solids_f64(ctx, f, blanking) bind(C, name="lbm_solids_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, blanking
      end function
      integer(c_int) function lbm_inflow_turbulence_forcing_f64(ctx, df, rho, u, v, w, uu, vv, ww, ampl, it, &
            nrturb) bind(C, name="lbm_inflow_turbulence_forcing_f64")
         import :: c_ptr, c_int, c_double, c_int32_t
         type(c_ptr), value        :: ctx, df, rho, u, v, w, uu, vv, ww
         real(c_double), value     :: ampl
         integer(c_int32_t), value :: it, nrturb
      end function
      integer(c_int) function lbm_inflow_turbulence_apply_f64(ctx, f, df) bind(C, name="lbm_inflow_turbulence_apply_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, df
      end function
      integer(c_int) function lbm_fillghosts_f64(ctx, f) bind(C, name="lbm_fillghosts_f64")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f
      end function

      ! ---- fused state API ----------------------------------------------------------------
      integer(c_int) function lbm_state_import(ctx, f1, f2, rho, u, v, w, it) bind(C, name="lbm_state_import")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx, f1, f2, rho, u, v, w
         integer(c_int32_t), value :: it
      end function
      integer(c_int) function lbm_state_export(ctx, f1, f2) bind(C, name="lbm_state_export")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f1, f2
      end function
      integer(c_int) function lbm_get_macro(ctx, rho, u, v, w) bind(C, name="lbm_get_macro")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, rho, u, v, w
      end function
      integer(c_int) function lbm_set_solids(ctx, blanking) bind(C, name="lbm_set_solids")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, blanking
      end function
      integer(c_int) function lbm_set_turbulence(ctx, uu, vv, ww, nrturb, ampl) bind(C, name="lbm_set_turbulence")
         import :: c_ptr, c_int, c_float, c_int32_t
         type(c_ptr), value        :: ctx, uu, vv, ww
         integer(c_int32_t), value :: nrturb
         real(c_float), value      :: ampl
      end function
      integer(c_int) function lbm_set_inflow(ctx, uvel) bind(C, name="lbm_set_inflow")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, uvel
      end function
      integer(c_int) function lbm_step(ctx, nsteps) bind(C, name="lbm_step")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx
         integer(c_int32_t), value :: nsteps
      end function
      integer(c_int) function lbm_step_to(ctx, dst) bind(C, name="lbm_step_to")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, dst
      end function
      integer(c_int) function lbm_set_halo_j(ctx, on) bind(C, name="lbm_set_halo_j")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx
         integer(c_int32_t), value :: on
      end function
      integer(c_int) function lbm_halo_plane_bytes(ctx, bytes) bind(C, name="lbm_halo_plane_bytes")
         import :: c_ptr, c_int, c_int64_t
         type(c_ptr), value     :: ctx
         integer(c_int64_t)     :: bytes
      end function
      integer(c_int) function lbm_halo_pack_j(ctx, to_south, to_north) bind(C, name="lbm_halo_pack_j")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, to_south, to_north
      end function
      integer(c_int) function lbm_halo_unpack_j(ctx, from_south, from_north) bind(C, name="lbm_halo_unpack_j")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, from_south, from_north
      end function
      integer(c_int) function lbm_state_snapshot_bytes(ctx, bytes) bind(C, name="lbm_state_snapshot_bytes")
         import :: c_ptr, c_int, c_int64_t
         type(c_ptr), value     :: ctx
         integer(c_int64_t)     :: bytes
      end function
      integer(c_int) function lbm_state_snapshot(ctx, dst) bind(C, name="lbm_state_snapshot")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, dst
      end function
      integer(c_int) function lbm_state_restore(ctx, src) bind(C, name="lbm_state_restore")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, src
      end function
      integer(c_int) function lbm_step_host(ctx, nsteps, uvel_host, status) bind(C, name="lbm_step_host")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx, uvel_host
         integer(c_int32_t), value :: nsteps
         integer(c_int32_t)        :: status
      end function
      integer(c_int) function lbm_status(ctx, flags) bind(C, name="lbm_status")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value :: ctx
         integer(c_int32_t) :: flags
      end function
      ! call forcings_apply(f1,external_forcing,rho,u,v,w)   m_forcings_apply.F90:3
      integer(c_int) function lbm_forcings_apply(ctx, f, external_forcing, rho, u, v, w) &
            bind(C, name="lbm_forcings_apply")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, external_forcing, rho, u, v, w
      end function
      integer(c_int) function lbm_set_forcing(ctx, external_forcing) bind(C, name="lbm_set_forcing")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, external_forcing
      end function
      integer(c_int) function lbm_inflow_turbulence_compute(ctx, uu, vv, ww, rr, nrturb, seed) &
            bind(C, name="lbm_inflow_turbulence_compute")
         import :: c_ptr, c_int, c_int32_t, c_int64_t
         type(c_ptr), value        :: ctx, uu, vv, ww, rr
         integer(c_int32_t), value :: nrturb
         integer(c_int64_t), value :: seed
      end function
      integer(c_int) function lbm_set_kernel(ctx, which) bind(C, name="lbm_set_kernel")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx
         integer(c_int32_t), value :: which
      end function

      ! ---- adjoints of the per-call entry points (no reference counterpart) -------------------
      integer(c_int) function lbm_postcoll_adj(ctx, fhat, f, tau, rho, u, v, w, ablvisc, rhohat, uhat, vhat, what, &
                                               blanking) bind(C, name="lbm_postcoll_adj")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, fhat, f, tau, rho, u, v, w, ablvisc, rhohat, uhat, vhat, what, blanking
      end function
      integer(c_int) function lbm_macrovars_adj(ctx, fhat, rhohat, uhat, vhat, what, f) bind(C, name="lbm_macrovars_adj")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, fhat, rhohat, uhat, vhat, what, f
      end function
      integer(c_int) function lbm_drift_adj(ctx, fhat_in, fhat_out) bind(C, name="lbm_drift_adj")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, fhat_in, fhat_out
      end function
      integer(c_int) function lbm_macrovars_drift_adj(ctx, fhat_in, fhat_out, rhohat, uhat, vhat, what, rho, u, v, w) &
            bind(C, name="lbm_macrovars_drift_adj")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, fhat_in, fhat_out, rhohat, uhat, vhat, what, rho, u, v, w
      end function
      integer(c_int) function lbm_boundarycond_adj(ctx, f1hat, f2hat, uvelhat) bind(C, name="lbm_boundarycond_adj")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f1hat, f2hat, uvelhat
      end function

      integer(c_int) function lbm_state_bytes(ctx, bytes) bind(C, name="lbm_state_bytes")
         import :: c_ptr, c_int, c_int64_t
         type(c_ptr), value   :: ctx
         integer(c_int64_t)   :: bytes
      end function
      integer(c_int) function lbm_state_copy(ctx, dst) bind(C, name="lbm_state_copy")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, dst
      end function
      integer(c_int) function lbm_state_adjoint_step(ctx, w, a, p, pull, uvelhat) bind(C, name="lbm_state_adjoint_step")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx, w, a, p, uvelhat
         integer(c_int32_t), value :: pull
      end function
      integer(c_int) function lbm_state_adjoint_seed(ctx, a, p, probes, uhat, nprobes) &
            bind(C, name="lbm_state_adjoint_seed")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx, a, p, probes, uhat
         integer(c_int32_t), value :: nprobes
      end function
      integer(c_int) function lbm_state_adjoint_export(ctx, fhat, a) bind(C, name="lbm_state_adjoint_export")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, fhat, a
      end function

      ! ---- batched ensemble (no reference counterpart) -------------------------------------
      integer(c_int) function lbm_ensemble_create(ens, members, nmembers) bind(C, name="lbm_ensemble_create")
         import :: c_ptr, c_int, c_int32_t, lbm_params
         type(c_ptr), intent(out)        :: ens
         type(lbm_params), intent(in)    :: members(*)
         integer(c_int32_t), value       :: nmembers
      end function
      integer(c_int) function lbm_ensemble_destroy(ens) bind(C, name="lbm_ensemble_destroy")
         import :: c_ptr, c_int
         type(c_ptr), value :: ens
      end function
      integer(c_int) function lbm_ensemble_member(ens, m, ctx) bind(C, name="lbm_ensemble_member")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ens
         integer(c_int32_t), value :: m
         type(c_ptr), intent(out)  :: ctx
      end function
      integer(c_int) function lbm_ensemble_step(ens, nsteps) bind(C, name="lbm_ensemble_step")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ens
         integer(c_int32_t), value :: nsteps
      end function
      integer(c_int) function lbm_ensemble_autotune(ens, trial_steps, variant, ms_per_step) &
            bind(C, name="lbm_ensemble_autotune")
         import :: c_ptr, c_int, c_int32_t, c_float
         type(c_ptr), value        :: ens
         integer(c_int32_t), value :: trial_steps
         integer(c_int32_t)        :: variant
         real(c_float)             :: ms_per_step(*)
      end function
      integer(c_int) function lbm_ensemble_profile(ens, nsteps, step_kernel_ms, boundary_kernel_ms) &
            bind(C, name="lbm_ensemble_profile")
         import :: c_ptr, c_int, c_int32_t, c_float
         type(c_ptr), value        :: ens
         integer(c_int32_t), value :: nsteps
         real(c_float)             :: step_kernel_ms, boundary_kernel_ms
      end function
      integer(c_int) function lbm_ensemble_size(ens, nmembers) bind(C, name="lbm_ensemble_size")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value  :: ens
         integer(c_int32_t)  :: nmembers
      end function
      integer(c_int) function lbm_ensemble_set_variant(ens, variant) bind(C, name="lbm_ensemble_set_variant")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ens
         integer(c_int32_t), value :: variant
      end function
      integer(c_int) function lbm_ensemble_get_config(ens, variant, graph_steps) bind(C, name="lbm_ensemble_get_config")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ens
         integer(c_int32_t)        :: variant, graph_steps
      end function
      integer(c_int) function lbm_ensemble_variant_shape(variant, threads, min_blocks, tiles) &
            bind(C, name="lbm_ensemble_variant_shape")
         import :: c_int, c_int32_t
         integer(c_int32_t), value :: variant
         integer(c_int32_t)        :: threads, min_blocks, tiles
      end function
      integer(c_int) function lbm_ensemble_set_graph(ens, graph_steps) bind(C, name="lbm_ensemble_set_graph")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ens
         integer(c_int32_t), value :: graph_steps
      end function
      type(c_ptr) function lbm_ensemble_last_error(ens) bind(C, name="lbm_ensemble_last_error")
         import :: c_ptr
         type(c_ptr), value :: ens            ! C string (c_f_pointer to read it); c_null_ptr: the last failed create
      end function
      ! ---- conservation, step counter, instrumentation ----
      integer(c_int) function lbm_abi_version() bind(C, name="lbm_abi_version")
         import :: c_int
      end function
      integer(c_int) function lbm_get_step(ctx, it) bind(C, name="lbm_get_step")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value  :: ctx
         integer(c_int32_t)  :: it
      end function
      integer(c_int) function lbm_mass_momentum(ctx, f, out) bind(C, name="lbm_mass_momentum")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, f, out      ! out: 4 doubles on the device
      end function
      integer(c_int) function lbm_mass_momentum_noalloc(f, nx, ny, nz, nl, out, stream) &
            bind(C, name="lbm_mass_momentum_noalloc")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: f, out, stream
         integer(c_int32_t), value :: nx, ny, nz, nl
      end function
      integer(c_int) function lbm_conservation(ctx, out_host) bind(C, name="lbm_conservation")
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double)     :: out_host(4)      ! mass, x, y, z momentum of the fused state
      end function
      integer(c_int) function lbm_launch_count(ctx, n) bind(C, name="lbm_launch_count")
         import :: c_ptr, c_int, c_int64_t
         type(c_ptr), value  :: ctx
         integer(c_int64_t)  :: n
      end function
      integer(c_int) function lbm_profile(ctx, enable) bind(C, name="lbm_profile")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value        :: ctx
         integer(c_int32_t), value :: enable
      end function
      integer(c_int) function lbm_profile_read(ctx, step_kernel_ms, step_kernel_launches) &
            bind(C, name="lbm_profile_read")
         import :: c_ptr, c_int, c_int64_t, c_double
         type(c_ptr), value  :: ctx
         real(c_double)      :: step_kernel_ms
         integer(c_int64_t)  :: step_kernel_launches
      end function
      integer(c_int) function lbm_profile_read_boundary(ctx, boundary_ms, steps) &
            bind(C, name="lbm_profile_read_boundary")
         import :: c_ptr, c_int, c_int64_t, c_double
         type(c_ptr), value  :: ctx
         real(c_double)      :: boundary_ms
         integer(c_int64_t)  :: steps
      end function
   end interface
end module lbm_b200_iface
