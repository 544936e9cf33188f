/*
 * lbm_b200.h -- C ABI of the B200 (sm_100a) LBM per-timestep library.
 *
 * Two groups of entry points:
 *
 *  1. Per-call entry points with the reference's subroutine interfaces
 *     (geirev/LBM, the src/ Fortran sources).  Arrays are DEVICE pointers in the reference
 *     layout: f(nl,0:nx+1,0:ny+1,0:nz+1) column-major (l fastest), scalars
 *     (0:nx+1,0:ny+1,0:nz+1), uvel(nz), ablvisc(nz), uu/vv/ww(ny,nz,0:nrturb),
 *     turbulence_df(nl,ny,nz), lblanking logical(4).  Fortran passes arrays by
 *     reference, so each Fortran dummy array becomes one C pointer.  The
 *     caller owns every buffer.  Dimensions and options come from the context
 *     (the reference takes them from module variables).
 *
 *  2. A fused state API: the context owns a structure-of-arrays copy of the
 *     two distribution buffers and advances whole time steps with one fused
 *     kernel per step (streaming, moments, equilibrium, regularized
 *     collision, Vreman, turbulence forcing, solids) followed by the
 *     boundary-condition kernels, in the reference's step order
 *     (main.F90:288-329).
 *
 * Conventions: every entry point returns LBM_OK (0) or a negative LBM_ERR_*
 * code and never traps; lbm_last_error() gives the message.  All work is
 * stream-ordered on the context's stream (the legacy default stream unless
 * lbm_set_stream names another); entry points that return results to host
 * memory synchronise that stream.  Floating-point data is FP32, the
 * reference's default precision, except in the _f64 entry points, which take
 * the FP64 arrays of its DP build.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_B200_ABI_VERSION 1

enum {
    LBM_OK = 0,
    LBM_ERR_ARG = -1,          /* bad argument, dimension or null pointer  */
    LBM_ERR_UNSUPPORTED = -2,  /* option the library does not implement   */
    LBM_ERR_CUDA = -3,         /* CUDA runtime error                       */
    LBM_ERR_STATE = -4,        /* call out of order (e.g. step before import) */
    LBM_ERR_NUMERIC = -5,      /* NaN/Inf or non-positive density detected */
    LBM_ERR_OOM = -6           /* device allocation failed                 */
};

/* storage of the fused state */
enum {
    LBM_STORE_F32 = 0,     /* f - w_l stored in FP32                          */
    LBM_STORE_F16 = 1      /* (f - w_l) * 2^8 stored in FP16, computed in FP32 */
};

/* status bits returned by lbm_status() */
enum {
    LBM_STATUS_BAD_DENSITY = 1,  /* some cell had rho <= 0, NaN or Inf (m_rhotest.F90) */
    LBM_STATUS_TIMEOUT = 4       /* a pipeline wait in the step kernel gave up (the step is incomplete) */
};

/* steady step kernel of the fused state (lbm_set_kernel) */
enum {
    LBM_KERNEL_PULL = 1,   /* direct coalesced global loads, one cell per thread              */
    LBM_KERNEL_PAIR = 2    /* (default) two cells per thread on the packed f32x2 pipes; needs
                              ihrr=1, even nx >= 4 (other cases run LBM_KERNEL_PULL)          */
};

/* Run-time options.  Field meanings follow m_readinfile.F90:3-58 and
 * mod_dimensions.F90; values are in lattice units. */
typedef struct lbm_params {
    int32_t nx, ny, nz;     /* interior grid; ghosts add one cell per side      */
    int32_t nl;             /* 19 (D3Q19) or 27 (D3Q27)                          */
    int32_t ibgk;           /* 2 or 3: order of the Hermite equilibrium          */
    int32_t ihrr;           /* 1: regularized non-equilibrium R(fneq)            */
    int32_t ivreman;        /* 1: Vreman eddy viscosity                          */
    int32_t ibnd, jbnd, kbnd; /* 0 periodic, 1 inflow/outflow (i only), 11,12,21,22 closed */
    int32_t iturb_pos;      /* i index of the turbulence forcing slice (10)      */
    int32_t storage;        /* LBM_STORE_F32 or LBM_STORE_F16 (fused state only) */
    float kinevisc;         /* kinematic viscosity                               */
    float smagorinsky;      /* model constant; Vreman uses 2.5*smagorinsky^2     */
    float rho0;             /* reference density (1.0)                           */
    float udir;             /* inflow direction, degrees                         */
} lbm_params;

typedef struct lbm_ctx lbm_ctx;

/* ---- context --------------------------------------------------------------- */
int lbm_create(lbm_ctx** ctx, const lbm_params* p);
int lbm_destroy(lbm_ctx* ctx);
const char* lbm_last_error(const lbm_ctx* ctx);
int lbm_abi_version(void);
/* stream is a cudaStream_t for all later work of the context; NULL (the default)
 * is the legacy default stream, where the reference launches its kernels */
int lbm_set_stream(lbm_ctx* ctx, void* stream);
int lbm_synchronize(lbm_ctx* ctx);

/* ---- per-call entry points (reference interfaces) -------------------------- */

/* fequil3(feq,rho,u,v,w)           m_fequil3.F90:4; kernel m_fequil3_kernel.F90:7 */
int lbm_fequil3(lbm_ctx* ctx, float* feq, const float* rho, const float* u, const float* v, const float* w);

/* postcoll(f,tau,rho,u,v,w)        m_postcoll.F90:4; kernel m_postcoll_kernel.F90:7.
 * ablvisc(nz) replaces the module array m_mechanical_ablvisc::ablvisc (may be NULL = 0). */
int lbm_postcoll(lbm_ctx* ctx, float* f, float* tau, const float* rho, const float* u, const float* v,
                 const float* w, const float* ablvisc);

/* drift(f,feq): f = streamed feq     m_drift.F90:3; kernel m_drift_kernel.F90:7 */
int lbm_drift(lbm_ctx* ctx, float* f, const float* feq);

/* macrovars(rho,u,v,w,f)           m_macrovars.F90:4; kernel m_macrovars_kernel.F90:6 */
int lbm_macrovars(lbm_ctx* ctx, float* rho, float* u, float* v, float* w, const float* f);

/* regularization(f,feq,u,v,w): f = R(f - feq)   m_regularization.F90:4 */
int lbm_regularization(lbm_ctx* ctx, float* f, const float* feq, const float* u, const float* v, const float* w);

/* vreman(f,tau): tau from non-equilibrium f     m_vreman.F90:5 */
int lbm_vreman(lbm_ctx* ctx, const float* f, float* tau);

/* compute_fneq(f,feq): f = f - feq              m_compute_fneq.F90:4 */
int lbm_compute_fneq(lbm_ctx* ctx, float* f, const float* feq);

/* compute_f(f,feq): f = feq + f                 m_compute_f.F90:4 */
int lbm_compute_f(lbm_ctx* ctx, float* f, const float* feq);

/* boundarycond(f1,f2,uvel,...)     m_boundarycond.F90:14 (tracer/pottemp are off this path) */
int lbm_boundarycond(lbm_ctx* ctx, float* f1, float* f2, const float* uvel);

/* call forcings_apply(f1,external_forcing,rho,u,v,w)    m_forcings_apply.F90:3-64
 * external_forcing(3,0:nx+1,0:ny+1,0:nz+1): f += feq2(rho, u - F/rho) - feq2(rho, u) at
 * interior cells with rho > 0 (main.F90:306, between postcoll and solids) */
int lbm_forcings_apply(lbm_ctx* ctx, float* f, const float* external_forcing, const float* rho, const float* u,
                       const float* v, const float* w);

/* solids(f,blanking)               m_solids.F90:3; blanking is logical(4) over the ghost-inclusive grid */
int lbm_solids(lbm_ctx* ctx, float* f, const int32_t* blanking);

/* inflow_turbulence_forcing(rho,u,v,w,ampl,it,nrturb)  m_inflow_turbulence_forcing.F90:5.
 * The reference keeps turbulence_df and uu,vv,ww in module m_inflow_turbulence_init;
 * here they are explicit arguments: df(nl,ny,nz) out, uu/vv/ww(ny,nz,0:nrturb) in. */
int lbm_inflow_turbulence_forcing(lbm_ctx* ctx, float* df, const float* rho, const float* u, const float* v,
                                  const float* w, const float* uu, const float* vv, const float* ww,
                                  float ampl, int32_t it, int32_t nrturb);

/* inflow_turbulence_apply(f,turbulence_df)      m_inflow_turbulence_apply.F90:4 */
int lbm_inflow_turbulence_apply(lbm_ctx* ctx, float* f, const float* df);

/* fillghosts(f)                    m_fillghosts.F90:4 */
int lbm_fillghosts(lbm_ctx* ctx, float* f);

/* ---- per-call entry points of the DP build ----------------------------------
 * The reference built with DP=1 (src/makefile:82-86: -DDOUBLE_PRECISION with
 * -fdefault-real-8 or -r8) holds every real in double precision, tiny() and
 * eps = sqrt(tiny) included.  Each _f64 entry point takes the same arguments
 * as the entry point above it with double arrays, runs the same kernel
 * computing in FP64, and has the same error behaviour.  The context's
 * kinevisc, smagorinsky, rho0 and udir enter these as doubles converted from
 * lbm_params; lbm_set_params_f64 gives them at double precision instead
 * (the DP build reads them from its infile as real(8), m_readinfile.F90:22,129). */
int lbm_set_params_f64(lbm_ctx* ctx, double kinevisc, double smagorinsky, double rho0, double udir);
int lbm_fequil3_f64(lbm_ctx* ctx, double* feq, const double* rho, const double* u, const double* v,
                    const double* w);
int lbm_postcoll_f64(lbm_ctx* ctx, double* f, double* tau, const double* rho, const double* u, const double* v,
                     const double* w, const double* ablvisc);
int lbm_drift_f64(lbm_ctx* ctx, double* f, const double* feq);
int lbm_macrovars_f64(lbm_ctx* ctx, double* rho, double* u, double* v, double* w, const double* f);
int lbm_regularization_f64(lbm_ctx* ctx, double* f, const double* feq, const double* u, const double* v,
                           const double* w);
int lbm_vreman_f64(lbm_ctx* ctx, const double* f, double* tau);
int lbm_compute_fneq_f64(lbm_ctx* ctx, double* f, const double* feq);
int lbm_compute_f_f64(lbm_ctx* ctx, double* f, const double* feq);
int lbm_boundarycond_f64(lbm_ctx* ctx, double* f1, double* f2, const double* uvel);
int lbm_forcings_apply_f64(lbm_ctx* ctx, double* f, const double* external_forcing, const double* rho,
                           const double* u, const double* v, const double* w);
int lbm_solids_f64(lbm_ctx* ctx, double* f, const int32_t* blanking);
int lbm_inflow_turbulence_forcing_f64(lbm_ctx* ctx, double* df, const double* rho, const double* u,
                                      const double* v, const double* w, const double* uu, const double* vv,
                                      const double* ww, double ampl, int32_t it, int32_t nrturb);
int lbm_inflow_turbulence_apply_f64(lbm_ctx* ctx, double* f, const double* df);
int lbm_fillghosts_f64(lbm_ctx* ctx, double* f);

/* ---- fused state API ---------------------------------------------------------
 * The state mirrors main.F90 between time steps: f1 (pre-collision, after
 * drift), f2 (the previous post-collision buffer with its ghost cells), and
 * rho,u,v,w (the moments postcoll will use).  `it` is the number of the last
 * completed step (nt0 after initialisation). */
int lbm_state_import(lbm_ctx* ctx, const float* f1, const float* f2, const float* rho, const float* u,
                     const float* v, const float* w, int32_t it);
int lbm_state_export(lbm_ctx* ctx, float* f1, float* f2);
/* rho,u,v,w of the current state over the ghost-inclusive grid (macrovars of f1) */
int lbm_get_macro(lbm_ctx* ctx, float* rho, float* u, float* v, float* w);
/* solid mask for solids() inside the step; NULL removes it */
int lbm_set_solids(lbm_ctx* ctx, const int32_t* blanking);
/* inflow turbulence inside the step; uu == NULL disables it */
int lbm_set_turbulence(lbm_ctx* ctx, const float* uu, const float* vv, const float* ww, int32_t nrturb, float ampl);
/* inflow profile uvel(nz) (device pointer) used by boundarycond from the next step on */
int lbm_set_inflow(lbm_ctx* ctx, const float* uvel);
/* external_forcing(3,0:nx+1,0:ny+1,0:nz+1) of the fused step (main.F90:291-306), a device
 * array the caller owns and updates between steps; it is read at every step, applied after
 * the collision and before the solid swap.  NULL turns the forcing off.  It runs in the
 * two-cells-per-thread kernel: lbm_step returns LBM_ERR_UNSUPPORTED where that kernel does not
 * apply (ihrr = 0, odd nx, another lbm_set_kernel choice) and ensembles refuse forced members. */
int lbm_set_forcing(lbm_ctx* ctx, const float* external_forcing);
/* advance nsteps time steps */
int lbm_step(lbm_ctx* ctx, int32_t nsteps);
/* j-slab decomposition of one domain over several contexts (GPUs), as the
 * reference's MPI tiling (m_mpi_decomp_init.F90:123-134, m_mpi_halo_exchange_j.F90:3-121).
 * A tile is a context whose ny is the tile's rows; lbm_set_halo_j(ctx, 1), before
 * the first import, makes it keep stored j ghost planes that the caller fills
 * (the step reads them instead of wrapping j).  The boundary conditions of a
 * tile run as in the reference, tile by tile, whose periodic j copies are
 * tile-local; in the folded configuration that is the folded boundary kernel
 * wrapping j within the tile, which needs the two-cells-per-thread kernel
 * (LBM_KERNEL_PAIR, ihrr = 1, even nx >= 4).  After
 * each lbm_step the caller packs planes j = 1 and j = ny of the current state
 * (all i = 0..nx+1, k = 0..nz+1 and directions; lbm_halo_plane_bytes each),
 * sends them to the south and north neighbours, and unpacks what it receives
 * from the south into j = 0 and from the north into j = ny+1 -- the reference's
 * exchange after boundarycond and before drift (main.F90:310-318).  NULL skips a
 * plane (no neighbour).  Device buffers; plane layout [l][k][i] of the storage
 * type. */
int lbm_set_halo_j(lbm_ctx* ctx, int32_t on);
int lbm_halo_plane_bytes(lbm_ctx* ctx, int64_t* bytes);
int lbm_halo_pack_j(lbm_ctx* ctx, void* to_south, void* to_north);
int lbm_halo_unpack_j(lbm_ctx* ctx, const void* from_south, const void* from_north);

/* Snapshots of a stepped state in device memory: everything a context needs to
 * resume from that step (its state buffer, the ghost shell the next boundaries
 * read, the compact x-ghost columns and the step number).  A snapshot restores
 * into any context created with the same parameters.  lbm_state_snapshot needs
 * a state that has been stepped at least once (after an import the caller
 * holds f1, f2 already); dst and src are 256-byte aligned device memory of
 * lbm_state_snapshot_bytes bytes.  The first lbm_state_bytes bytes of a
 * snapshot are the state buffer (as lbm_state_copy). */
int lbm_state_snapshot_bytes(lbm_ctx* ctx, int64_t* bytes);
int lbm_state_snapshot(lbm_ctx* ctx, void* dst);
int lbm_state_restore(lbm_ctx* ctx, const void* src);
/* one time step whose result (the state buffer lbm_state_copy would give) is
 * written to dst, device memory of lbm_state_bytes bytes, 256-byte aligned, that
 * the caller owns, instead of to the context's other buffer.  The context reads
 * the following step from dst, so dst must stay allocated until the context has
 * stepped twice more or imported a state.  The first step after an import (a
 * collision in place) is written to the context's buffer and copied to dst.
 * Otherwise the ghost shell of the buffer the step would have overwritten is
 * copied to dst first (the boundaries read ghost values of two steps before),
 * so dst ends up holding what that buffer would.  Used to keep every state of
 * a replayed segment without copying whole buffers. */
int lbm_step_to(lbm_ctx* ctx, void* dst);
/* choose the steady step kernel (LBM_KERNEL_*); both give the same results to round-off */
int lbm_set_kernel(lbm_ctx* ctx, int32_t which);
/* host-buffer step: copies uvel(nz) from host memory before each step (NULL keeps the
 * current profile), runs nsteps steps, and writes the status word to *status_host */
int lbm_step_host(lbm_ctx* ctx, int32_t nsteps, const float* uvel_host, int32_t* status_host);
int lbm_get_step(lbm_ctx* ctx, int32_t* it);
/* accumulated LBM_STATUS_* bits since the last call; synchronises and clears them */
int lbm_status(lbm_ctx* ctx, int32_t* flags);

/* ---- conservation (FP64) ---------------------------------------------------------
 * Mass sum(rho) and momentum sum(rho u) over the interior cells, accumulated in FP64
 * (the reference prints averages of rho, u in m_diag.F90; it has no such reduction). */
/* f: reference-layout device array; out: 4 doubles (mass, mx, my, mz) in device memory */
int lbm_mass_momentum(lbm_ctx* ctx, const float* f, double* out);
/* the same for the current fused state (the reference's f1); out_host: 4 doubles, synchronises */
int lbm_conservation(lbm_ctx* ctx, double* out_host);

/* ---- allocation-free variant (no counterpart in the reference) -------------------------
 * The same sums as lbm_mass_momentum, for callers that must not allocate device memory:
 * a host program whose device memory is owned by another runtime's pool or budget (every
 * byte has to go through that allocator), a monitoring hook inside a solver loop where
 * the implicit device synchronisation of cudaMalloc/cudaFree is not acceptable, or an
 * embedder whose only allocator is a fixed arena.  It needs no context (lbm_create
 * allocates) and calls no cudaMalloc/cudaFree: the per-block
 * partial sums live in a fixed 64 KiB device array inside the library, so grids are
 * limited to 134,217,728 interior cells (nx*ny*nz); larger grids return LBM_ERR_ARG.
 * f: reference-layout device array f(nl,0:nx+1,0:ny+1,0:nz+1); out: 4 doubles
 * (mass, mx, my, mz) in device memory; stream: cudaStream_t (NULL = legacy default).
 * The first call on a device looks up the array's device address, so make that call
 * before any stream capture; the address is kept for the life of the device's context,
 * so a process that calls cudaDeviceReset cannot use this entry point afterwards.
 * Every call reuses the same array, each block overwriting its own partial before the
 * final sum reads it: calls that may overlap on the GPU (different streams, or
 * different host threads) race and must be serialised.  LBM_ERR_CUDA reports a failed
 * launch of this call (or a context already broken by earlier work); an error left
 * pending by the caller's own earlier launches is neither reported nor cleared. */
int lbm_mass_momentum_noalloc(const float* f, int32_t nx, int32_t ny, int32_t nz, int32_t nl, double* out,
                              void* stream);

/* inflow_turbulence_compute (m_inflow_turbulence_compute.F90:3-62 with the
 * Gaussian-spectrum random fields of m_pseudo2D.F90:3-169): fills uu, vv, ww and,
 * if not NULL, rr -- device arrays (ny, nz, 0:nrturb) -- with levels chained by
 * AR(1) (correlation 0.98) and normalised to zero mean and unit standard deviation
 * from level 1 on.  The random phases come from a counter-based hash of seed (the
 * reference draws them from the compiler's random_number).  Synchronises the
 * context's stream before it returns (it frees its temporaries). */
int lbm_inflow_turbulence_compute(lbm_ctx* ctx, float* uu, float* vv, float* ww, float* rr, int32_t nrturb,
                                  uint64_t seed);

/* ---- adjoint (reverse-mode) kernels of the per-call path ----
 * No counterpart in the reference, which has no gradients.  Each entry point
 * takes the adjoint (gradient of a scalar loss) of a forward call's outputs and
 * returns the adjoint of its inputs, evaluated at the forward inputs passed in;
 * chaining them in the reverse of main.F90's step order (macrovars, drift,
 * boundarycond, solids, postcoll) back-propagates through time steps.  Arrays
 * are device arrays in the reference layout, like the forward calls.  The
 * adjoint of lbm_solids is lbm_solids itself (a swap of opposite directions). */
/* postcoll: fhat holds the adjoint of postcoll's output f on entry and the adjoint
 * of its input f on exit (interior cells; ghost cells untouched); rhohat..what
 * are incremented by the adjoints of rho, u, v, w.  f, tau, rho..w, ablvisc: the
 * forward inputs (tau is read only when ivreman = 0 and may be NULL otherwise;
 * ablvisc may be NULL).  blanking (may be NULL): the adjoint of a lbm_solids call
 * that followed postcoll is applied first.  Regularized collision (ihrr = 1) only. */
int lbm_postcoll_adj(lbm_ctx* ctx, float* fhat, const float* f, const float* tau, const float* rho, const float* u,
                     const float* v, const float* w, const float* ablvisc, float* rhohat, float* uhat, float* vhat,
                     float* what, const int32_t* blanking);
/* macrovars: fhat += (d rho,u,v,w / d f)^T (rhohat, uhat, vhat, what) at the forward input f, all cells */
int lbm_macrovars_adj(lbm_ctx* ctx, float* fhat, const float* rhohat, const float* uhat, const float* vhat,
                      const float* what, const float* f);
/* drift(f_out, f_in): fhat_in += pull^T fhat_out, then the interior of fhat_out is
 * zeroed (drift overwrote it); the ghost cells of fhat_out stay (they belong to
 * the older values drift left in place) */
int lbm_drift_adj(lbm_ctx* ctx, float* fhat_in, float* fhat_out);
/* lbm_macrovars_adj on the drift's output followed by lbm_drift_adj, in one pass:
 * the macrovars adjoints (at interior cells) enter through the forward outputs
 * rho, u, v, w of that macrovars call, so the drift's output f is not read */
int lbm_macrovars_drift_adj(lbm_ctx* ctx, float* fhat_in, float* fhat_out, const float* rhohat, const float* uhat,
                            const float* vhat, const float* what, const float* rho, const float* u, const float* v,
                            const float* w);
/* boundarycond(f1, f2, uvel): the adjoint of every ghost value it wrote in f1 is
 * passed to its sources in f1hat / f2hat and, for the inflow ghosts, to uvelhat
 * (incremented; needed when ibnd = 1), then zeroed */
int lbm_boundarycond_adj(lbm_ctx* ctx, float* f1hat, float* f2hat, float* uvelhat);

/* The same reverse sweep for forward runs made with the fused step.  The adjoint
 * arrays are FP32 arrays of lbm_state_bytes bytes in the state's own layout
 * with an explicit ghost shell (zero them before use).  FP32 state storage,
 * ihrr = 1, no turbulence slice and no external forcing. */
/* bytes of one state buffer (also the size of a state-layout adjoint array) */
int lbm_state_bytes(lbm_ctx* ctx, int64_t* bytes);
/* copy the newest state buffer (after an import: the imported f1; after a step:
 * that step's post-collision populations with their ghosts) to dst */
int lbm_state_copy(lbm_ctx* ctx, void* dst);
/* one time step in reverse.  On entry W is the adjoint of f2 and A that of f1
 * after the step; on exit W is the adjoint of f1 and A that of f2 before it.
 * The interior of W is not read on entry (the interior of f2 is overwritten by
 * the next step's collision, so its adjoint is zero) and the interior of A is
 * left as it was on exit (read as zero by the next call, which takes it as W).
 * P: lbm_state_copy of the buffer the step started from -- pull = 1 when that
 * was a stepped state (the step pulled from it), 0 when it was an import.
 * uvelhat (nz) is incremented with the inflow profile's adjoint. */
int lbm_state_adjoint_step(lbm_ctx* ctx, float* W, float* A, const void* P, int32_t pull, float* uvelhat);
/* A += d(u, v, w at the probes)/df1^T uhat, with f1 = the reference's f1 after the
 * step that produced P (lbm_state_copy); probes: nprobes (i, j, k) 1-based, uhat:
 * nprobes x 3 (device arrays) */
int lbm_state_adjoint_seed(lbm_ctx* ctx, float* A, const void* P, const int32_t* probes, const float* uhat,
                           int32_t nprobes);
/* a state-layout adjoint array to the reference layout f(nl,0:nx+1,0:ny+1,0:nz+1) */
int lbm_state_adjoint_export(lbm_ctx* ctx, float* fhat, const float* A);

/* ---- batched ensemble ----
 * No counterpart in the reference, which runs one domain per process (main.F90).
 * An ensemble holds many independent members of different sizes, each an
 * ordinary context created by the ensemble: import, inflow, turbulence fields,
 * export and macro reads go through the per-member entry points above on the
 * context lbm_ensemble_member returns.  lbm_ensemble_step advances every member
 * together with two launches per step for the whole ensemble (one step kernel,
 * one boundary kernel), replayed from a CUDA graph of LBM_ENS_GRAPH_STEPS steps
 * on the ensemble's own stream; the work is ordered after earlier work on, and
 * before later work on, member 0's stream.  Members need the folded
 * configuration (ibnd = 1, jbnd = 0, kbnd in {11,12,21,22}), ihrr = 1, an even
 * nx >= 4, and one lattice and storage for all. */
typedef struct lbm_ensemble lbm_ensemble;
enum {
    LBM_ENS_VARIANTS = 8,      /* launch shapes of the step kernel: lbm_ensemble_variant_shape   */
    LBM_ENS_GRAPH_STEPS = 16   /* steps per captured graph (default; lbm_ensemble_set_graph)       */
};
int lbm_ensemble_create(lbm_ensemble** ens, const lbm_params* members, int32_t nmembers);
int lbm_ensemble_destroy(lbm_ensemble* ens);
/* with ens = NULL: why the calling thread's last lbm_ensemble_create failed */
const char* lbm_ensemble_last_error(const lbm_ensemble* ens);
int lbm_ensemble_size(const lbm_ensemble* ens, int32_t* nmembers);
/* member m's context (owned by the ensemble; do not lbm_destroy it) */
int lbm_ensemble_member(lbm_ensemble* ens, int32_t m, lbm_ctx** ctx);
/* advance every member by nsteps.  Members imported since their last step take
 * their first step alone; all members must be imported before the first call
 * and afterwards be stepped only through the ensemble. */
int lbm_ensemble_step(lbm_ensemble* ens, int32_t nsteps);
/* autotuner: time each launch shape over trial_steps steps (direct launches,
 * one warm-up step each) and keep the fastest; then time that shape over
 * LBM_ENS_GRAPH_STEPS steps replayed from a CUDA graph and as many launched
 * directly, and keep the faster (graph_steps LBM_ENS_GRAPH_STEPS or 0, as
 * lbm_ensemble_set_graph sets it).  This advances every member by
 * LBM_ENS_VARIANTS * (trial_steps + 1) + 3 * LBM_ENS_GRAPH_STEPS steps, one more
 * to bring the graphs to parity 0 where needed, plus the first step of members
 * imported since their last step.  variant and ms_per_step[LBM_ENS_VARIANTS]
 * (the shapes' times) may be NULL. */
int lbm_ensemble_autotune(lbm_ensemble* ens, int32_t trial_steps, int32_t* variant, float* ms_per_step);
int lbm_ensemble_set_variant(lbm_ensemble* ens, int32_t variant);
/* the launch shape and graph steps in use (either pointer may be NULL) */
int lbm_ensemble_get_config(const lbm_ensemble* ens, int32_t* variant, int32_t* graph_steps);
/* launch shape `variant` of the step kernel: threads per block, the minimum
 * resident blocks per SM it is compiled for (which caps its registers) and the
 * tiles of `threads` pairs each block covers (any pointer may be NULL) */
int lbm_ensemble_variant_shape(int32_t variant, int32_t* threads, int32_t* min_blocks, int32_t* tiles);
/* advance nsteps batched steps with direct launches (no graph), timing every
 * launch with CUDA events; returns the mean duration of the step kernel and of
 * the boundary kernel in ms.  Synchronises the ensemble's stream. */
int lbm_ensemble_profile(lbm_ensemble* ens, int32_t nsteps, float* step_kernel_ms, float* boundary_kernel_ms);
/* steps per captured graph: 0 = direct launches, else a positive even count */
int lbm_ensemble_set_graph(lbm_ensemble* ens, int32_t graph_steps);

/* ---- instrumentation (no counterpart in the reference, whose timers are m_wtime.F90) ---- */
/* number of kernel launches this context has issued */
int lbm_launch_count(lbm_ctx* ctx, int64_t* n);
/* enable (1) or disable (0) CUDA-event timing of every steady step: its step
 * kernel, and the boundary launches that follow it; resets the totals */
int lbm_profile(lbm_ctx* ctx, int32_t enable);
/* synchronise and return the summed device time and number of timed step-kernel launches */
int lbm_profile_read(lbm_ctx* ctx, double* step_kernel_ms, int64_t* step_kernel_launches);
/* synchronise and return the summed device time of the boundary launches of the
 * timed steps (in the folded configuration: k_bc_fold) and the number of steps */
int lbm_profile_read_boundary(lbm_ctx* ctx, double* boundary_ms, int64_t* steps);

#ifdef __cplusplus
}
#endif
#endif
